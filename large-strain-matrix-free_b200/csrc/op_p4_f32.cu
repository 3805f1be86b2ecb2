// Operator kernels for degree 4 (4+1 Gauss points per direction) in float.
#include "op_kernels.cuh"

namespace lsmf {
template <>
const OpsTable &ops_table<4, float>() {
  return DegreeOps<4, float>::table();
}
}  // namespace lsmf
