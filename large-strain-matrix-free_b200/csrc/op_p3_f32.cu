// Operator kernels for degree 3 (3+1 Gauss points per direction) in float.
#include "op_kernels.cuh"

namespace lsmf {
template <>
const OpsTable &ops_table<3, float>() {
  return DegreeOps<3, float>::table();
}
}  // namespace lsmf
