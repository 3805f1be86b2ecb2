// Operator kernels for degree 2 (2+1 Gauss points per direction) in float.
#include "op_kernels.cuh"

namespace lsmf {
template <>
const OpsTable &ops_table<2, float>() {
  return DegreeOps<2, float>::table();
}
}  // namespace lsmf
