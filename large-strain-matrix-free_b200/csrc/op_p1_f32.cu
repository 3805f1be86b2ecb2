// Operator kernels for degree 1 (1+1 Gauss points per direction) in float.
#include "op_kernels.cuh"

namespace lsmf {
template <>
const OpsTable &ops_table<1, float>() {
  return DegreeOps<1, float>::table();
}
}  // namespace lsmf
