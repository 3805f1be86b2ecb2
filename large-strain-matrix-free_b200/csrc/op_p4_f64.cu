// Operator kernels for degree 4 (4+1 Gauss points per direction) in double.
#include "op_kernels.cuh"

namespace lsmf {
template <>
const OpsTable &ops_table<4, double>() {
  return DegreeOps<4, double>::table();
}
}  // namespace lsmf
