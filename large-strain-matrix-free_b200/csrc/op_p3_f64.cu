// Operator kernels for degree 3 (3+1 Gauss points per direction) in double.
#include "op_kernels.cuh"

namespace lsmf {
template <>
const OpsTable &ops_table<3, double>() {
  return DegreeOps<3, double>::table();
}
}  // namespace lsmf
