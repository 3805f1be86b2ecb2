// Operator kernels for degree 2 (2+1 Gauss points per direction) in double.
#include "op_kernels.cuh"

namespace lsmf {
template <>
const OpsTable &ops_table<2, double>() {
  return DegreeOps<2, double>::table();
}
}  // namespace lsmf
