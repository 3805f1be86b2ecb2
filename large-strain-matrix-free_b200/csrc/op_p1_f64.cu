// Operator kernels for degree 1 (1+1 Gauss points per direction) in double.
#include "op_kernels.cuh"

namespace lsmf {
template <>
const OpsTable &ops_table<1, double>() {
  return DegreeOps<1, double>::table();
}
}  // namespace lsmf
