// Per-degree / per-precision entry points of the operator kernels.  Each
// (P, Number) pair is compiled in its own unit (op_p<P>_<f64|f32>.cu) so
// that the instantiations build in parallel; kernels.cu dispatches here.
#pragma once
#include "lsmf_internal.h"

namespace lsmf {

// A cell loop runs over `cells[0 .. n_list)` when `cells` is given (one
// colour of the lattice: no two listed cells share a node, so the scatter
// is a plain read-modify-write), else over all cells of the level with
// atomic scatter, or, with `cellbuf` (full vmult cell loop only), storing
// every cell's results to cellbuf[cell][local node][component] for a node
// sum that follows.
struct CellRange {
  const int *cells = nullptr;
  int n_list = 0;
  bool plain = false;
  void *cellbuf = nullptr;
  // fused interface exchange of a partitioned FP64 vmult (full cell loop,
  // atomic scatter): `peer_nodes` replaces the level's index map; its nodes
  // with PEER_BIT are the neighbour part's, gathered from peer_src / peer_u
  // and added to peer_dst (device pointers the launching device can reach)
  const int *peer_nodes = nullptr;
  const void *peer_src = nullptr;
  void *peer_dst = nullptr;
  const void *peer_u = nullptr;
  // contiguous cells first .. first + count - 1 of the level (count >= 0,
  // atomic scatter), launched on `stream` (nullptr: the operator's stream):
  // one chunk of a cell loop split over concurrent streams
  int first = 0, count = -1;
  cudaStream_t stream = nullptr;
};

struct OpsTable {
  lsmf_status (*cache)(lsmf_op *op);
  // cell loop only: dst += sum of the cell contributions (MFMask stages in
  // `mask`, internal bit MASK_INHOM_BIT: gather constrained entries)
  lsmf_status (*apply)(const lsmf_op *op, void *dst, const void *src, unsigned mask, CellRange range);
  lsmf_status (*diag)(lsmf_op *op, void *diag, CellRange range);
};

// gather constrained entries instead of zeroing them (the inhomogeneity
// term of the right-hand side)
constexpr unsigned MASK_INHOM_BIT = 1u << 8;

template <int P, typename T>
const OpsTable &ops_table();
template <> const OpsTable &ops_table<1, double>();
template <> const OpsTable &ops_table<1, float>();
template <> const OpsTable &ops_table<2, double>();
template <> const OpsTable &ops_table<2, float>();
template <> const OpsTable &ops_table<3, double>();
template <> const OpsTable &ops_table<3, float>();
template <> const OpsTable &ops_table<4, double>();
template <> const OpsTable &ops_table<4, float>();

// the partitioned vmult's cell loop with the fused interface exchange
// (kernels.cu)
lsmf_status launch_apply_peer(const lsmf_op *op, double *dst, const double *src, const CellRange &range,
                              const int *d_con, int n_con);

// the table of a level's degree and an operator's precision (nullptr for an
// unsupported degree)
inline const OpsTable *ops_for(int p, bool fp32) {
  switch (p) {
    case 1: return fp32 ? &ops_table<1, float>() : &ops_table<1, double>();
    case 2: return fp32 ? &ops_table<2, float>() : &ops_table<2, double>();
    case 3: return fp32 ? &ops_table<3, float>() : &ops_table<3, double>();
    case 4: return fp32 ? &ops_table<4, float>() : &ops_table<4, double>();
  }
  return nullptr;
}

}  // namespace lsmf
