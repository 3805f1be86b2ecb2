// Internal data model of liblsmf: host-side mesh hierarchy, device buffers,
// operator state.  Device layouts (HBM):
//   cell_nodes  int32 [n_cells][(p+1)^3], node id | (constrained comps << 29)
//   X           double [n_nodes][3] reference node coordinates
//   vectors     Number [n_nodes][3] (dof = 3*node + comp)
//   cache table Number [n_cells][n_comp][Q^3] (one contiguous record per cell)
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/lsmf.h"

namespace lsmf {

void set_error(const std::string &msg);

#define LSMF_CUDA(...)                                                            \
  do {                                                                            \
    cudaError_t e_ = (__VA_ARGS__);                                               \
    if (e_ != cudaSuccess) {                                                      \
      ::lsmf::set_error(std::string(#__VA_ARGS__) + ": " + cudaGetErrorString(e_)); \
      return LSMF_ERR_CUDA;                                                       \
    }                                                                             \
  } while (0)
#define LSMF_TRY(...)                        \
  do {                                       \
    lsmf_status s_ = (__VA_ARGS__);          \
    if (s_ != LSMF_OK) return s_;            \
  } while (0)

constexpr int NODE_BITS = 29;
constexpr int NODE_MASK = (1 << NODE_BITS) - 1;
// index maps of a partitioned operator's fused interface exchange: a node
// with PEER_BIT set is the neighbour part's node PEER_BIT ^ id (its vectors
// are read and added to directly); nodes stay below PEER_BIT
constexpr int PEER_BIT = 1 << (NODE_BITS - 1);
constexpr int PEER_NODE_MASK = PEER_BIT - 1;

// 1D Lagrange basis on Gauss-Lobatto nodes at Gauss points on [0,1].
struct Basis {
  int p = 0, q = 0;
  std::vector<double> nodes, qpts, qw, N, D;  // N, D: [q][p+1]
  std::vector<double> Dc;  // [q][q]: derivative of the Lagrange basis on the points, at the points
  void init(int p, int q);
  void eval(double x, double *val, double *der) const;
};

// LSMF_POISON_ALLOC set (any value) in the environment: every new device
// buffer of floating-point values (and the byte buffers that hold them:
// records, level vectors, diagonals) is filled with 0xFF bytes, a NaN in
// FP32 and FP64, so that a value read before it is written shows up as a
// NaN instead of whatever the allocator hands back.  Index and mask buffers
// are left alone.  Read at every allocation, so a process can switch it.
inline bool poison_alloc() { return std::getenv("LSMF_POISON_ALLOC") != nullptr; }

template <typename T>
struct DevBuf {
  T *ptr = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : ptr(o.ptr), n(o.n) { o.ptr = nullptr; o.n = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept {
    if (this != &o) { release(); ptr = o.ptr; n = o.n; o.ptr = nullptr; o.n = 0; }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr; n = 0;
  }
  lsmf_status alloc(size_t count) {
    if (count == n && ptr) return LSMF_OK;
    release();
    if (count == 0) return LSMF_OK;
    cudaError_t e = cudaMalloc((void **)&ptr, count * sizeof(T));
    if (e != cudaSuccess) {
      ptr = nullptr;
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return LSMF_ERR_ALLOC;
    }
    n = count;
    if constexpr (std::is_floating_point<T>::value || std::is_same<T, char>::value) {
      if (poison_alloc()) {
        e = cudaMemset(ptr, 0xFF, count * sizeof(T));
        if (e == cudaSuccess) e = cudaDeviceSynchronize();  // ordered before every stream's work
        if (e != cudaSuccess) { set_error(std::string("cudaMemset: ") + cudaGetErrorString(e)); return LSMF_ERR_CUDA; }
      }
    }
    return LSMF_OK;
  }
  lsmf_status upload(const T *h, size_t count) {
    LSMF_TRY(alloc(count));
    if (count) LSMF_CUDA(cudaMemcpy(ptr, h, count * sizeof(T), cudaMemcpyHostToDevice));
    return LSMF_OK;
  }
};

// One level of the structured hierarchy.
struct Level {
  int p = 2, q = 3;
  int nc[3] = {0, 0, 0}, nn[3] = {0, 0, 0};
  int n_cells = 0, n_nodes = 0;
  bool affine = false;          // every cell an affine image of the unit cube (box meshes)
  std::vector<int> lattice_to_node, node_lattice, cell_of_lattice;
  std::vector<double> X;
  std::vector<int> cell_nodes;  // raw node ids
  std::vector<int> cell_ijk;
  std::vector<int> bfaces;      // (cell, face, id)
  std::vector<uint8_t> cmask;   // per dof
  std::vector<int> constrained;
  // cells grouped by lattice colour (i&1) + 2 (j&1) + 4 (k&1): cells of one
  // colour share no node; colour c is colour_cells[colour_off[c] ..
  // colour_off[c+1])
  std::vector<int> colour_cells;
  int colour_off[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  DevBuf<int> d_colour_cells;
  // node -> its cells, for the node-sum scatter (built on first use): the
  // entries of node n are node_cell_off[n] .. node_cell_off[n+1], each the
  // offset (cell * ncn + local node) * 3 of the node's slot in a per-cell
  // buffer [cell][local node][component], in increasing cell order
  DevBuf<int> d_node_cell_off, d_node_cell_ent;
  // device
  DevBuf<int> d_cell_nodes;     // packed with constraint bits
  DevBuf<double> d_X;
  DevBuf<int> d_constrained;
  DevBuf<uint8_t> d_cmask;      // per dof constrained flag
  int ncn() const { return (p + 1) * (p + 1) * (p + 1); }
  int nq() const { return q * q * q; }
  int n_dofs() const { return 3 * n_nodes; }
};

// Cell-wise transfer from level l-1 to level l.
struct TransferMap {
  std::vector<int> fine_nodes;   // per coarse cell (2p+1)^3
  std::vector<double> weight;    // per fine node
  std::vector<double> P1;        // (2p+1) x (p+1)
  DevBuf<int> d_fine_nodes;
  DevBuf<double> d_weight;
  // interpolation of the fine displacement onto the coarse nodes
  std::vector<int> interp_fine_cell;   // per coarse node: fine cell
  std::vector<double> interp_xi;       // per coarse node: 3 local coords in that fine cell
  DevBuf<int> d_interp_cell;
  DevBuf<double> d_interp_w;           // per coarse node: (p+1)^3 weights
};

// Layout of one z-slab partition of the finest level: the part owns the
// coarse cells with k in [k0, k1) (all their refinements).  Local nodes are
// numbered in lattice order like the whole mesh, so both parts of an
// interface list its shared nodes in the same (global) order.  The shared
// nodes of an interface plane are owned by the upper part: upper_shared are
// this part's ghosts (their values live on part + 1), lower_shared are owned
// here and are ghosts of part - 1.
struct PartLayout {
  int n_parts = 1, part = 0, k0 = 0, k1 = 0;
  std::vector<int> global_node;   // local node -> node of the whole mesh
  std::vector<int> lower_shared;  // local nodes shared with part - 1
  std::vector<int> upper_shared;  // local nodes shared with part + 1
  int n_global_nodes = 0;
};

}  // namespace lsmf

struct lsmf_mesh {
  lsmf_mesh_desc desc{};
  std::vector<uint8_t> coarse_active;
  // z-slab partition (n_parts == 1: the whole mesh)
  lsmf::PartLayout layout;
  // build the host-side levels and layout only (no device buffers, no
  // constraints or transfers): the partition query needs no GPU
  bool host_only = false;
  lsmf::Basis basis;
  std::vector<lsmf::Level *> levels;          // 0 = coarsest
  std::vector<lsmf::TransferMap *> transfer;  // transfer[l] : l-1 -> l (l>=1)
  std::vector<int> dir_ids, dir_masks;
  ~lsmf_mesh();
};

namespace lsmf {
// The vmult cell loop of a large level split into k contiguous cell chunks
// on concurrent streams (kernels.cu).  Chunk c zeroes the dst node range
// node0[c] .. node0[c+1] (every node its cells touch lies in its own or the
// next chunk's range), applies the identity rows of the constrained dofs
// there, then runs its cell loop once chunk c + 1 has zeroed its range.
struct ChunkPlan {
  int requested = 0;                 // chunk count asked for
  int k = 0;                         // 0: the plan does not apply to this level
  std::vector<int> cell0, node0;     // k + 1 offsets
  cudaStream_t stream[8] = {};
  cudaEvent_t fork = nullptr, zero[8] = {}, done[8] = {};
  ~ChunkPlan() {
    for (int c = 0; c < 8; ++c) {
      if (stream[c]) cudaStreamDestroy(stream[c]);
      if (zero[c]) cudaEventDestroy(zero[c]);
      if (done[c]) cudaEventDestroy(done[c]);
    }
    if (fork) cudaEventDestroy(fork);
  }
};
}  // namespace lsmf

struct lsmf_op {
  lsmf_mesh *mesh = nullptr;
  int level = 0;
  int caching = LSMF_CACHE_TENSOR4, formulation = 1;
  lsmf_precision precision = LSMF_FP64;
  int ncomp = 0;                     // table components per qp
  int rec_elems = 0;                 // values per cell record (ncomp * nq, plus per-cell values and padding)
  bool ref_per_cell = false;         // scalar caching on affine cells: reference metric once per cell
  double nu = 0.3;
  std::vector<double> mu_host;
  lsmf::DevBuf<double> d_mu;         // per cell
  lsmf::DevBuf<char> d_table;        // [cell][ncomp][nq] of Number
  lsmf::DevBuf<char> d_diag, d_inv_diag;
  lsmf::DevBuf<int> d_flag;          // device error word
  const void *d_u = nullptr;         // borrowed displacement
  bool cached = false, have_diag = false;
  int stages = -1;                   // bulk-copy (TMA) ring depth of the vmult kernel (0 = plain loads, -1 auto)
  bool basic = false;                // use the basic (smem-sweep) vmult kernel
  int max_warps = 0;                 // warps per block cap of the vmult kernel (<= 8, 0 auto)
  int wait_tries = -1;               // bulk-copy wait bound (try_wait calls; -1 = default 2^22)
  int prefetch = -1;                 // plain-load kernels: L1 prefetch of the record (0, 1 this cell, 2 next; -1 auto)
  int pairs = -1;                    // FP32 vmult: two cells per warp in packed f32x2 arithmetic (0 off, 1 on, -1 auto)
  int device = 0;                    // CUDA device the operator's buffers live on
  int scatter = LSMF_SCATTER_ATOMIC; // cell-loop scatter: atomics, the 8 colour launches, or node sums
  lsmf::DevBuf<char> d_cellbuf;      // node-sum scatter: per-cell results [cell][local node][component]
  // concurrent chunks of the atomic-scatter vmult cell loop (-1 auto, 1 off,
  // 2..8); the plan for the chosen count is built on first use
  int chunks = -1;
  mutable std::unique_ptr<lsmf::ChunkPlan> chunk_plan;
  cudaStream_t stream = 0;
  // CG workspace (outer FP64 CG driven through this operator)
  lsmf::DevBuf<double> cg_g, cg_h, cg_d, sc, partial;
  size_t elem() const { return precision == LSMF_FP64 ? 8 : 4; }
  lsmf::Level &L() const { return *mesh->levels[level]; }
};

namespace lsmf {
// kernels.cu launchers
lsmf_status launch_cache(lsmf_op *op);
lsmf_status launch_apply(const lsmf_op *op, void *dst, const void *src, unsigned mask, bool add);
// only the cell loop: dst += sum of cell contributions (no zeroing, no
// identity rows); callers fold those into their own element-wise kernels
lsmf_status launch_apply_cells(const lsmf_op *op, void *dst, const void *src);
lsmf_status launch_diagonal(lsmf_op *op);
// select the cell-loop scatter of an operator (LSMF_SCATTER_*); the
// node-sum mode builds the level's node -> cell lists and the operator's
// cell buffer on first use
lsmf_status set_scatter_mode(lsmf_op *op, int mode);
// chunks the operator's next full vmult cell loop runs in (1: one launch)
lsmf_status effective_chunks(const lsmf_op *op, int *k);
lsmf_status upload_basis_tables(const Basis &b);
int table_components(int caching, int formulation, lsmf_precision precision);
}  // namespace lsmf
