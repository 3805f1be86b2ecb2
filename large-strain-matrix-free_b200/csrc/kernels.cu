// Launchers of the matrix-free tangent operator (cache, vmult, diagonal,
// Jacobi) and the small element-wise kernels around the cell loops.  The
// cell-loop kernels themselves are templates in op_kernels.cuh, compiled per
// degree and precision in op_p<P>_<f64|f32>.cu and reached through
// ops_for().
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "cell_kernels.cuh"
#include "lsmf_internal.h"
#include "op_dispatch.h"

namespace lsmf {

namespace {

// ------------------------------------------------------ element-wise ops
template <typename T>
__global__ void constrained_add_kernel(T *dst, const T *src, const int *idx, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = idx[i];
    dst[k] += src[k];
  }
}
template <typename T>
__global__ void constrained_set_kernel(T *dst, const int *idx, int n, T val) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[idx[i]] = val;
}
template <typename T>
__global__ void invert_kernel(T *inv, const T *d, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    inv[i] = T(1) / d[i];
}
template <typename T>
__global__ void scaled_mul_kernel(T *dst, const T *a, const T *b, T s, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = s * a[i] * b[i];
}

int g_num_sms = 0;
int num_sms() {
  if (!g_num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

const OpsTable *table_of(const lsmf_op *op) {
  const Level &L = op->L();
  const OpsTable *t = L.q == L.p + 1 ? ops_for(L.p, op->precision == LSMF_FP32) : nullptr;
  if (!t) set_error("unsupported (degree, n_q_points_1d): only q = p + 1, p = 1..4");
  return t;
}

// node-sum scatter: dst (+)= the sum over the node's cells, in increasing
// cell order, of the node's slot in the per-cell buffer (a fixed order: the
// result is the same from call to call)
template <typename T>
__global__ void node_sum_kernel(T *dst, const T *__restrict__ buf, const int *__restrict__ off,
                                const int *__restrict__ ent, int n_nodes, int add) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < n_nodes; n += gridDim.x * blockDim.x) {
    T s0 = 0, s1 = 0, s2 = 0;
    const int e1 = __ldg(off + n + 1);
    for (int e = __ldg(off + n); e < e1; ++e) {
      const int b = __ldg(ent + e);
      s0 += buf[b];
      s1 += buf[b + 1];
      s2 += buf[b + 2];
    }
    T *d = dst + 3 * (size_t)n;
    if (add) {
      d[0] += s0; d[1] += s1; d[2] += s2;
    } else {
      d[0] = s0; d[1] = s1; d[2] = s2;
    }
  }
}

}  // namespace

// Components per quadrature point of the cell record (the record's length
// is rounded up to 16 bytes at its end, for the bulk-copy engine).
int table_components(int caching, int formulation, lsmf_precision precision) {
  (void)formulation;
  (void)precision;
  if (caching == LSMF_CACHE_TENSOR4) return variant_ncomp(VAR_TENSOR4);
  if (caching == LSMF_CACHE_TENSOR2) return variant_ncomp(VAR_TENSOR2);
  if (caching == LSMF_CACHE_SCALAR_REFERENTIAL) return variant_ncomp(VAR_SCALAR_REF);
  if (caching == LSMF_CACHE_TENSOR4_NS) return variant_ncomp(VAR_TENSOR4_NS);
  return variant_ncomp(VAR_SCALAR_F1);
}

lsmf_status launch_cache(lsmf_op *op) {
  const OpsTable *t = table_of(op);
  if (!t) return LSMF_ERR_UNSUPPORTED;
  LSMF_CUDA(cudaMemsetAsync(op->d_flag.ptr, 0, sizeof(int), op->stream));
  return t->cache(op);
}

// Run a cell loop f(range) over all cells with atomic scatter, or, with the
// colour8 scatter option, once per lattice colour in the fixed order 0..7
// (the launches are ordered on the operator's stream, so every node sums
// its cell contributions in the same order on every call).
template <typename F>
lsmf_status for_cell_ranges(const Level &L, int scatter, F &&f) {
  // the node-sum scatter serves the full vmult cell loop; every other cell
  // loop of a node-sum operator runs the (equally deterministic) colours
  if (scatter != LSMF_SCATTER_ATOMIC) {
    for (int c = 0; c < 8; ++c) {
      CellRange r;
      r.cells = L.d_colour_cells.ptr + L.colour_off[c];
      r.n_list = L.colour_off[c + 1] - L.colour_off[c];
      r.plain = true;
      if (r.n_list > 0) LSMF_TRY(f(r));
    }
    return LSMF_OK;
  }
  return f(CellRange{});
}

// the node-sum path applies: the operator asks for it and the launch is the
// full production cell loop
static bool node_sum_path(const lsmf_op *op, unsigned mask) {
  const unsigned all = LSMF_MASK_RW | LSMF_MASK_SF | LSMF_MASK_QD;
  return op->scatter == LSMF_SCATTER_NODESUM && !op->basic && (mask & all) == all && !(mask & MASK_INHOM_BIT);
}

// cell loop into the operator's cell buffer, then dst (+)= node sums
static lsmf_status apply_node_sum(const lsmf_op *op, const OpsTable *t, void *dst, const void *src, unsigned mask,
                                  bool add) {
  const Level &L = op->L();
  if (!op->d_cellbuf.ptr || !L.d_node_cell_off.ptr) {
    set_error("node-sum scatter selected without its buffers");
    return LSMF_ERR_NOT_INITIALIZED;
  }
  CellRange r;
  r.cellbuf = op->d_cellbuf.ptr;
  LSMF_TRY(t->apply(op, dst, src, mask, r));
  const int g = std::min((L.n_nodes + 255) / 256, 8 * num_sms());
  if (op->precision == LSMF_FP64)
    node_sum_kernel<double><<<g, 256, 0, op->stream>>>((double *)dst, (const double *)op->d_cellbuf.ptr,
                                                      L.d_node_cell_off.ptr, L.d_node_cell_ent.ptr, L.n_nodes, add);
  else
    node_sum_kernel<float><<<g, 256, 0, op->stream>>>((float *)dst, (const float *)op->d_cellbuf.ptr,
                                                     L.d_node_cell_off.ptr, L.d_node_cell_ent.ptr, L.n_nodes, add);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

lsmf_status set_scatter_mode(lsmf_op *op, int mode) {
  if (mode != LSMF_SCATTER_ATOMIC && mode != LSMF_SCATTER_COLOUR8 && mode != LSMF_SCATTER_NODESUM) {
    set_error("scatter must be 0 (atomic), 1 (colour8) or 2 (nodesum)");
    return LSMF_ERR_INVALID_ARG;
  }
  if (mode == LSMF_SCATTER_NODESUM) {
    Level &L = op->L();
    const int ncn = L.ncn();
    if ((double)L.n_cells * ncn * 3 > 2147483647.0) {
      set_error("the node-sum scatter indexes its cell buffer with 32-bit offsets; this level is too large");
      return LSMF_ERR_UNSUPPORTED;
    }
    if (!L.d_node_cell_off.ptr) {
      // counting sort of the (cell, local node) slots by node, cells in
      // increasing order within a node
      std::vector<int> off(L.n_nodes + 1, 0), ent((size_t)L.n_cells * ncn);
      for (size_t k = 0; k < ent.size(); ++k) ++off[L.cell_nodes[k] + 1];
      for (int n = 0; n < L.n_nodes; ++n) off[n + 1] += off[n];
      std::vector<int> pos(off.begin(), off.end() - 1);
      for (int c = 0; c < L.n_cells; ++c)
        for (int a = 0; a < ncn; ++a) ent[pos[L.cell_nodes[(size_t)c * ncn + a]]++] = (c * ncn + a) * 3;
      LSMF_TRY(L.d_node_cell_off.upload(off.data(), off.size()));
      LSMF_TRY(L.d_node_cell_ent.upload(ent.data(), ent.size()));
    }
    LSMF_TRY(op->d_cellbuf.alloc((size_t)L.n_cells * ncn * 3 * op->elem()));
  }
  op->scatter = mode;
  return LSMF_OK;
}

// Chunks of an operator's atomic-scatter cell loop: the option, or the
// measured choice.  Swept on B200 over 1 / 2 / 4 / 6 / 8 chunks for every
// variant and precision at 64^3 Q2 and for tensor4 at 32^3 / 40^3 Q2 and
// 48^3 Q3 / Q4 (vmult time against one launch): from 131,072 cells 8 for
// the referential variants (scalar_referential FP64 -7 %, tensor4_ns FP64 /
// FP32 -4 / -6 %), 2 for tensor2 (-1 / -2 %), 4 for the others (tensor4
// FP64 / FP32 -3.5 / -4 %, scalar -2 %); from 32,768 cells 2 (32^3 Q2
// tensor4 FP64 / FP32 -4.5 / -10 %, 48^3 Q3 / Q4 under -1 %); fewer cells
// run in one launch.
static int chunk_count(const lsmf_op *op) {
  if (op->chunks > 0) return op->chunks;
  const int n = op->L().n_cells;
  if (n >= 131072) {
    if (op->caching == LSMF_CACHE_TENSOR4_NS || op->caching == LSMF_CACHE_SCALAR_REFERENTIAL) return 8;
    return op->caching == LSMF_CACHE_TENSOR2 ? 2 : 4;
  }
  return n >= 32768 ? 2 : 1;
}

// The operator's plan for k chunks (*out = nullptr where it does not apply:
// k < 2, fewer than 1024 cells per chunk, or a chunk whose cells reach past
// the next chunk's node range).  Cells and nodes are numbered z-slowest, so
// contiguous cell chunks touch nearly contiguous node ranges; chunk c owns
// the nodes from the lowest one its cells touch up to the next chunk's.
static lsmf_status chunk_plan(const lsmf_op *op, int k, const ChunkPlan **out) {
  *out = nullptr;
  if (k < 2) return LSMF_OK;
  if (op->chunk_plan && op->chunk_plan->requested == k) {
    if (op->chunk_plan->k) *out = op->chunk_plan.get();
    return LSMF_OK;
  }
  auto plan = std::make_unique<ChunkPlan>();
  plan->requested = k;
  const Level &L = op->L();
  const int ncn = L.ncn();
  bool ok = k <= 8 && L.n_cells >= 1024 * k;
  if (ok) {
    plan->cell0.resize(k + 1);
    plan->node0.resize(k + 1);
    std::vector<int> nmax(k);
    for (int c = 0; c <= k; ++c) plan->cell0[c] = (int)((long long)L.n_cells * c / k);
    for (int c = 0; c < k; ++c) {
      int lo = L.n_nodes, hi = -1;
      for (size_t i = (size_t)plan->cell0[c] * ncn; i < (size_t)plan->cell0[c + 1] * ncn; ++i) {
        lo = std::min(lo, L.cell_nodes[i]);
        hi = std::max(hi, L.cell_nodes[i]);
      }
      plan->node0[c] = c == 0 ? 0 : lo;
      nmax[c] = hi;
    }
    plan->node0[k] = L.n_nodes;
    for (int c = 0; c < k && ok; ++c) {
      ok = plan->node0[c] <= plan->node0[c + 1];
      if (c + 2 <= k) ok = ok && nmax[c] < plan->node0[c + 2];
    }
  }
  if (ok) {
    for (int c = 0; c < k; ++c) {
      LSMF_CUDA(cudaStreamCreateWithFlags(&plan->stream[c], cudaStreamNonBlocking));
      LSMF_CUDA(cudaEventCreateWithFlags(&plan->zero[c], cudaEventDisableTiming));
      LSMF_CUDA(cudaEventCreateWithFlags(&plan->done[c], cudaEventDisableTiming));
    }
    LSMF_CUDA(cudaEventCreateWithFlags(&plan->fork, cudaEventDisableTiming));
    plan->k = k;
  }
  op->chunk_plan = std::move(plan);
  if (op->chunk_plan->k) *out = op->chunk_plan.get();
  return LSMF_OK;
}

// the chunked path applies: atomic scatter, fast kernels, the full cell loop
static bool chunkable(const lsmf_op *op, unsigned mask) {
  const unsigned all = LSMF_MASK_RW | LSMF_MASK_SF | LSMF_MASK_QD;
  return op->scatter == LSMF_SCATTER_ATOMIC && !op->basic && (mask & all) == all && !(mask & MASK_INHOM_BIT);
}

// chunks the operator's next full vmult cell loop runs in (1: one launch)
lsmf_status effective_chunks(const lsmf_op *op, int *k) {
  *k = 1;
  if (!chunkable(op, LSMF_MASK_RW | LSMF_MASK_SF | LSMF_MASK_QD)) return LSMF_OK;
  const ChunkPlan *cp = nullptr;
  LSMF_TRY(chunk_plan(op, chunk_count(op), &cp));
  if (cp) *k = cp->k;
  return LSMF_OK;
}


// The vmult over the plan's chunks, forked from and joined back into the
// operator's stream: chunk c zeroes its node range of dst (zero) and adds
// the identity rows of the constrained dofs in it (rows), then runs its
// cells once chunk c + 1 has zeroed its range (its cells add into that
// range's first node layer).  The scatter skips constrained components, so
// the identity rows are never touched by another chunk.
static lsmf_status apply_chunked(const lsmf_op *op, const OpsTable *t, const ChunkPlan &cp, void *dst,
                                 const void *src, unsigned mask, bool zero, bool rows) {
  const Level &L = op->L();
  const size_t e = op->elem();
  const int g_max = 4 * num_sms();
  LSMF_CUDA(cudaEventRecord(cp.fork, op->stream));
  for (int c = 0; c < cp.k; ++c) {
    cudaStream_t st = cp.stream[c];
    LSMF_CUDA(cudaStreamWaitEvent(st, cp.fork, 0));
    const size_t d0 = 3 * (size_t)cp.node0[c], d1 = 3 * (size_t)cp.node0[c + 1];
    if (zero && d1 > d0) LSMF_CUDA(cudaMemsetAsync((char *)dst + d0 * e, 0, (d1 - d0) * e, st));
    if (rows) {
      // L.constrained is in increasing dof order
      const int a0 = (int)(std::lower_bound(L.constrained.begin(), L.constrained.end(), (int)d0) - L.constrained.begin());
      const int a1 = (int)(std::lower_bound(L.constrained.begin(), L.constrained.end(), (int)d1) - L.constrained.begin());
      const int nc = a1 - a0;
      if (nc > 0) {
        const int g = (nc + 255) / 256 < g_max ? (nc + 255) / 256 : g_max;
        if (op->precision == LSMF_FP64)
          constrained_add_kernel<double><<<g, 256, 0, st>>>((double *)dst, (const double *)src, L.d_constrained.ptr + a0, nc);
        else
          constrained_add_kernel<float><<<g, 256, 0, st>>>((float *)dst, (const float *)src, L.d_constrained.ptr + a0, nc);
        LSMF_CUDA(cudaGetLastError());
      }
    }
    LSMF_CUDA(cudaEventRecord(cp.zero[c], st));
  }
  for (int c = 0; c < cp.k; ++c) {
    if (c + 1 < cp.k) LSMF_CUDA(cudaStreamWaitEvent(cp.stream[c], cp.zero[c + 1], 0));
    CellRange r;
    r.first = cp.cell0[c];
    r.count = cp.cell0[c + 1] - cp.cell0[c];
    r.stream = cp.stream[c];
    LSMF_TRY(t->apply(op, dst, src, mask, r));
    LSMF_CUDA(cudaEventRecord(cp.done[c], cp.stream[c]));
  }
  for (int c = 0; c < cp.k; ++c) LSMF_CUDA(cudaStreamWaitEvent(op->stream, cp.done[c], 0));
  return LSMF_OK;
}

lsmf_status launch_apply(const lsmf_op *op, void *dst, const void *src, unsigned mask, bool add) {
  const Level &L = op->L();
  const OpsTable *t = table_of(op);
  if (!t) return LSMF_ERR_UNSUPPORTED;
  const size_t n = (size_t)L.n_dofs();
  if (node_sum_path(op, mask)) {
    LSMF_TRY(apply_node_sum(op, t, dst, src, mask, add || !(mask & LSMF_MASK_ZERO)));
  } else {
    if (chunkable(op, mask)) {
      const ChunkPlan *cp = nullptr;
      LSMF_TRY(chunk_plan(op, chunk_count(op), &cp));
      if (cp) return apply_chunked(op, t, *cp, dst, src, mask, !add && (mask & LSMF_MASK_ZERO), true);
    }
    if (!add && (mask & LSMF_MASK_ZERO)) LSMF_CUDA(cudaMemsetAsync(dst, 0, n * op->elem(), op->stream));
    LSMF_TRY(for_cell_ranges(L, op->scatter, [&](CellRange r) { return t->apply(op, dst, src, mask, r); }));
  }
  // constrained rows: dst += src (mf_nh_operator.h:702-705)
  const int nc = (int)L.constrained.size();
  if (nc && (mask & LSMF_MASK_RW)) {
    const int g = (nc + 255) / 256 < 4 * num_sms() ? (nc + 255) / 256 : 4 * num_sms();
    if (op->precision == LSMF_FP64)
      constrained_add_kernel<double><<<g, 256, 0, op->stream>>>((double *)dst, (const double *)src, L.d_constrained.ptr, nc);
    else
      constrained_add_kernel<float><<<g, 256, 0, op->stream>>>((float *)dst, (const float *)src, L.d_constrained.ptr, nc);
    LSMF_CUDA(cudaGetLastError());
  }
  return LSMF_OK;
}

// Cell loop of a partitioned FP64 vmult with the interface exchange fused
// in (range.peer_*: the ghost nodes' values are read from, and their
// contributions added to, the neighbour part's vectors), then the identity
// rows of the part's owned constrained dofs d_con[0 .. n_con).  dst is not
// zeroed here: the caller orders the zeroing of this part's and of the
// neighbour's dst before the launch.
lsmf_status launch_apply_peer(const lsmf_op *op, double *dst, const double *src, const CellRange &range,
                              const int *d_con, int n_con) {
  const OpsTable *t = table_of(op);
  if (!t) return LSMF_ERR_UNSUPPORTED;
  if (op->precision != LSMF_FP64 || op->basic || op->scatter != LSMF_SCATTER_ATOMIC || !range.peer_nodes) {
    set_error("the fused interface exchange needs an FP64 operator with the fast kernel and atomic scatter");
    return LSMF_ERR_INVALID_ARG;
  }
  LSMF_TRY(t->apply(op, dst, src, LSMF_MASK_RW | LSMF_MASK_SF | LSMF_MASK_QD, range));
  if (n_con) {
    const int g = (n_con + 255) / 256 < 4 * num_sms() ? (n_con + 255) / 256 : 4 * num_sms();
    constrained_add_kernel<double><<<g, 256, 0, op->stream>>>(dst, src, d_con, n_con);
    LSMF_CUDA(cudaGetLastError());
  }
  return LSMF_OK;
}

lsmf_status launch_apply_cells(const lsmf_op *op, void *dst, const void *src) {
  const OpsTable *t = table_of(op);
  if (!t) return LSMF_ERR_UNSUPPORTED;
  const unsigned mask = LSMF_MASK_RW | LSMF_MASK_SF | LSMF_MASK_QD;
  if (node_sum_path(op, mask)) return apply_node_sum(op, t, dst, src, mask, true);
  if (chunkable(op, mask)) {
    // the chunks' cell loops only, concurrent (nothing to zero)
    const ChunkPlan *cp = nullptr;
    LSMF_TRY(chunk_plan(op, chunk_count(op), &cp));
    if (cp) {
      LSMF_CUDA(cudaEventRecord(cp->fork, op->stream));
      for (int c = 0; c < cp->k; ++c) {
        LSMF_CUDA(cudaStreamWaitEvent(cp->stream[c], cp->fork, 0));
        CellRange r;
        r.first = cp->cell0[c];
        r.count = cp->cell0[c + 1] - cp->cell0[c];
        r.stream = cp->stream[c];
        LSMF_TRY(t->apply(op, dst, src, mask, r));
        LSMF_CUDA(cudaEventRecord(cp->done[c], cp->stream[c]));
      }
      for (int c = 0; c < cp->k; ++c) LSMF_CUDA(cudaStreamWaitEvent(op->stream, cp->done[c], 0));
      return LSMF_OK;
    }
  }
  return for_cell_ranges(op->L(), op->scatter, [&](CellRange r) { return t->apply(op, dst, src, mask, r); });
}

// K g over the constrained columns: gather without zeroing, scatter skipping
// constrained rows (dst zeroed first, no identity rows)
lsmf_status launch_apply_inhomogeneous(const lsmf_op *op, void *dst, const void *g) {
  const Level &L = op->L();
  const OpsTable *t = table_of(op);
  if (!t) return LSMF_ERR_UNSUPPORTED;
  LSMF_CUDA(cudaMemsetAsync(dst, 0, (size_t)L.n_dofs() * op->elem(), op->stream));
  const unsigned mask = LSMF_MASK_RW | LSMF_MASK_SF | LSMF_MASK_QD | MASK_INHOM_BIT;
  return for_cell_ranges(L, op->scatter, [&](CellRange r) { return t->apply(op, dst, g, mask, r); });
}

lsmf_status launch_diagonal(lsmf_op *op) {
  const Level &L = op->L();
  const OpsTable *t = table_of(op);
  if (!t) return LSMF_ERR_UNSUPPORTED;
  const size_t n = (size_t)L.n_dofs();
  LSMF_CUDA(cudaMemsetAsync(op->d_diag.ptr, 0, n * op->elem(), op->stream));
  LSMF_TRY(for_cell_ranges(L, op->scatter, [&](CellRange r) { return t->diag(op, op->d_diag.ptr, r); }));
  const int nc = (int)L.constrained.size();
  const int g = 4 * num_sms();
  if (op->precision == LSMF_FP64) {
    if (nc) constrained_set_kernel<double><<<g, 256, 0, op->stream>>>((double *)op->d_diag.ptr, L.d_constrained.ptr, nc, 1.0);
    invert_kernel<double><<<g, 256, 0, op->stream>>>((double *)op->d_inv_diag.ptr, (const double *)op->d_diag.ptr, n);
  } else {
    if (nc) constrained_set_kernel<float><<<g, 256, 0, op->stream>>>((float *)op->d_diag.ptr, L.d_constrained.ptr, nc, 1.0f);
    invert_kernel<float><<<g, 256, 0, op->stream>>>((float *)op->d_inv_diag.ptr, (const float *)op->d_diag.ptr, n);
  }
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

lsmf_status launch_jacobi(const lsmf_op *op, void *dst, const void *src, double omega) {
  const size_t n = (size_t)op->L().n_dofs();
  const int g = 4 * num_sms();
  if (op->precision == LSMF_FP64)
    scaled_mul_kernel<double><<<g, 256, 0, op->stream>>>((double *)dst, (const double *)op->d_inv_diag.ptr,
                                                         (const double *)src, omega, n);
  else
    scaled_mul_kernel<float><<<g, 256, 0, op->stream>>>((float *)dst, (const float *)op->d_inv_diag.ptr,
                                                        (const float *)src, (float)omega, n);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

}  // namespace lsmf
