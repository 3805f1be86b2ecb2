// C ABI: status strings, mesh and operator entry points (include/lsmf.h).
#include <cstring>
#include <new>
#include <string>

#include "lsmf_internal.h"

namespace lsmf {
namespace {
thread_local std::string g_last_error;
}
void set_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }
lsmf_status build_mesh(lsmf_mesh &M);
lsmf_status level_constraints(const lsmf_mesh &M, Level &L);
lsmf_status launch_jacobi(const lsmf_op *op, void *dst, const void *src, double omega);
}  // namespace lsmf

using namespace lsmf;

extern "C" {

const char *lsmf_status_string(lsmf_status s) {
  switch (s) {
    case LSMF_OK: return "ok";
    case LSMF_ERR_INVALID_ARG: return "invalid argument";
    case LSMF_ERR_UNKNOWN_CACHING: return "Unknown caching";
    case LSMF_ERR_DETF_NONPOSITIVE: return "det_F is not positive";
    case LSMF_ERR_NOT_INITIALIZED: return "not initialized";
    case LSMF_ERR_CG_NOT_CONVERGED: return "CG did not converge";
    case LSMF_ERR_NEWTON_NOT_CONVERGED: return "No convergence in nonlinear solver!";
    case LSMF_ERR_CUDA: return "CUDA error";
    case LSMF_ERR_TIMEOUT: return "device wait timed out";
    case LSMF_ERR_PRM: return "parameter file error";
    case LSMF_ERR_UNSUPPORTED: return "unsupported configuration";
    case LSMF_ERR_ALLOC: return "device allocation failed";
  }
  return "unknown status";
}

const char *lsmf_last_error(void) { return last_error(); }
const char *lsmf_version(void) { return "lsmf 0.1 (sm_100a)"; }

lsmf_status lsmf_mesh_create(const lsmf_mesh_desc *desc, lsmf_mesh **out) {
  if (!desc || !out) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  *out = nullptr;
  lsmf_mesh *m = new (std::nothrow) lsmf_mesh();
  if (!m) return LSMF_ERR_ALLOC;
  m->desc = *desc;
  if (desc->coarse_active) {
    const size_t n = (size_t)desc->coarse[0] * desc->coarse[1] * desc->coarse[2];
    m->coarse_active.assign(desc->coarse_active, desc->coarse_active + n);
  }
  m->desc.coarse_active = nullptr;
  lsmf_status s = build_mesh(*m);
  if (s != LSMF_OK) { delete m; return s; }
  *out = m;
  return LSMF_OK;
}

// the coarse z-cells [k0, k1) of part `part` of n_parts: as even as possible
static void slab_range(int nz, int n_parts, int part, int &k0, int &k1) {
  k0 = (int)((long long)nz * part / n_parts);
  k1 = (int)((long long)nz * (part + 1) / n_parts);
}

static lsmf_status make_part_mesh(const lsmf_mesh_desc *desc, int n_parts, int part, bool host_only, lsmf_mesh **out) {
  if (!desc || !out) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  *out = nullptr;
  if (n_parts < 1 || part < 0 || part >= n_parts) { set_error("bad part / n_parts"); return LSMF_ERR_INVALID_ARG; }
  if (desc->coarse[2] < n_parts) {
    set_error("a partition needs at least one coarse cell layer in z per part");
    return LSMF_ERR_INVALID_ARG;
  }
  lsmf_mesh *m = new (std::nothrow) lsmf_mesh();
  if (!m) return LSMF_ERR_ALLOC;
  m->desc = *desc;
  if (desc->coarse_active) {
    const size_t n = (size_t)desc->coarse[0] * desc->coarse[1] * desc->coarse[2];
    m->coarse_active.assign(desc->coarse_active, desc->coarse_active + n);
  }
  m->desc.coarse_active = nullptr;
  m->host_only = host_only;
  m->layout.n_parts = n_parts;
  m->layout.part = part;
  slab_range(desc->coarse[2], n_parts, part, m->layout.k0, m->layout.k1);
  lsmf_status s = build_mesh(*m);
  if (s != LSMF_OK) { delete m; return s; }
  *out = m;
  return LSMF_OK;
}

lsmf_status lsmf_mesh_create_part(const lsmf_mesh_desc *desc, int n_parts, int part, lsmf_mesh **out) {
  return make_part_mesh(desc, n_parts, part, false, out);
}

lsmf_status lsmf_partition_layout(const lsmf_mesh_desc *desc, int n_parts, int part, int *n_nodes, int *n_global_nodes,
                                  int *global_node, int *n_lower, int *lower, int *n_upper, int *upper) {
  lsmf_mesh *m = nullptr;
  LSMF_TRY(make_part_mesh(desc, n_parts, part, true, &m));
  const PartLayout &P = m->layout;
  const int nn = m->levels.back()->n_nodes;
  if (n_nodes) *n_nodes = nn;
  if (n_global_nodes) *n_global_nodes = n_parts > 1 ? P.n_global_nodes : nn;
  if (global_node)
    for (int i = 0; i < nn; ++i) global_node[i] = n_parts > 1 ? P.global_node[i] : i;
  if (n_lower) *n_lower = (int)P.lower_shared.size();
  if (lower) std::memcpy(lower, P.lower_shared.data(), P.lower_shared.size() * sizeof(int));
  if (n_upper) *n_upper = (int)P.upper_shared.size();
  if (upper) std::memcpy(upper, P.upper_shared.data(), P.upper_shared.size() * sizeof(int));
  delete m;
  return LSMF_OK;
}

void lsmf_mesh_destroy(lsmf_mesh *m) { delete m; }

int lsmf_mesh_n_levels(const lsmf_mesh *m) { return m ? (int)m->levels.size() : 0; }

static const Level *level_of(const lsmf_mesh *m, int level) {
  if (!m) return nullptr;
  if (level < 0) level = (int)m->levels.size() - 1;
  if (level >= (int)m->levels.size()) return nullptr;
  return m->levels[level];
}

lsmf_status lsmf_mesh_info(const lsmf_mesh *m, int level, int *n_cells, int *n_nodes, int *n_dofs) {
  const Level *L = level_of(m, level);
  if (!L) { set_error("bad mesh/level"); return LSMF_ERR_INVALID_ARG; }
  if (n_cells) *n_cells = L->n_cells;
  if (n_nodes) *n_nodes = L->n_nodes;
  if (n_dofs) *n_dofs = L->n_dofs();
  return LSMF_OK;
}

lsmf_status lsmf_mesh_arrays(const lsmf_mesh *m, int level, double *X, int *cell_nodes, int *cell_ijk) {
  const Level *L = level_of(m, level);
  if (!L) { set_error("bad mesh/level"); return LSMF_ERR_INVALID_ARG; }
  if (X) std::memcpy(X, L->X.data(), L->X.size() * sizeof(double));
  if (cell_nodes) std::memcpy(cell_nodes, L->cell_nodes.data(), L->cell_nodes.size() * sizeof(int));
  if (cell_ijk) std::memcpy(cell_ijk, L->cell_ijk.data(), L->cell_ijk.size() * sizeof(int));
  return LSMF_OK;
}

lsmf_status lsmf_mesh_set_dirichlet(lsmf_mesh *m, int n, const int *ids, const int *comp_masks) {
  if (!m || n < 0 || (n > 0 && (!ids || !comp_masks))) { set_error("bad arguments"); return LSMF_ERR_INVALID_ARG; }
  m->dir_ids.assign(ids, ids + n);
  m->dir_masks.assign(comp_masks, comp_masks + n);
  for (auto *L : m->levels) LSMF_TRY(level_constraints(*m, *L));
  return LSMF_OK;
}

lsmf_status lsmf_mesh_constraint_mask(const lsmf_mesh *m, int level, uint8_t *mask) {
  const Level *L = level_of(m, level);
  if (!L || !mask) { set_error("bad mesh/level"); return LSMF_ERR_INVALID_ARG; }
  std::memcpy(mask, L->cmask.data(), L->cmask.size());
  return LSMF_OK;
}

lsmf_status lsmf_operator_create(lsmf_mesh *m, int level, lsmf_caching caching, int formulation,
                                 lsmf_precision precision, lsmf_op **out) {
  if (!m || !out) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  *out = nullptr;
  if (level < 0) level = (int)m->levels.size() - 1;
  if (level >= (int)m->levels.size()) { set_error("bad level"); return LSMF_ERR_INVALID_ARG; }
  if (caching != LSMF_CACHE_SCALAR && caching != LSMF_CACHE_TENSOR2 && caching != LSMF_CACHE_TENSOR4 &&
      caching != LSMF_CACHE_SCALAR_REFERENTIAL && caching != LSMF_CACHE_TENSOR4_NS) {
    set_error("Unknown caching");  // mf_nh_operator.h:439-442
    return LSMF_ERR_UNKNOWN_CACHING;
  }
  if (formulation != 0 && formulation != 1) { set_error("Unknown material formulation"); return LSMF_ERR_INVALID_ARG; }
  if (formulation == 0 && caching != LSMF_CACHE_SCALAR) {
    // the reference only caches J^{-1/dim} for formulation 0 (mf_nh_operator.h:466-486)
    set_error("formulation 0 requires scalar caching");
    return LSMF_ERR_UNSUPPORTED;
  }
  if (precision != LSMF_FP64 && precision != LSMF_FP32) { set_error("bad precision"); return LSMF_ERR_INVALID_ARG; }
  lsmf_op *op = new (std::nothrow) lsmf_op();
  if (!op) return LSMF_ERR_ALLOC;
  op->mesh = m; op->level = level; op->caching = caching; op->formulation = formulation;
  op->precision = precision;
  if (cudaGetDevice(&op->device) != cudaSuccess) { delete op; set_error("cudaGetDevice failed"); return LSMF_ERR_CUDA; }
  op->ncomp = table_components(caching, formulation, precision);
  const Level &L = op->L();
  // scalar caching on affine cells: the reference inverse Jacobian is one
  // 3x3 block per cell after the 11 per-point values (c, Eulerian inverse
  // Jacobian, JxW); otherwise ncomp values per point.  Every record is
  // padded at its end to a multiple of 16 bytes (bulk copies and aligned
  // records), never with whole components.
  op->ref_per_cell = caching == LSMF_CACHE_SCALAR && L.affine;
  const int al = 16 / (int)op->elem();
  if (op->ref_per_cell) {
    op->ncomp = 11;
    op->rec_elems = (11 * L.nq() + 9 + al - 1) / al * al;
  } else {
    op->rec_elems = (op->ncomp * L.nq() + al - 1) / al * al;
  }
  lsmf_status s;
  if ((s = op->d_table.alloc((size_t)L.n_cells * op->rec_elems * op->elem())) != LSMF_OK ||
      (s = op->d_diag.alloc((size_t)L.n_dofs() * op->elem())) != LSMF_OK ||
      (s = op->d_inv_diag.alloc((size_t)L.n_dofs() * op->elem())) != LSMF_OK ||
      (s = op->d_flag.alloc(1)) != LSMF_OK) {
    delete op;
    return s;
  }
  op->mu_host.assign(L.n_cells, 1.0);
  if ((s = op->d_mu.upload(op->mu_host.data(), op->mu_host.size())) != LSMF_OK) { delete op; return s; }
  *out = op;
  return LSMF_OK;
}

void lsmf_operator_destroy(lsmf_op *op) { delete op; }

lsmf_status lsmf_operator_set_material(lsmf_op *op, const double *mu, double nu) {
  if (!op || !mu) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (!(nu > -1.0 && nu < 0.5)) { set_error("Poisson's ratio must be in (-1, 0.5)"); return LSMF_ERR_INVALID_ARG; }
  const int n = op->L().n_cells;
  for (int i = 0; i < n; ++i)
    if (!(mu[i] > 0.0)) { set_error("shear modulus must be positive"); return LSMF_ERR_INVALID_ARG; }
  op->mu_host.assign(mu, mu + n);
  op->nu = nu;
  LSMF_TRY(op->d_mu.upload(op->mu_host.data(), n));
  op->cached = false;
  return LSMF_OK;
}

lsmf_status lsmf_operator_set_option(lsmf_op *op, int option, int value) {
  if (!op) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (option == LSMF_OPT_BULK_PIPELINE) {
    if (value < -1 || value > 3) { set_error("pipeline depth must be -1 (auto) or 0..3"); return LSMF_ERR_INVALID_ARG; }
    op->stages = value;
    return LSMF_OK;
  }
  if (option == LSMF_OPT_BASIC_KERNEL) { op->basic = value != 0; return LSMF_OK; }
  if (option == LSMF_OPT_MAX_WARPS) {
    if (value < 0 || value > 8) { set_error("warps per block must be 0 (auto) or 1..8"); return LSMF_ERR_INVALID_ARG; }
    op->max_warps = value;
    return LSMF_OK;
  }
  if (option == LSMF_OPT_WAIT_TRIES) {
    if (value < -1) { set_error("wait tries must be -1 (default) or >= 0"); return LSMF_ERR_INVALID_ARG; }
    op->wait_tries = value;
    return LSMF_OK;
  }
  if (option == LSMF_OPT_RECORD_PREFETCH) {
    if (value < -1 || value > 2) { set_error("record prefetch must be -1 (auto), 0, 1 or 2"); return LSMF_ERR_INVALID_ARG; }
    op->prefetch = value;
    return LSMF_OK;
  }
  if (option == LSMF_OPT_CELL_PAIRS) {
    if (value < -1 || value > 1) { set_error("cell pairs must be -1 (auto), 0 or 1"); return LSMF_ERR_INVALID_ARG; }
    op->pairs = value;
    return LSMF_OK;
  }
  if (option == LSMF_OPT_CHUNKS) {
    if (value < -1 || value == 0 || value > 8) { set_error("chunks must be -1 (auto) or 1..8"); return LSMF_ERR_INVALID_ARG; }
    op->chunks = value;
    // a cached operator builds the plan for the new count now, not inside
    // the first vmult (which may run in a stream capture)
    int k = 1;
    return op->cached ? effective_chunks(op, &k) : LSMF_OK;
  }
  if (option == LSMF_OPT_SCATTER) return set_scatter_mode(op, value);
  set_error("unknown option");
  return LSMF_ERR_INVALID_ARG;
}

lsmf_status lsmf_operator_get_option(lsmf_op *op, int option, int *value) {
  if (!op || !value) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  switch (option) {
    case LSMF_OPT_BULK_PIPELINE: *value = op->stages; return LSMF_OK;
    case LSMF_OPT_BASIC_KERNEL: *value = op->basic ? 1 : 0; return LSMF_OK;
    case LSMF_OPT_MAX_WARPS: *value = op->max_warps; return LSMF_OK;
    case LSMF_OPT_WAIT_TRIES: *value = op->wait_tries; return LSMF_OK;
    case LSMF_OPT_SCATTER: *value = op->scatter; return LSMF_OK;
    case LSMF_OPT_RECORD_PREFETCH: *value = op->prefetch; return LSMF_OK;
    case LSMF_OPT_CELL_PAIRS: *value = op->pairs; return LSMF_OK;
    case LSMF_OPT_CHUNKS: return effective_chunks(op, value);
  }
  set_error("unknown option");
  return LSMF_ERR_INVALID_ARG;
}

lsmf_status lsmf_operator_set_stream(lsmf_op *op, void *stream) {
  if (!op) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  op->stream = (cudaStream_t)stream;
  return LSMF_OK;
}

lsmf_status lsmf_operator_cache(lsmf_op *op, const void *d_u) {
  if (!op || !d_u) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  op->d_u = d_u;
  LSMF_TRY(launch_cache(op));
  int flag = 0;
  LSMF_CUDA(cudaMemcpyAsync(&flag, op->d_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, op->stream));
  LSMF_CUDA(cudaStreamSynchronize(op->stream));
  op->have_diag = false;
  if (flag) {
    op->cached = false;
    set_error("det_F is not positive at some quadrature point");
    return LSMF_ERR_DETF_NONPOSITIVE;
  }
  op->cached = true;
  // the chunk plan of the vmult (streams, events, node ranges) is built
  // here, outside any stream capture a caller may later run the vmult in
  int k = 1;
  return effective_chunks(op, &k);
}

lsmf_status lsmf_operator_vmult(lsmf_op *op, void *d_dst, const void *d_src, unsigned mask) {
  if (!op || !d_dst || !d_src) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (!op->cached) { set_error("cache() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  return launch_apply(op, d_dst, d_src, mask, false);
}

lsmf_status lsmf_operator_vmult_add(lsmf_op *op, void *d_dst, const void *d_src) {
  if (!op || !d_dst || !d_src) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (!op->cached) { set_error("cache() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  return launch_apply(op, d_dst, d_src, LSMF_MASK_DEFAULT, true);
}

lsmf_status lsmf_operator_sync(lsmf_op *op) {
  if (!op) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  int flag = 0;
  LSMF_CUDA(cudaMemcpyAsync(&flag, op->d_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, op->stream));
  LSMF_CUDA(cudaStreamSynchronize(op->stream));
  if (flag & 2) {
    // reported once: the word is cleared for the calls that follow
    LSMF_CUDA(cudaMemsetAsync(op->d_flag.ptr, 0, sizeof(int), op->stream));
    LSMF_CUDA(cudaStreamSynchronize(op->stream));
    set_error("a bounded device wait timed out in the vmult kernel; the result of that vmult is incomplete");
    return LSMF_ERR_TIMEOUT;
  }
  if (flag & 4) {
    LSMF_CUDA(cudaMemsetAsync(op->d_flag.ptr, 0, sizeof(int), op->stream));
    LSMF_CUDA(cudaStreamSynchronize(op->stream));
    set_error("a vmult kernel was launched with less shared memory than its layout needs and did no work");
    return LSMF_ERR_CUDA;
  }
  return LSMF_OK;
}

lsmf_status lsmf_operator_compute_diagonal(lsmf_op *op) {
  if (!op) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (!op->cached) { set_error("cache() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  LSMF_TRY(launch_diagonal(op));
  op->have_diag = true;
  return LSMF_OK;
}

lsmf_status lsmf_operator_get_diagonal(lsmf_op *op, const void **d_diag, const void **d_inv) {
  if (!op) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (!op->have_diag) { set_error("compute_diagonal() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  if (d_diag) *d_diag = op->d_diag.ptr;
  if (d_inv) *d_inv = op->d_inv_diag.ptr;
  return LSMF_OK;
}

lsmf_status lsmf_operator_precondition_jacobi(lsmf_op *op, void *d_dst, const void *d_src, double omega) {
  if (!op || !d_dst || !d_src) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (!op->have_diag) { set_error("compute_diagonal() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  return launch_jacobi(op, d_dst, d_src, omega);
}

int lsmf_operator_m(const lsmf_op *op) { return op ? op->L().n_dofs() : 0; }

int lsmf_operator_n(const lsmf_op *op) { return op ? op->L().n_dofs() : 0; }

lsmf_status lsmf_operator_el(lsmf_op *op, int row, int col, double *value) {
  if (!op || !value) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (row != col) { set_error("el() is only implemented on the diagonal (row == col)"); return LSMF_ERR_UNSUPPORTED; }
  if (row < 0 || row >= op->L().n_dofs()) { set_error("row out of range"); return LSMF_ERR_INVALID_ARG; }
  if (!op->have_diag) { set_error("compute_diagonal() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  LSMF_CUDA(cudaStreamSynchronize(op->stream));
  if (op->precision == LSMF_FP64) {
    LSMF_CUDA(cudaMemcpy(value, (const double *)op->d_diag.ptr + row, sizeof(double), cudaMemcpyDeviceToHost));
  } else {
    float f = 0;
    LSMF_CUDA(cudaMemcpy(&f, (const float *)op->d_diag.ptr + row, sizeof(float), cudaMemcpyDeviceToHost));
    *value = f;
  }
  return LSMF_OK;
}

size_t lsmf_operator_memory_consumption(const lsmf_op *op) {
  // cache tables + index maps (the reference excludes the diagonals too,
  // mf_nh_operator.h:300-328)
  if (!op) return 0;
  const Level &L = op->L();
  return op->d_table.n + L.d_cell_nodes.n * sizeof(int) + L.d_X.n * sizeof(double);
}

lsmf_status lsmf_operator_get_table(lsmf_op *op, int which, double *host, size_t *count) {
  if (!op || !count) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  const Level &L = op->L();
  const int nq = L.nq();
  int c0 = 0, nk = 0;
  const bool t4 = op->caching == LSMF_CACHE_TENSOR4, t2 = op->caching == LSMF_CACHE_TENSOR2;
  const bool sr = op->caching == LSMF_CACHE_SCALAR_REFERENTIAL, ns = op->caching == LSMF_CACHE_TENSOR4_NS;
  // tensor4 / tensor2 / tensor4_ns keep no JxW component: their
  // coefficients (times JxW) start at component 9
  const int cv = (t4 || t2 || ns) ? 9 : 10;
  switch (which) {
    case 0: if (t4 || ns) { set_error("no scalar table"); return LSMF_ERR_INVALID_ARG; } c0 = cv; nk = 1; break;
    case 1: if (!t2) { set_error("no second scalar table"); return LSMF_ERR_INVALID_ARG; } c0 = cv + 1; nk = 1; break;
    case 2: if (!t2 && !t4) { set_error("no tensor2 table"); return LSMF_ERR_INVALID_ARG; } c0 = t4 ? cv : cv + 2; nk = 6; break;
    case 3: if (!t4) { set_error("no tensor4 table"); return LSMF_ERR_INVALID_ARG; } c0 = cv + 6; nk = 36; break;
    case 4: c0 = 0; nk = 9; break;
    case 5:
      if (cv == 9) { set_error("JxW is folded into the coefficient tables of this caching"); return LSMF_ERR_INVALID_ARG; }
      c0 = 9; nk = 1; break;
    case 6: if (!sr) { set_error("no displacement table"); return LSMF_ERR_INVALID_ARG; } c0 = cv + 1; nk = 3; break;
    case 7: if (!ns) { set_error("no tensor4_ns table"); return LSMF_ERR_INVALID_ARG; } c0 = cv; nk = 81; break;
    default: set_error("bad table id"); return LSMF_ERR_INVALID_ARG;
  }
  const size_t n = (size_t)L.n_cells * nq * nk;
  *count = n;
  if (!host) return LSMF_OK;
  std::vector<char> raw(op->d_table.n);
  LSMF_CUDA(cudaStreamSynchronize(op->stream));
  LSMF_CUDA(cudaMemcpy(raw.data(), op->d_table.ptr, raw.size(), cudaMemcpyDeviceToHost));
  for (int cell = 0; cell < L.n_cells; ++cell)
    for (int q = 0; q < nq; ++q)
      for (int k = 0; k < nk; ++k) {
        const size_t src = (size_t)cell * op->rec_elems + (size_t)(c0 + k) * nq + q;
        const double v = op->precision == LSMF_FP64 ? ((const double *)raw.data())[src]
                                                    : (double)((const float *)raw.data())[src];
        host[((size_t)cell * nq + q) * nk + k] = v;
      }
  return LSMF_OK;
}

}  // extern "C"
