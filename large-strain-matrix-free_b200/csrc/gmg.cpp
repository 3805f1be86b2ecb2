// Geometric multigrid preconditioner and CG solver on the device.
//
// Replaces the deal.II objects set up in Solid::setup_matrix_free
// (mf_elasticity.h:2079-2238: PreconditionChebyshev smoothers, coarse
// Chebyshev-as-solver, MGTransferMatrixFree, Multigrid, PreconditionMG) and
// the SolverCG of Solid::solve_linear_system (mf_elasticity.h:3012-3214).
// Every level operator is an lsmf_op of the level precision; vectors stay
// resident on the device; the host only drives the iteration and reads one
// scalar (the residual norm) per CG iteration.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>

#include "solver_internal.h"

namespace lsmf {

double tridiag_eig(const std::vector<double> &d, const std::vector<double> &e, bool want_max) {
  const int n = (int)d.size();
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < n; ++i) {
    const double r = (i > 0 ? std::fabs(e[i - 1]) : 0) + (i < n - 1 ? std::fabs(e[i]) : 0);
    lo = std::min(lo, d[i] - r);
    hi = std::max(hi, d[i] + r);
  }
  auto count_below = [&](double x) {
    int cnt = 0;
    double q = 1.0;
    for (int i = 0; i < n; ++i) {
      const double ee = (i > 0) ? e[i - 1] * e[i - 1] : 0.0;
      q = d[i] - x - (i > 0 ? ee / q : 0.0);
      if (q == 0.0) q = -1e-300;
      if (q < 0) ++cnt;
    }
    return cnt;
  };
  const int k = want_max ? n - 1 : 0;
  double a = lo, b = hi;
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (a + b);
    if (count_below(mid) > k) b = mid; else a = mid;
    if (b - a <= 1e-15 * std::max(std::fabs(a), std::fabs(b))) break;
  }
  return 0.5 * (a + b);
}

std::vector<double> coarsen_cell_field(const lsmf_mesh &M, int level, const std::vector<double> &fine) {
  const Level &F = *M.levels.back();
  const Level &L = *M.levels[level];
  const int sh = (int)M.levels.size() - 1 - level;
  std::vector<double> out(L.n_cells, 0.0);
  for (int c = 0; c < L.n_cells; ++c) {
    const int i0 = L.cell_ijk[3 * c] << sh, j0 = L.cell_ijk[3 * c + 1] << sh, k0 = L.cell_ijk[3 * c + 2] << sh;
    double s = 0;
    int n = 0;
    for (int k = k0; k < k0 + (1 << sh); ++k)
      for (int j = j0; j < j0 + (1 << sh); ++j)
        for (int i = i0; i < i0 + (1 << sh); ++i) {
          const int fc = F.cell_of_lattice[((size_t)k * F.nc[1] + j) * F.nc[0] + i];
          if (fc >= 0) { s += fine[fc]; ++n; }
        }
    out[c] = n ? s / n : 1.0;
  }
  return out;
}

namespace {

// CG with the inverse diagonal on a level operator (PreconditionChebyshev's
// eigenvalue estimate): start vector (i % 11) - mean, ReductionControl with
// absolute sqrt(eps) and relative 1e-10, extreme eigenvalues of the Lanczos
// tridiagonal matrix built from the CG coefficients.
template <typename T>
lsmf_status estimate_eigenvalues(lsmf_gmg *g, int l, int max_it, double &emin, double &emax, int &its) {
  lsmf_gmg_level &GL = g->levels[l];
  lsmf_op *op = GL.op;
  const size_t n = (size_t)op->L().n_dofs();
  cudaStream_t st = g->stream;
  // work vectors at 16-byte-aligned offsets (whole multiples of 4 values)
  const size_t ns = (n + 3) / 4 * 4;
  T *x = (T *)g->eig_vecs.ptr, *gg = x + ns, *h = gg + ns, *d = h + ns;
  const T *invd = (const T *)op->d_inv_diag.ptr;
  const uint8_t *cm = op->L().d_cmask.ptr;
  // start vector (i mod 11) - mean, made on the device; the mean of the
  // integers i mod 11 is exact in closed form (the sum is below 2^53)
  const size_t q11 = n / 11, r11 = n % 11;
  const double mean = (double)(55 * q11 + r11 * (r11 - 1) / 2) / (double)n;
  LSMF_TRY(eig_start_async<T>(gg, n, mean, st));  // g = A 0 - b
  LSMF_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), st));
  double *sc = g->sc.ptr, *part = g->partial.ptr;
  const bool fp32 = sizeof(T) == 4;
  auto dot = [&](const T *a, const T *b, double &out) -> lsmf_status {
    LSMF_TRY(dot_async(a, b, fp32, n, part, sc, SC_TMP, st));
    LSMF_CUDA(cudaMemcpyAsync(&out, sc + SC_TMP, sizeof(double), cudaMemcpyDeviceToHost, st));
    LSMF_CUDA(cudaStreamSynchronize(st));
    return LSMF_OK;
  };
  double res2;
  LSMF_TRY(dot(gg, gg, res2));
  const double res0 = std::sqrt(res2);
  const double tol = std::max(std::sqrt((double)std::numeric_limits<T>::epsilon()), 1e-10 * res0);
  std::vector<double> dT, oT;
  its = 0;
  if (res0 > tol) {
    LSMF_TRY(jacobi_async<T>(h, invd, gg, 1.0, n, st));
    LSMF_CUDA(cudaMemsetAsync(d, 0, n * sizeof(T), st));
    LSMF_TRY(dir_async<T>(d, h, 0.0, n, st));  // d = -h
    LSMF_TRY(dot_async(gg, h, fp32, n, part, sc, SC_GH0, st));
    LSMF_CUDA(cudaMemsetAsync(h, 0, n * sizeof(T), st));  // the cell loop accumulates into h
    // CG iterations run in batches of 8 with device-resident scalars; the
    // alpha / beta / residual history is read once per batch and the Lanczos
    // matrix is cut at the first iteration that meets the tolerance, so the
    // estimate equals the one of an iteration checked every step
    // one history buffer for every level (sized for the largest iteration
    // budget, so no level re-allocates it)
    size_t need = 0;
    for (const auto &L : g->levels) need = std::max(need, (size_t)L.op->L().n_dofs());
    need = 3 * (std::max(need, (size_t)g->desc.eig_cg_iterations) + 8);
    if (g->eig_hist.n < need) LSMF_TRY(g->eig_hist.alloc(need));
    const size_t stride = need / 3;
    double *ha = g->eig_hist.ptr, *hb = ha + stride, *hr = hb + stride;
    // one batch of iterations k0 + j, j < batch; with kbase the history
    // index is *kbase + j and the batch is the same launch sequence every
    // time (parity of k0 even), so it can be captured once and replayed
    auto batch_launch = [&](int k0, int batch, const int *kbase) -> lsmf_status {
      // per iteration: cell loop into h (zero on entry), identity rows + d.h,
      // g update + Jacobi + g.g and g.h, direction update that clears h
      for (int j = 0; j < batch; ++j) {
        const int k = k0 + j;
        const int gh = SC_GH0 + (k & 1), ghn = SC_GH0 + ((k + 1) & 1);
        const int kh = kbase ? j : k;
        LSMF_TRY(launch_apply_cells(op, h, d));
        LSMF_TRY(eig_dh_async<T>(d, h, cm, n, part, sc, st));
        LSMF_TRY(eig_update_precond_async<T>(gg, h, invd, n, sc, gh, ghn, ha, hr, kh, kbase, part, st));
        LSMF_TRY(eig_dir_clear_async<T>(d, h, n, sc, ghn, gh, hb, kh, kbase, st));
      }
      if (kbase) LSMF_TRY(eig_advance_async(const_cast<int *>(kbase), batch, st));
      return LSMF_OK;
    };
    // long estimates (the coarse solver's, up to n iterations) replay a
    // captured batch: one graph launch instead of ~70 kernel launches
    cudaGraphExec_t bexec = nullptr;
    if (g->use_graph && max_it >= 64) {
      if (g->eig_kbase.n < 1) LSMF_TRY(g->eig_kbase.alloc(1));
      LSMF_CUDA(cudaMemsetAsync(g->eig_kbase.ptr, 0, sizeof(int), st));
      if (!g->cap_stream) LSMF_CUDA(cudaStreamCreateWithFlags(&g->cap_stream, cudaStreamNonBlocking));
      const cudaStream_t user = st;
      lsmf_gmg_set_stream(g, g->cap_stream);
      st = g->cap_stream;
      LSMF_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
      const lsmf_status s = batch_launch(0, 8, g->eig_kbase.ptr);
      cudaGraph_t graph = nullptr;
      const cudaError_t e = cudaStreamEndCapture(st, &graph);
      lsmf_gmg_set_stream(g, user);
      st = user;
      if (s != LSMF_OK) { if (graph) cudaGraphDestroy(graph); return s; }
      if (e != cudaSuccess) { set_error(std::string("eigenvalue CG capture: ") + cudaGetErrorString(e)); return LSMF_ERR_CUDA; }
      const cudaError_t ei = cudaGraphInstantiate(&bexec, graph, 0);
      cudaGraphDestroy(graph);
      if (ei != cudaSuccess) { set_error(std::string("eigenvalue CG graph: ") + cudaGetErrorString(ei)); return LSMF_ERR_CUDA; }
    }
    // Batches are pipelined: batch i + 1 is launched before the host reads
    // the history of batch i (pinned copies + an event), so the GPU does not
    // wait for the host's convergence check.  A batch launched after the
    // converged one only writes history past the cut and scratch vectors.
    if (!g->eig_pinned && cudaMallocHost((void **)&g->eig_pinned, 2 * 3 * 8 * sizeof(double)) != cudaSuccess) {
      g->eig_pinned = nullptr;
      if (bexec) cudaGraphExecDestroy(bexec);
      set_error("cudaMallocHost of the eigenvalue-CG history copies failed");
      return LSMF_ERR_ALLOC;
    }
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int slot_n[2] = {0, 0};
    bool slot_busy[2] = {false, false};
    lsmf_status status = LSMF_OK;
    for (int s = 0; s < 2 && status == LSMF_OK; ++s)
      if (cudaEventCreateWithFlags(&ev[s], cudaEventDisableTiming) != cudaSuccess) {
        set_error("cudaEventCreate failed");
        status = LSMF_ERR_CUDA;
      }
    int k = 0;  // first iteration not launched yet
    // launch the batch k .. k + n - 1 and the copies of its history into slot s
    auto issue = [&](int s) -> lsmf_status {
      const int batch = std::min(8, max_it - k);
      if (bexec && batch == 8) {
        // the replayed batch writes history k .. k + 7 (its base is k)
        const cudaError_t e = cudaGraphLaunch(bexec, st);
        if (e != cudaSuccess) { set_error(std::string("cudaGraphLaunch: ") + cudaGetErrorString(e)); return LSMF_ERR_CUDA; }
      } else {
        LSMF_TRY(batch_launch(k, batch, nullptr));
      }
      double *P = g->eig_pinned + s * 24;
      cudaError_t e = cudaMemcpyAsync(P, ha + k, batch * sizeof(double), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(P + 8, hb + k, batch * sizeof(double), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(P + 16, hr + k, batch * sizeof(double), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaEventRecord(ev[s], st);
      if (e != cudaSuccess) { set_error(std::string("eigenvalue CG history: ") + cudaGetErrorString(e)); return LSMF_ERR_CUDA; }
      slot_n[s] = batch;
      slot_busy[s] = true;
      k += batch;
      return LSMF_OK;
    };
    bool done = false;
    double prev_beta = 0, prev_alpha = 0;
    int cur = 0;
    if (status == LSMF_OK && max_it > 0) status = issue(cur);
    while (status == LSMF_OK && !done && slot_busy[cur]) {
      if (k < max_it && (status = issue(cur ^ 1)) != LSMF_OK) break;
      const cudaError_t e = cudaEventSynchronize(ev[cur]);
      slot_busy[cur] = false;
      if (e != cudaSuccess) { set_error(std::string("eigenvalue CG history: ") + cudaGetErrorString(e)); status = LSMF_ERR_CUDA; break; }
      const double *P = g->eig_pinned + cur * 24;
      for (int j = 0; j < slot_n[cur] && !done; ++j) {
        ++its;
        const double alpha = P[j];
        if (its > 1) {
          dT.push_back(1.0 / alpha + prev_beta / prev_alpha);
          oT.push_back(std::sqrt(prev_beta) / prev_alpha);
        } else {
          dT.push_back(1.0 / alpha);
        }
        if (std::sqrt(P[16 + j]) <= tol || its >= max_it) done = true;
        prev_beta = P[8 + j];
        prev_alpha = alpha;
      }
      cur ^= 1;
    }
    // a batch launched past the converged one may still be copying into
    // the pinned slots: wait for it before they can be reused
    for (int s = 0; s < 2; ++s) {
      if (slot_busy[s]) cudaEventSynchronize(ev[s]);
      if (ev[s]) cudaEventDestroy(ev[s]);
    }
    if (bexec) cudaGraphExecDestroy(bexec);
    if (status != LSMF_OK) return status;
  }
  emin = emax = 1.0;
  if (!dT.empty()) {
    emin = tridiag_eig(dT, oT, false);
    emax = tridiag_eig(dT, oT, true);
  }
  return LSMF_OK;
}

// Chebyshev data from the eigenvalue estimates (degree <= 0: "solver" mode
// with range = requested reduction, the degree from the Chebyshev error bound)
void chebyshev_coefficients(lsmf_cheb &c, int degree, double range) {
  const double max_eig = 1.2 * c.eig_max;
  const double alpha = (range > 1.0) ? max_eig / range : std::min(0.9 * max_eig, c.eig_min);
  c.degree = degree;
  if (degree <= 0) {
    const double actual_range = max_eig / alpha;
    const double sigma = (1. - std::sqrt(1. / actual_range)) / (1. + std::sqrt(1. / actual_range));
    const double eps = range;
    c.degree = 1 + (int)(std::log(1. / eps + std::sqrt(1. / eps / eps - 1.)) / std::log(1. / sigma));
  }
  c.theta = 0.5 * (max_eig + alpha);
  c.delta = 0.5 * (max_eig - alpha);
}

// PreconditionChebyshev::vmult (zero_start) / step on the vectors x, b of
// level l (the level's r and xold are the smoother's work vectors)
template <typename T>
lsmf_status chebyshev_run(lsmf_gmg *g, int l, T *x, const T *b, bool zero_start) {
  lsmf_gmg_level &GL = g->levels[l];
  lsmf_op *op = GL.op;
  const size_t n = (size_t)op->L().n_dofs();
  cudaStream_t st = g->stream;
  T *xold = (T *)GL.xold.ptr, *r = (T *)GL.r.ptr;
  const T *invd = (const T *)op->d_inv_diag.ptr;
  const lsmf_cheb &c = GL.cheb;
  const uint8_t *cm = op->L().d_cmask.ptr;
  // r is kept at zero between the steps by the update kernels
  if (zero_start) {
    LSMF_TRY(cheb_zero_async<T>(x, b, invd, c.theta, n, st));
    LSMF_CUDA(cudaMemsetAsync(r, 0, n * sizeof(T), st));
  } else {
    LSMF_CUDA(cudaMemsetAsync(r, 0, n * sizeof(T), st));
    LSMF_TRY(launch_apply_cells(op, r, x));
    LSMF_TRY(cheb_first_async<T>(x, xold, b, r, invd, cm, c.theta, n, st));
  }
  if (c.degree < 2 || std::fabs(c.delta) < 1e-40) return LSMF_OK;
  double rhok = c.delta / c.theta;
  const double sigma = c.theta / c.delta;
  for (int k = 0; k < c.degree - 1; ++k) {
    LSMF_TRY(launch_apply_cells(op, r, x));
    const double rhokp = 1. / (2. * sigma - rhok);
    const double f1 = rhokp * rhok, f2 = 2. * rhokp / c.delta;
    rhok = rhokp;
    LSMF_TRY(cheb_step_async<T>(x, xold, b, r, invd, cm, f1, f2, !(zero_start && k == 0), n, st));
  }
  return LSMF_OK;
}

// MGCoarseGridIterativeSolver (mf_elasticity.h:2116-2127): CG on level 0,
// preconditioned by the level-0 Chebyshev smoother, ReductionControl with
// max(m, 100) steps, absolute 1e-10, relative 1e-3, zero initial guess
template <typename T>
lsmf_status coarse_cg(lsmf_gmg *g) {
  lsmf_gmg_level &GL = g->levels[0];
  lsmf_op *op = GL.op;
  const size_t n = (size_t)op->L().n_dofs();
  cudaStream_t st = g->stream;
  const bool fp32 = sizeof(T) == 4;
  T *x = (T *)GL.x.ptr, *b = (T *)GL.b.ptr;
  const size_t ns = (n + 3) / 4 * 4;  // 16-byte-aligned work vectors
  T *gg = (T *)g->eig_vecs.ptr, *h = gg + ns, *d = h + ns;
  double *sc = g->sc.ptr, *part = g->partial.ptr;
  auto dot = [&](const T *a, const T *c, double &out) -> lsmf_status {
    LSMF_TRY(dot_async(a, c, fp32, n, part, sc, SC_TMP, st));
    LSMF_CUDA(cudaMemcpyAsync(&out, sc + SC_TMP, sizeof(double), cudaMemcpyDeviceToHost, st));
    LSMF_CUDA(cudaStreamSynchronize(st));
    return LSMF_OK;
  };
  LSMF_CUDA(cudaMemsetAsync(x, 0, n * sizeof(T), st));
  LSMF_CUDA(cudaMemsetAsync(gg, 0, n * sizeof(T), st));
  LSMF_TRY(dir_async<T>(gg, b, 0.0, n, st));  // g = A 0 - b
  double res2;
  LSMF_TRY(dot(gg, gg, res2));
  const double tol = std::max(1e-10, 1e-3 * std::sqrt(res2));
  if (std::sqrt(res2) <= tol) return LSMF_OK;
  const int max_it = std::max((int)n, 100);
  LSMF_TRY(chebyshev_run<T>(g, 0, h, gg, true));
  LSMF_CUDA(cudaMemsetAsync(d, 0, n * sizeof(T), st));
  LSMF_TRY(dir_async<T>(d, h, 0.0, n, st));
  double gh;
  LSMF_TRY(dot(gg, h, gh));
  for (int it = 1; it <= max_it; ++it) {
    LSMF_TRY(launch_apply(op, h, d, LSMF_MASK_DEFAULT, false));
    double dh;
    LSMF_TRY(dot(d, h, dh));
    const double alpha = gh / dh;
    LSMF_TRY(axpy_async<T>(x, alpha, d, n, st));
    LSMF_TRY(axpy_async<T>(gg, alpha, h, n, st));
    LSMF_TRY(dot(gg, gg, res2));
    if (std::sqrt(res2) <= tol || !(res2 == res2)) break;
    LSMF_TRY(chebyshev_run<T>(g, 0, h, gg, true));
    const double gh_old = gh;
    LSMF_TRY(dot(gg, h, gh));
    LSMF_TRY(dir_async<T>(d, h, gh / gh_old, n, st));
  }
  return LSMF_OK;
}

// Multigrid::level_v_step
template <typename T>
lsmf_status vcycle(lsmf_gmg *g, int l) {
  if (l == 0) {
    if (!g->desc.coarse_chebyshev) return coarse_cg<T>(g);
    // MGCoarseGridApplySmoother
    return chebyshev_run<T>(g, 0, (T *)g->levels[0].x.ptr, (const T *)g->levels[0].b.ptr, true);
  }
  lsmf_gmg_level &GL = g->levels[l], &GC = g->levels[l - 1];
  cudaStream_t st = g->stream;
  const lsmf_mesh &M = *g->mesh;
  LSMF_TRY(chebyshev_run<T>(g, l, (T *)GL.x.ptr, (const T *)GL.b.ptr, true));  // pre-smoothing (apply)
  LSMF_TRY(launch_apply(GL.op, GL.r.ptr, GL.x.ptr, LSMF_MASK_DEFAULT, false));
  LSMF_CUDA(cudaMemsetAsync(GC.b.ptr, 0, (size_t)GC.op->L().n_dofs() * sizeof(T), st));
  LSMF_TRY(restrict_add_async<T>(*M.levels[l - 1], *M.transfer[l], (const T *)GL.b.ptr, (const T *)GL.r.ptr,
                                 (T *)GC.b.ptr, g->scatter, st));
  LSMF_TRY(vcycle<T>(g, l - 1));
  LSMF_TRY(prolongate_add_async<T>(*M.levels[l - 1], *M.transfer[l], (const T *)GC.x.ptr, (T *)GL.x.ptr, g->scatter,
                                   st));
  LSMF_TRY(chebyshev_run<T>(g, l, (T *)GL.x.ptr, (const T *)GL.b.ptr, false));  // post-smoothing (step)
  return LSMF_OK;
}

template <typename T>
lsmf_status gmg_setup_impl(lsmf_gmg *g, const double *d_u) {
  const lsmf_mesh &M = *g->mesh;
  const int nl = (int)g->levels.size();
  cudaStream_t st = g->stream;
  for (auto &GL : g->levels) GL.op->stream = st;
  // interpolate_to_mg in level precision
  const size_t nf = (size_t)M.levels[nl - 1]->n_dofs();
  LSMF_TRY(convert_async<T, double>((T *)g->levels[nl - 1].u.ptr, d_u, nf, st));
  for (int l = nl - 1; l > 0; --l)
    LSMF_TRY(interpolate_async<T>(*M.levels[l - 1], *M.levels[l], *M.transfer[l], (const T *)g->levels[l].u.ptr,
                                  (T *)g->levels[l - 1].u.ptr, st));
  for (int l = 0; l < nl; ++l) {
    lsmf_gmg_level &GL = g->levels[l];
    LSMF_TRY(lsmf_operator_cache(GL.op, GL.u.ptr));
    LSMF_TRY(lsmf_operator_compute_diagonal(GL.op));
    const bool coarse_solver = (l == 0 && g->desc.coarse_chebyshev);
    const int eig_its = coarse_solver && g->desc.coarse_accurate_eig ? GL.op->L().n_dofs() : g->desc.eig_cg_iterations;
    LSMF_TRY(estimate_eigenvalues<T>(g, l, eig_its, GL.cheb.eig_min, GL.cheb.eig_max, GL.cheb.eig_iterations));
    if (coarse_solver) chebyshev_coefficients(GL.cheb, 0, 1e-3);
    else chebyshev_coefficients(GL.cheb, g->desc.smoother_degree, g->desc.smoothing_range);
  }
  g->ready = true;
  return LSMF_OK;
}

template <typename T>
lsmf_status gmg_vmult_impl(lsmf_gmg *g, double *dst, const double *src) {
  const int nl = (int)g->levels.size();
  lsmf_gmg_level &GT = g->levels[nl - 1];
  const size_t n = (size_t)GT.op->L().n_dofs();
  cudaStream_t st = g->stream;
  LSMF_TRY(convert_async<T, double>((T *)GT.b.ptr, src, n, st));  // copy_to_mg
  LSMF_TRY(vcycle<T>(g, nl - 1));
  LSMF_TRY(convert_async<double, T>(dst, (const T *)GT.x.ptr, n, st));  // copy_from_mg
  return LSMF_OK;
}

}  // namespace
}  // namespace lsmf

using namespace lsmf;

static void drop_graph(lsmf_gmg *g) {
  if (g->vexec) cudaGraphExecDestroy(g->vexec);
  g->vexec = nullptr;
  g->vsrc = nullptr;
  g->vdst = nullptr;
}

lsmf_gmg::~lsmf_gmg() {
  drop_graph(this);
  if (eig_pinned) cudaFreeHost(eig_pinned);
  if (cap_stream) cudaStreamDestroy(cap_stream);
  for (auto &GL : levels) lsmf_operator_destroy(GL.op);
}

extern "C" {

lsmf_status lsmf_gmg_create(lsmf_mesh *m, const lsmf_gmg_desc *desc, lsmf_gmg **out) {
  if (!m || !desc || !out) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  *out = nullptr;
  if (desc->smoother_degree < 1 || desc->eig_cg_iterations < 1 || !(desc->smoothing_range > 1.0)) {
    set_error("bad Chebyshev parameters");
    return LSMF_ERR_INVALID_ARG;
  }
  lsmf_gmg *g = new (std::nothrow) lsmf_gmg();
  if (!g) return LSMF_ERR_ALLOC;
  g->mesh = m;
  g->desc = *desc;
  const int nl = (int)m->levels.size();
  g->levels.resize(nl);
  lsmf_status s = LSMF_OK;
  size_t nmax = 0;
  for (int l = 0; l < nl && s == LSMF_OK; ++l) {
    lsmf_gmg_level &GL = g->levels[l];
    s = lsmf_operator_create(m, l, (lsmf_caching)desc->caching, desc->formulation, desc->precision, &GL.op);
    if (s != LSMF_OK) break;
    // level cell loops in one launch: the chunked form measured slower in
    // the GMG-preconditioned Newton solve (voids 60^3 Q2: +4 % per Newton
    // iteration); the option still selects it per level
    GL.op->chunks = 1;
    const size_t n = (size_t)m->levels[l]->n_dofs() * g->elem();
    nmax = std::max(nmax, ((size_t)m->levels[l]->n_dofs() + 3) / 4 * 4 * g->elem());
    if ((s = GL.x.alloc(n)) != LSMF_OK || (s = GL.b.alloc(n)) != LSMF_OK || (s = GL.r.alloc(n)) != LSMF_OK ||
        (s = GL.xold.alloc(n)) != LSMF_OK || (s = GL.u.alloc(n)) != LSMF_OK)
      break;
  }
  if (s == LSMF_OK) s = g->sc.alloc(SC_N);
  if (s == LSMF_OK) s = g->partial.alloc(2 * (size_t)reduce_blocks());  // two partial-sum arrays
  if (s == LSMF_OK) s = g->eig_vecs.alloc(4 * nmax);
  if (s != LSMF_OK) { delete g; return s; }
  g->mu_fine.assign(m->levels.back()->n_cells, 1.0);
  *out = g;
  return LSMF_OK;
}

void lsmf_gmg_destroy(lsmf_gmg *g) { delete g; }

lsmf_status lsmf_gmg_set_material(lsmf_gmg *g, const double *mu, double nu) {
  if (!g || !mu) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  const int nf = g->mesh->levels.back()->n_cells;
  g->mu_fine.assign(mu, mu + nf);
  g->nu = nu;
  for (int l = 0; l < (int)g->levels.size(); ++l) {
    const std::vector<double> ml = coarsen_cell_field(*g->mesh, l, g->mu_fine);
    LSMF_TRY(lsmf_operator_set_material(g->levels[l].op, ml.data(), nu));
  }
  g->ready = false;
  drop_graph(g);
  return LSMF_OK;
}

lsmf_status lsmf_gmg_setup(lsmf_gmg *g, const double *d_u) {
  if (!g || !d_u) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  // the executable V-cycle graph is kept: the next vmult captures the new
  // launch sequence and updates it in place
  g->vstale = true;
  return g->desc.precision == LSMF_FP64 ? gmg_setup_impl<double>(g, d_u) : gmg_setup_impl<float>(g, d_u);
}

lsmf_status lsmf_gmg_level_operator(lsmf_gmg *g, int level, lsmf_op **op) {
  if (!g || !op) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (level < 0 || level >= (int)g->levels.size()) { set_error("bad level"); return LSMF_ERR_INVALID_ARG; }
  *op = g->levels[level].op;
  g->vstale = true;  // options of the returned operator may change the captured V-cycle
  return LSMF_OK;
}

lsmf_status lsmf_gmg_set_option(lsmf_gmg *g, int option, int value) {
  if (!g) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (option == LSMF_GMG_OPT_GRAPH) {
    g->use_graph = value != 0;
    drop_graph(g);
    return LSMF_OK;
  }
  if (option == LSMF_GMG_OPT_SCATTER) {
    // level operators take the mode (node sums for their vmult cell loops);
    // transfers run the colours for every mode but atomic
    for (auto &GL : g->levels) LSMF_TRY(set_scatter_mode(GL.op, value));
    g->scatter = value;
    // the captured V-cycle holds the old launch sequence
    drop_graph(g);
    return LSMF_OK;
  }
  set_error("unknown option");
  return LSMF_ERR_INVALID_ARG;
}

lsmf_status lsmf_gmg_vmult(lsmf_gmg *g, double *dst, const double *src) {
  if (!g || !dst || !src) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (!g->ready) { set_error("lsmf_gmg_setup has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  auto run = [&]() {
    return g->desc.precision == LSMF_FP64 ? gmg_vmult_impl<double>(g, dst, src) : gmg_vmult_impl<float>(g, dst, src);
  };
  // the CG coarse solver reads scalars on the host, so that V-cycle is not
  // captured
  if (!g->use_graph || !g->desc.coarse_chebyshev) return run();
  if (!g->vexec || g->vstale || g->vsrc != src || g->vdst != dst) {
    // capture the V-cycle (a fixed sequence of launches once the Chebyshev
    // coefficients are known) on a private stream, then replay it
    if (!g->cap_stream) LSMF_CUDA(cudaStreamCreateWithFlags(&g->cap_stream, cudaStreamNonBlocking));
    const cudaStream_t user = g->stream;
    lsmf_gmg_set_stream(g, g->cap_stream);
    LSMF_CUDA(cudaStreamBeginCapture(g->cap_stream, cudaStreamCaptureModeRelaxed));
    const lsmf_status s = run();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(g->cap_stream, &graph);
    lsmf_gmg_set_stream(g, user);
    if (s != LSMF_OK) { if (graph) cudaGraphDestroy(graph); drop_graph(g); return s; }
    if (e != cudaSuccess) { drop_graph(g); set_error(std::string("V-cycle capture: ") + cudaGetErrorString(e)); return LSMF_ERR_CUDA; }
    // same launch sequence as the executable graph (same levels, degrees
    // and kernels; new scalars and pointers): update it in place, which
    // skips the instantiation (~2.4 ms for the ~1,600 nodes of a 762-step
    // coarse solve); a changed sequence (another coarse degree) is
    // instantiated anew
    bool updated = false;
    if (g->vexec) {
      cudaGraphExecUpdateResultInfo info{};
      updated = cudaGraphExecUpdate(g->vexec, graph, &info) == cudaSuccess;
      if (!updated) {
        (void)cudaGetLastError();  // the failed update is not sticky
        drop_graph(g);
      }
    }
    if (!updated) {
      const cudaError_t ei = cudaGraphInstantiate(&g->vexec, graph, 0);
      if (ei != cudaSuccess) {
        cudaGraphDestroy(graph);
        g->vexec = nullptr;
        set_error(std::string("V-cycle graph: ") + cudaGetErrorString(ei));
        return LSMF_ERR_CUDA;
      }
    }
    cudaGraphDestroy(graph);
    g->vsrc = src;
    g->vdst = dst;
    g->vstale = false;
  }
  LSMF_CUDA(cudaGraphLaunch(g->vexec, g->stream));
  return LSMF_OK;
}

lsmf_status lsmf_gmg_level_info(const lsmf_gmg *g, int level, double *out6) {
  if (!g || !out6 || level < 0 || level >= (int)g->levels.size()) { set_error("bad arguments"); return LSMF_ERR_INVALID_ARG; }
  const lsmf_cheb &c = g->levels[level].cheb;
  out6[0] = c.eig_min; out6[1] = c.eig_max; out6[2] = c.degree; out6[3] = c.theta; out6[4] = c.delta;
  out6[5] = c.eig_iterations;
  return LSMF_OK;
}

lsmf_status lsmf_gmg_set_stream(lsmf_gmg *g, void *stream) {
  if (!g) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  g->stream = (cudaStream_t)stream;
  for (auto &GL : g->levels) GL.op->stream = g->stream;
  return LSMF_OK;
}

// SolverCG (deal.II form: g = A x - b, d = -P g; convergence on ||g||)
lsmf_status lsmf_cg_solve(lsmf_op *A, int precond, double omega, lsmf_gmg *gmg, double *x, const double *b,
                          double tol_abs, int max_it, lsmf_solve_info *info) {
  if (!A || !x || !b) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (A->precision != LSMF_FP64) { set_error("the outer CG operator must be FP64"); return LSMF_ERR_INVALID_ARG; }
  if (!A->cached) { set_error("cache() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  if (precond == 1 && !A->have_diag) { set_error("Jacobi needs compute_diagonal()"); return LSMF_ERR_NOT_INITIALIZED; }
  if (precond == 2 && (!gmg || !gmg->ready)) { set_error("GMG is not set up"); return LSMF_ERR_NOT_INITIALIZED; }
  if (precond < 0 || precond > 2) { set_error("precond must be 0, 1 or 2"); return LSMF_ERR_INVALID_ARG; }
  const size_t n = (size_t)A->L().n_dofs();
  cudaStream_t st = A->stream;
  if (gmg) lsmf_gmg_set_stream(gmg, st);
  LSMF_TRY(A->cg_g.alloc(n));
  LSMF_TRY(A->cg_h.alloc(n));
  LSMF_TRY(A->cg_d.alloc(n));
  LSMF_TRY(A->sc.alloc(SC_N));
  LSMF_TRY(A->partial.alloc(reduce_blocks()));
  double *g = A->cg_g.ptr, *h = A->cg_h.ptr, *d = A->cg_d.ptr, *sc = A->sc.ptr, *part = A->partial.ptr;
  auto read = [&](int slot, double &v) -> lsmf_status {
    LSMF_CUDA(cudaMemcpyAsync(&v, sc + slot, sizeof(double), cudaMemcpyDeviceToHost, st));
    LSMF_CUDA(cudaStreamSynchronize(st));
    return LSMF_OK;
  };
  auto prec = [&](double *dst, const double *src) -> lsmf_status {
    if (precond == 0) {
      LSMF_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
      return LSMF_OK;
    }
    if (precond == 1) return jacobi_async<double>(dst, (const double *)A->d_inv_diag.ptr, src, omega, n, st);
    return lsmf_gmg_vmult(gmg, dst, src);
  };
  LSMF_TRY(launch_apply(A, h, x, LSMF_MASK_DEFAULT, false));
  LSMF_TRY(neg_residual_async<double>(g, h, b, n, st));
  LSMF_TRY(dot_async(g, g, false, n, part, sc, SC_RES2, st));
  double res2;
  LSMF_TRY(read(SC_RES2, res2));
  double res = std::sqrt(res2);
  int it = 0;
  bool conv = res <= tol_abs;
  if (!conv && max_it > 0) {
    LSMF_TRY(prec(h, g));
    LSMF_TRY(dot_async(g, h, false, n, part, sc, SC_GH0, st));
    LSMF_TRY(cg_dir_async(d, h, n, sc, SC_GH0, SC_GH0, true, st));
    int k = 0;
    while (true) {
      ++it;
      LSMF_TRY(launch_apply(A, h, d, LSMF_MASK_DEFAULT, false));
      LSMF_TRY(dot_async(d, h, false, n, part, sc, SC_DH, st));
      LSMF_TRY(cg_update_async(x, g, d, h, n, sc, SC_GH0 + (k & 1), part, st));
      LSMF_TRY(read(SC_RES2, res2));
      res = std::sqrt(res2);
      if (!(res == res)) break;  // NaN: report non-convergence
      if (res <= tol_abs) { conv = true; break; }
      if (it >= max_it) break;
      LSMF_TRY(prec(h, g));
      LSMF_TRY(dot_async(g, h, false, n, part, sc, SC_GH0 + ((k + 1) & 1), st));
      LSMF_TRY(cg_dir_async(d, h, n, sc, SC_GH0 + ((k + 1) & 1), SC_GH0 + (k & 1), false, st));
      ++k;
    }
  }
  int flag = 0;
  LSMF_CUDA(cudaMemcpyAsync(&flag, A->d_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  LSMF_CUDA(cudaStreamSynchronize(st));
  if (info) { info->iterations = it; info->residual = res; info->converged = conv ? 1 : 0; }
  if (flag & 2) {
    // reported once: the word is cleared for the calls that follow
    LSMF_CUDA(cudaMemsetAsync(A->d_flag.ptr, 0, sizeof(int), st));
    LSMF_CUDA(cudaStreamSynchronize(st));
    set_error("a bounded device wait timed out in the vmult kernel");
    return LSMF_ERR_TIMEOUT;
  }
  if (flag & 4) {
    LSMF_CUDA(cudaMemsetAsync(A->d_flag.ptr, 0, sizeof(int), st));
    LSMF_CUDA(cudaStreamSynchronize(st));
    set_error("a vmult kernel was launched with less shared memory than its layout needs and did no work");
    return LSMF_ERR_CUDA;
  }
  if (!conv) {
    // the facts of deal.II's SolverControl::NoConvergence: last step and value
    char msg[160];
    std::snprintf(msg, sizeof msg, "CG did not reach the tolerance (|g| = %.3e after %d iterations, tolerance %.3e)",
                  res, it, tol_abs);
    set_error(msg);
    return LSMF_ERR_CG_NOT_CONVERGED;
  }
  return LSMF_OK;
}

}  // extern "C"
