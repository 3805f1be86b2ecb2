// Internal interfaces of the solver layer (CG, GMG, Newton) and its kernels.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "lsmf_internal.h"

namespace lsmf {

// device scalar slots used by the CG kernels
enum { SC_DH = 0, SC_RES2 = 1, SC_GH0 = 2, SC_GH1 = 3, SC_TMP = 4, SC_N = 8 };

int reduce_blocks();
lsmf_status dot_async(const void *a, const void *b, bool fp32, size_t n, double *partial, double *sc, int slot,
                      cudaStream_t st);
lsmf_status cg_update_async(double *x, double *g, const double *d, const double *h, size_t n, double *sc, int gh_slot,
                            double *partial, cudaStream_t st);
lsmf_status cg_dir_async(double *d, const double *h, size_t n, const double *sc, int gh_new, int gh_old, bool first,
                         cudaStream_t st);
lsmf_status eig_advance_async(int *kbase, int by, cudaStream_t st);
// fused eigenvalue-CG step (h holds the cell part of A d on entry):
//   eig_dh: identity rows h_c += d_c, sc[DH] = d.h
//   eig_update_precond: alpha = sc[gh]/sc[DH] (hist), g += alpha h,
//     h = D^-1 g, hist_res2 = g.g, sc[gh_new] = g.h
//   eig_dir_clear: beta = sc[gh_new]/sc[gh] (hist), d = beta d - h, h = 0
// (partial needs 2 * reduce_blocks() doubles)
template <typename T>
lsmf_status eig_dh_async(const T *d, T *h, const uint8_t *cmask, size_t n, double *partial, double *sc, cudaStream_t st);
template <typename T>
lsmf_status eig_update_precond_async(T *g, T *h, const T *invd, size_t n, double *sc, int gh_slot, int gh_new,
                                     double *hist_alpha, double *hist_res2, int k, const int *kbase, double *partial,
                                     cudaStream_t st);
template <typename T>
lsmf_status eig_dir_clear_async(T *d, T *h, size_t n, const double *sc, int gh_new, int gh_old, double *hist_beta, int k,
                                const int *kbase, cudaStream_t st);
// g = A 0 - b for the start vector b_i = (i mod 11) - mean
template <typename T>
lsmf_status eig_start_async(T *g, size_t n, double mean, cudaStream_t st);
template <typename T>
lsmf_status neg_residual_async(T *g, const T *ax, const T *b, size_t n, cudaStream_t st);
template <typename T>
lsmf_status jacobi_async(T *dst, const T *invd, const T *src, double omega, size_t n, cudaStream_t st);
template <typename TD, typename TS>
lsmf_status convert_async(TD *dst, const TS *src, size_t n, cudaStream_t st);
template <typename T>
lsmf_status axpy_async(T *y, double a, const T *x, size_t n, cudaStream_t st);
template <typename T>
lsmf_status dir_async(T *d, const T *h, double beta, size_t n, cudaStream_t st);  // d = beta d - h
template <typename T>
lsmf_status set_indexed_async(T *v, const int *idx, int n, double val, cudaStream_t st);
template <typename T>
lsmf_status copy_indexed_async(T *dst, const T *src, const int *idx, int n, cudaStream_t st);
template <typename T>
lsmf_status cheb_zero_async(T *x, const T *b, const T *invd, double theta, size_t n, cudaStream_t st);
// r: cell contributions of A x only; identity rows added from cmask, r cleared
template <typename T>
lsmf_status cheb_first_async(T *x, T *xold, const T *b, T *r, const T *invd, const uint8_t *cmask, double theta,
                             size_t n, cudaStream_t st);
template <typename T>
lsmf_status cheb_step_async(T *x, T *xold, const T *b, T *r, const T *invd, const uint8_t *cmask, double f1, double f2,
                            bool has_old, size_t n, cudaStream_t st);
// scatter: LSMF_SCATTER_ATOMIC, or any other mode: one launch per colour
// of the coarse cells, plain adds, bit-reproducible
template <typename T>
lsmf_status restrict_add_async(const Level &C, const TransferMap &TM, const T *b, const T *r, T *coarse, int scatter,
                               cudaStream_t st);
template <typename T>
lsmf_status prolongate_add_async(const Level &C, const TransferMap &TM, const T *coarse, T *fine, int scatter,
                                 cudaStream_t st);
template <typename T>
lsmf_status interpolate_async(const Level &C, const Level &F, const TransferMap &TM, const T *fine_u, T *coarse_u,
                              cudaStream_t st);
lsmf_status internal_force_async(const Level &L, const Basis &B, const double *u, const double *mu, double nu,
                                 int formulation, double *R, int scatter, cudaStream_t st);
lsmf_status adjoint_cell_grad_async(const Level &L, const Basis &B, const double *u, const double *mu, double nu,
                                    int formulation, const double *lam, double *grad, cudaStream_t st);
// apply with an un-zeroed gather of constrained entries (K g over the
// constrained columns, the inhomogeneity term of the rhs)
lsmf_status launch_apply_inhomogeneous(const lsmf_op *op, void *dst, const void *g);

// Eigenvalues of a symmetric tridiagonal matrix (Sturm bisection).
double tridiag_eig(const std::vector<double> &d, const std::vector<double> &e, bool want_max);

// per-cell values of a coarser level from a fine per-cell field: mean of
// the fine cells inside each coarse cell
std::vector<double> coarsen_cell_field(const lsmf_mesh &M, int level, const std::vector<double> &fine);

}  // namespace lsmf

// Chebyshev smoother data of one level (PreconditionChebyshev)
struct lsmf_cheb {
  int degree = 5;
  double theta = 1, delta = 0, eig_min = 1, eig_max = 1;
  int eig_iterations = 0;
};

struct lsmf_gmg_level {
  lsmf_op *op = nullptr;
  lsmf::DevBuf<char> x, b, r, xold, u;  // level precision
  lsmf_cheb cheb;
};

struct lsmf_gmg {
  lsmf_mesh *mesh = nullptr;
  lsmf_gmg_desc desc{};
  std::vector<lsmf_gmg_level> levels;
  std::vector<double> mu_fine;
  double nu = 0.3;
  lsmf::DevBuf<double> sc, partial;
  lsmf::DevBuf<char> eig_vecs;  // scratch for the eigenvalue CG (4 level vectors)
  lsmf::DevBuf<double> eig_hist; // alpha / beta / residual history of the eigenvalue CG
  lsmf::DevBuf<int> eig_kbase;   // history base of the replayed eigenvalue-CG batches
  // pinned host copies of two batches of alpha / beta / residual history
  // (2 slots x 3 x 8 doubles), read while the next batch runs
  double *eig_pinned = nullptr;
  cudaStream_t stream = 0;
  bool ready = false;
  // the V-cycle replayed as one CUDA graph: captured again after each
  // set-up (vstale) and applied to the executable graph in place when the
  // launch sequence is unchanged
  bool use_graph = true;
  int scatter = LSMF_SCATTER_ATOMIC;  // LSMF_SCATTER_* of the level operators; transfers: atomics or colours
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t vexec = nullptr;
  bool vstale = true;
  const double *vsrc = nullptr;
  double *vdst = nullptr;
  size_t elem() const { return desc.precision == LSMF_FP64 ? 8 : 4; }
  ~lsmf_gmg();
};
