// sm_100a kernels of the solver around the tangent operator:
//   deterministic dot products / norms (fixed grid, two-pass reduction)
//   fused CG vector updates with device-resident scalars
//   Chebyshev smoother updates
//   level transfer (MGTransferMatrixFree semantics) and displacement
//   interpolation onto the coarse levels
//   FP64 residual (internal force) and the adjoint cell gradient
#include <cuda_runtime.h>

#include <cstdint>
#include <initializer_list>

#include "cell_kernels.cuh"
#include "lsmf_internal.h"
#include "solver_internal.h"

namespace lsmf {

namespace {

constexpr int RED_THREADS = 256;

template <typename A, typename B>
__global__ void dot_partial_kernel(const A *a, const B *b, size_t n, double *partial) {
  __shared__ double sh[RED_THREADS / 32];
  double s = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    s += (double)a[i] * (double)b[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

// sums partial[0..n) in a fixed order into out[*koff] (out[0] without koff)
__global__ void reduce_final_kernel(const double *partial, int n, double *out, const int *koff = nullptr) {
  __shared__ double sh[32];
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[koff ? *koff : 0] = s;
  }
}

// CG: alpha = sc[gh] / sc[DH]; x += alpha d; g += alpha h; partial sums of g.g
__global__ void cg_update_kernel(double *x, double *g, const double *d, const double *h, size_t n,
                                 const double *sc, int gh_slot, double *partial) {
  __shared__ double sh[RED_THREADS / 32];
  const double alpha = sc[gh_slot] / sc[SC_DH];
  double s = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    x[i] += alpha * d[i];
    const double gi = g[i] + alpha * h[i];
    g[i] = gi;
    s += gi * gi;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

// CG direction: beta = sc[gh_new] / sc[gh_old]; d = beta d - h (beta = 0: d = -h)
__global__ void cg_dir_kernel(double *d, const double *h, size_t n, const double *sc, int gh_new, int gh_old,
                              int first) {
  // the first direction does not read d: it holds whatever the allocation
  // held (0 * NaN would be NaN)
  const double beta = first ? 0.0 : sc[gh_new] / sc[gh_old];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    d[i] = first ? -h[i] : beta * d[i] - h[i];
}

// 16-byte vectors of level values (4 floats / 2 doubles) for the
// bandwidth-bound element-wise kernels: one load instruction moves 16 bytes,
// so a warp keeps 4x (2x) more bytes in flight than with scalar loads.  The
// launchers use them only when every operand is 16-byte aligned (vec_ok).
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
  static constexpr int W = 4;
  __device__ static float get(const float4 &v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
  __device__ static void set(float4 &v, int k, float a) {
    if (k == 0) v.x = a; else if (k == 1) v.y = a; else if (k == 2) v.z = a; else v.w = a;
  }
};
template <>
struct Vec16<double> {
  using type = double2;
  static constexpr int W = 2;
  __device__ static double get(const double2 &v, int k) { return k == 0 ? v.x : v.y; }
  __device__ static void set(double2 &v, int k, double a) {
    if (k == 0) v.x = a; else v.y = a;
  }
};
// true when every vector (and the mask, at W-byte granularity) allows the
// 16-byte loads; sub-arrays of work buffers may not
template <typename T>
inline int vec_ok(std::initializer_list<const void *> ptrs, const uint8_t *cmask) {
  for (const void *p : ptrs)
    if ((uintptr_t)p % 16 != 0) return 0;
  return (cmask == nullptr || (uintptr_t)cmask % Vec16<T>::W == 0) ? 1 : 0;
}
// W mask bytes starting at a multiple of W
template <int W>
__device__ __forceinline__ unsigned load_mask(const uint8_t *cm, size_t i) {
  if (W == 4) return *(const unsigned *)(cm + i);
  return *(const unsigned short *)(cm + i);
}

// history base of a replayed batch of eigenvalue-CG iterations
__global__ void eig_advance_kernel(int *kbase, int by) { *kbase += by; }

// eigenvalue-CG start: g = A 0 - b with b_i = (i mod 11) - mean
template <typename T>
__global__ void eig_start_kernel(T *g, size_t n, double mean) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    g[i] = T(mean - (double)(i % 11));
}

// block sum of s into partial[blockIdx.x] (same pattern as dot_partial_kernel)
__device__ __forceinline__ void block_partial(double s, double *partial) {
  __shared__ double sh[RED_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
  __syncthreads();  // sh may be reused by a second call
}

template <typename T>
__global__ void eig_dh_kernel(const T *__restrict__ d, T *__restrict__ h, const uint8_t *__restrict__ cmask, size_t n,
                              double *partial, int vec) {
  using VT = Vec16<T>;
  using V = typename VT::type;
  constexpr int W = VT::W;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, st = (size_t)gridDim.x * blockDim.x;
  const size_t nv = vec ? n / W : 0;
  double s = 0;
  for (size_t v = t0; v < nv; v += st) {
    const V dv = ((const V *)d)[v];
    V hv = ((const V *)h)[v];
    const unsigned cm = load_mask<W>(cmask, v * W);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      T hi = VT::get(hv, k);
      if ((cm >> (8 * k)) & 0xff) hi = hi + VT::get(dv, k);  // constrained row: identity
      VT::set(hv, k, hi);
      s += (double)VT::get(dv, k) * (double)hi;
    }
    if (cm) ((V *)h)[v] = hv;
  }
  for (size_t i = nv * W + t0; i < n; i += st) {
    T hi = h[i];
    if (cmask[i]) {
      hi = hi + d[i];
      h[i] = hi;
    }
    s += (double)d[i] * (double)hi;
  }
  block_partial(s, partial);
}

template <typename T>
__device__ __forceinline__ void eig_update_at(T &g, T &h, T invd, double alpha, double &s1, double &s2) {
  const T gi = T((double)g + alpha * (double)h);
  g = gi;
  s1 += (double)gi * (double)gi;
  const T hi = T(1) * invd * gi;  // Jacobi, omega = 1
  h = hi;
  s2 += (double)gi * (double)hi;
}
template <typename T>
__global__ void eig_update_precond_kernel(T *__restrict__ g, T *__restrict__ h, const T *__restrict__ invd, size_t n,
                                          const double *sc, int gh_slot, double *hist_alpha, int k,
                                          const int *kbase, double *partial_gg, double *partial_gh, int vec) {
  using VT = Vec16<T>;
  using V = typename VT::type;
  constexpr int W = VT::W;
  const double alpha = sc[gh_slot] / sc[SC_DH];
  if (blockIdx.x == 0 && threadIdx.x == 0) hist_alpha[(kbase ? *kbase : 0) + k] = alpha;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, st = (size_t)gridDim.x * blockDim.x;
  const size_t nv = vec ? n / W : 0;
  double s1 = 0, s2 = 0;
  for (size_t v = t0; v < nv; v += st) {
    V gv = ((const V *)g)[v], hv = ((const V *)h)[v];
    const V dv = ((const V *)invd)[v];
#pragma unroll
    for (int q = 0; q < W; ++q) {
      T gq = VT::get(gv, q), hq = VT::get(hv, q);
      eig_update_at<T>(gq, hq, VT::get(dv, q), alpha, s1, s2);
      VT::set(gv, q, gq);
      VT::set(hv, q, hq);
    }
    ((V *)g)[v] = gv;
    ((V *)h)[v] = hv;
  }
  for (size_t i = nv * W + t0; i < n; i += st) eig_update_at<T>(g[i], h[i], invd[i], alpha, s1, s2);
  block_partial(s1, partial_gg);
  block_partial(s2, partial_gh);
}

// two fixed-order sums: p1 -> out1[*koff1], p2 -> *out2
__global__ void reduce2_final_kernel(const double *p1, const double *p2, int n, double *out1, const int *koff1,
                                     double *out2) {
  __shared__ double sh[32];
  for (int pass = 0; pass < 2; ++pass) {
    const double *p = pass == 0 ? p1 : p2;
    double s = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += p[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
      s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      if (threadIdx.x == 0) {
        if (pass == 0) out1[koff1 ? *koff1 : 0] = s;
        else *out2 = s;
      }
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void eig_dir_clear_kernel(T *__restrict__ d, T *__restrict__ h, size_t n, const double *sc, int gh_new,
                                     int gh_old, double *hist_beta, int k, const int *kbase, int vec) {
  using VT = Vec16<T>;
  using V = typename VT::type;
  constexpr int W = VT::W;
  const double beta = sc[gh_new] / sc[gh_old];
  if (blockIdx.x == 0 && threadIdx.x == 0) hist_beta[(kbase ? *kbase : 0) + k] = beta;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, st = (size_t)gridDim.x * blockDim.x;
  const size_t nv = vec ? n / W : 0;
  for (size_t v = t0; v < nv; v += st) {
    V dv = ((const V *)d)[v];
    const V hv = ((const V *)h)[v];
    V zero;
#pragma unroll
    for (int q = 0; q < W; ++q) {
      VT::set(dv, q, T(beta * (double)VT::get(dv, q) - (double)VT::get(hv, q)));
      VT::set(zero, q, T(0));
    }
    ((V *)d)[v] = dv;
    ((V *)h)[v] = zero;
  }
  for (size_t i = nv * W + t0; i < n; i += st) {
    d[i] = T(beta * (double)d[i] - (double)h[i]);
    h[i] = T(0);
  }
}

template <typename T>
__global__ void residual_init_kernel(T *g, const T *ax, const T *b, size_t n) {
  // g = A x - b (deal.II SolverCG's negative residual)
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    g[i] = ax[i] - b[i];
}

template <typename T>
__global__ void scaled_mul_kernel2(T *dst, const T *a, const T *b, T s, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = s * a[i] * b[i];
}

template <typename TD, typename TS>
__global__ void convert_kernel(TD *dst, const TS *src, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = TD(src[i]);
}

template <typename T>
__global__ void axpy_kernel(T *y, T a, const T *x, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}

template <typename T>
__global__ void dir_kernel(T *d, const T *h, double beta, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    d[i] = T(beta * (double)d[i] - (double)h[i]);
}

template <typename T>
__global__ void set_indexed_kernel(T *v, const int *idx, int n, T val) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[idx[i]] = val;
}

template <typename T>
__global__ void copy_indexed_kernel(T *dst, const T *src, const int *idx, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[idx[i]] = src[idx[i]];
}

// ---------------------------------------------------------------- Chebyshev
// x = D^-1 b / theta                                   (vmult, zero start)
// x_old = x; x += D^-1 (b - r) / theta                 (step, first update)
// x_new = x + f1 (x - x_old) + f2 D^-1 (b - r); x_old = x; x = x_new

template <typename T>
__global__ void cheb_zero_kernel(T *__restrict__ x, const T *__restrict__ b, const T *__restrict__ invd,
                                 double inv_theta, size_t n, int vec) {
  using VT = Vec16<T>;
  using V = typename VT::type;
  constexpr int W = VT::W;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, st = (size_t)gridDim.x * blockDim.x;
  const size_t nv = vec ? n / W : 0;  // vec: every pointer 16-byte aligned
  for (size_t v = t0; v < nv; v += st) {
    const V bv = ((const V *)b)[v], dv = ((const V *)invd)[v];
    V xv;
#pragma unroll
    for (int k = 0; k < W; ++k) VT::set(xv, k, T((double)VT::get(dv, k) * (double)VT::get(bv, k) * inv_theta));
    ((V *)x)[v] = xv;
  }
  for (size_t i = nv * W + t0; i < n; i += st) x[i] = T((double)invd[i] * (double)b[i] * inv_theta);
}
// r holds only the cell contributions of A x: the identity rows of the
// constrained dofs are added here (A x = x there), and r is cleared for the
// next cell loop, so a smoothing step is one cell-loop kernel plus this one
template <typename T>
__device__ __forceinline__ void cheb_first_at(T &x, T &xold, T b, T &r, T invd, bool cm, double inv_theta) {
  const T xi = x;
  const double ax = (double)r + (cm ? (double)xi : 0.0);
  r = T(0);
  xold = xi;
  x = T((double)xi + (double)invd * ((double)b - ax) * inv_theta);
}
template <typename T>
__global__ void cheb_first_kernel(T *__restrict__ x, T *__restrict__ xold, const T *__restrict__ b,
                                  T *__restrict__ r, const T *__restrict__ invd, const uint8_t *__restrict__ cmask,
                                  double inv_theta, size_t n, int vec) {
  using VT = Vec16<T>;
  using V = typename VT::type;
  constexpr int W = VT::W;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, st = (size_t)gridDim.x * blockDim.x;
  const size_t nv = vec ? n / W : 0;  // vec: every pointer 16-byte aligned
  for (size_t v = t0; v < nv; v += st) {
    V xv = ((const V *)x)[v], rv = ((const V *)r)[v], xo;
    const V bv = ((const V *)b)[v], dv = ((const V *)invd)[v];
    const unsigned cm = load_mask<W>(cmask, v * W);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      T xk = VT::get(xv, k), ok, rk = VT::get(rv, k);
      cheb_first_at<T>(xk, ok, VT::get(bv, k), rk, VT::get(dv, k), (cm >> (8 * k)) & 0xff, inv_theta);
      VT::set(xv, k, xk);
      VT::set(xo, k, ok);
      VT::set(rv, k, rk);
    }
    ((V *)x)[v] = xv;
    ((V *)xold)[v] = xo;
    ((V *)r)[v] = rv;
  }
  for (size_t i = nv * W + t0; i < n; i += st) cheb_first_at<T>(x[i], xold[i], b[i], r[i], invd[i], cmask[i], inv_theta);
}
template <typename T>
__device__ __forceinline__ void cheb_step_at(T &x, T &xold, T b, T &r, T invd, bool cm, double f1, double f2,
                                             bool has_old) {
  const double xi = (double)x;
  const double ax = (double)r + (cm ? xi : 0.0);
  r = T(0);
  const double xo = has_old ? (double)xold : 0.0;
  const double xn = xi + f1 * (xi - xo) + f2 * (double)invd * ((double)b - ax);
  xold = T(xi);
  x = T(xn);
}
template <typename T>
__global__ void cheb_step_kernel(T *__restrict__ x, T *__restrict__ xold, const T *__restrict__ b,
                                 T *__restrict__ r, const T *__restrict__ invd, const uint8_t *__restrict__ cmask,
                                 double f1, double f2, int has_old, size_t n, int vec) {
  using VT = Vec16<T>;
  using V = typename VT::type;
  constexpr int W = VT::W;
  const size_t t0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x, st = (size_t)gridDim.x * blockDim.x;
  const size_t nv = vec ? n / W : 0;  // vec: every pointer 16-byte aligned
  for (size_t v = t0; v < nv; v += st) {
    V xv = ((const V *)x)[v], rv = ((const V *)r)[v], xo;
    if (has_old) xo = ((const V *)xold)[v];
    const V bv = ((const V *)b)[v], dv = ((const V *)invd)[v];
    const unsigned cm = load_mask<W>(cmask, v * W);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      T xk = VT::get(xv, k), ok = has_old ? VT::get(xo, k) : T(0), rk = VT::get(rv, k);
      cheb_step_at<T>(xk, ok, VT::get(bv, k), rk, VT::get(dv, k), (cm >> (8 * k)) & 0xff, f1, f2, has_old != 0);
      VT::set(xv, k, xk);
      VT::set(xo, k, ok);
      VT::set(rv, k, rk);
    }
    ((V *)x)[v] = xv;
    ((V *)xold)[v] = xo;
    ((V *)r)[v] = rv;
  }
  for (size_t i = nv * W + t0; i < n; i += st)
    cheb_step_at<T>(x[i], xold[i], b[i], r[i], invd[i], cmask[i], f1, f2, has_old != 0);
}

// ------------------------------------------------------------------ transfer
// 1D prolongation matrix in the level's arithmetic type (FP32 levels add in
// FP32, FP64 levels in FP64)
template <int P, typename C>
struct Prol1D {
  C m[2 * P + 1][P + 1];
};

// one warp per coarse cell.  restriction: coarse += R (weight * (b - r))
// on the fine level, coarse Dirichlet entries dropped (restrict_and_add).
// cells / plain: the coarse cells of one lattice colour (no two share a
// node) with plain adds, or (cells == nullptr) all n_coarse cells with
// atomics.  Every load that depends only on the coarse cell (its fine
// block's node ids, its own node ids) is issued first, then every load that
// depends on those (weights, fine values), so a cell costs two round trips.
template <int P, typename T>
__global__ void restrict_kernel(int n_coarse, const int *__restrict__ cells, int plain, const int *__restrict__ coarse_cn,
                                const int *__restrict__ fine_nodes, const double *__restrict__ weight,
                                const T *__restrict__ b, const T *__restrict__ r, T *coarse, Prol1D<P, T> pm) {
  constexpr int N1 = P + 1, NF = 2 * P + 1, NFB = NF * NF * NF, NCN = N1 * N1 * N1;
  constexpr int SZ = 3 * NFB + 3 * NF * NF * N1 + 3 * NF * N1 * N1;
  constexpr int NPL = (NFB + 31) / 32, CPL = (3 * NCN + 31) / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  T *in = (T *)smem_raw + warp * SZ, *s1 = in + 3 * NFB, *s2 = s1 + 3 * NF * NF * N1;
  for (int ic = blockIdx.x * wpb + warp; ic < n_coarse; ic += gridDim.x * wpb) {
    const int c = cells ? __ldg(cells + ic) : ic;
    const int *fn = fine_nodes + (size_t)c * NFB;
    int node[NPL], cpk[CPL];
#pragma unroll
    for (int q = 0; q < NPL; ++q) node[q] = (lane + 32 * q < NFB) ? __ldg(fn + lane + 32 * q) : -1;
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int it = lane + 32 * q;
      cpk[q] = it < 3 * NCN ? __ldg(coarse_cn + (size_t)c * NCN + it % NCN) : 0;
    }
    // weights and values in chunks of CH fine nodes per lane (all of them
    // at degree <= 2; degree 3 / 4 blocks of 343 / 729 nodes would otherwise
    // hold 7 values x 11 / 23 nodes per lane in registers)
    constexpr int CH = NPL < 4 ? NPL : 4;
#pragma unroll
    for (int q0 = 0; q0 < NPL; q0 += CH) {
      T w[CH], bv[CH][3], rv[CH][3];
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const int q = q0 + j;
        if (q >= NPL || node[q] < 0) continue;
        w[j] = T(__ldg(weight + node[q]));
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const size_t d = 3 * (size_t)node[q] + k;
          bv[j][k] = b[d];
          rv[j][k] = r ? r[d] : T(0);
        }
      }
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const int q = q0 + j;
        if (q >= NPL || node[q] < 0) continue;
#pragma unroll
        for (int k = 0; k < 3; ++k) in[k * NFB + lane + 32 * q] = w[j] * (bv[j][k] - rv[j][k]);
      }
    }
    __syncwarp();
    // z: s1[k][z][fy][fx] = sum_fz P[fz][z] in[k][fz][fy][fx]
    for (int it = lane; it < 3 * N1 * NF * NF; it += 32) {
      const int fyx = it % (NF * NF), z = (it / (NF * NF)) % N1, k = it / (NF * NF * N1);
      T s = 0;
#pragma unroll
      for (int fz = 0; fz < NF; ++fz) s += pm.m[fz][z] * in[k * NFB + fz * NF * NF + fyx];
      s1[it] = s;
    }
    __syncwarp();
    // y: s2[k][z][y][fx]
    for (int it = lane; it < 3 * N1 * N1 * NF; it += 32) {
      const int fx = it % NF, y = (it / NF) % N1, kz = it / (NF * N1);
      T s = 0;
#pragma unroll
      for (int fy = 0; fy < NF; ++fy) s += pm.m[fy][y] * s1[(kz * NF + fy) * NF + fx];
      s2[it] = s;
    }
    __syncwarp();
    // x: coarse value of node (x, y, z)
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int it = lane + 32 * q;
      if (it >= 3 * NCN) continue;
      const int a = it % NCN, k = it / NCN, x = a % N1, zy = a / N1;
      T s = 0;
#pragma unroll
      for (int fx = 0; fx < NF; ++fx) s += pm.m[fx][x] * s2[zy * NF + fx + k * N1 * N1 * NF];
      const int packed = cpk[q];
      if (!((packed >> (NODE_BITS + k)) & 1)) {
        T *dst = coarse + 3 * (size_t)(packed & NODE_MASK) + k;
        if (plain) *dst += s;
        else atomicAdd(dst, s);
      }
    }
    __syncwarp();
  }
}

// prolongation: fine += weight * P coarse (coarse Dirichlet entries read as
// zero); the same two-round-trip load order as the restriction
template <int P, typename T>
__global__ void prolongate_kernel(int n_coarse, const int *__restrict__ cells, int plain,
                                  const int *__restrict__ coarse_cn, const int *__restrict__ fine_nodes,
                                  const double *__restrict__ weight, const T *__restrict__ coarse, T *fine,
                                  Prol1D<P, T> pm) {
  constexpr int N1 = P + 1, NF = 2 * P + 1, NFB = NF * NF * NF, NCN = N1 * N1 * N1;
  constexpr int SZ = 3 * NCN + 3 * N1 * N1 * NF + 3 * N1 * NF * NF;
  constexpr int NPL = (NFB + 31) / 32, CPL = (3 * NCN + 31) / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  T *v = (T *)smem_raw + warp * SZ, *s1 = v + 3 * NCN, *s2 = s1 + 3 * N1 * N1 * NF;
  for (int ic = blockIdx.x * wpb + warp; ic < n_coarse; ic += gridDim.x * wpb) {
    const int c = cells ? __ldg(cells + ic) : ic;
    const int *fn = fine_nodes + (size_t)c * NFB;
    int node[NPL], cpk[CPL];
#pragma unroll
    for (int q = 0; q < NPL; ++q) node[q] = (lane + 32 * q < NFB) ? __ldg(fn + lane + 32 * q) : -1;
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int it = lane + 32 * q;
      cpk[q] = it < 3 * NCN ? __ldg(coarse_cn + (size_t)c * NCN + it % NCN) : 0;
    }
    T w[NPL], cv[CPL];
#pragma unroll
    for (int q = 0; q < NPL; ++q) w[q] = node[q] >= 0 ? T(__ldg(weight + node[q])) : T(0);
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int it = lane + 32 * q, k = it / NCN;
      cv[q] = (it < 3 * NCN && !((cpk[q] >> (NODE_BITS + k)) & 1))
                  ? coarse[3 * (size_t)(cpk[q] & NODE_MASK) + k] : T(0);
    }
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int it = lane + 32 * q;
      if (it < 3 * NCN) v[it] = cv[q];
    }
    __syncwarp();
    // x: s1[k][z][y][fx]
    for (int it = lane; it < 3 * N1 * N1 * NF; it += 32) {
      const int fx = it % NF, zy = it / NF;  // zy = (k*N1 + z)*N1 + y
      T s = 0;
#pragma unroll
      for (int x = 0; x < N1; ++x) s += pm.m[fx][x] * v[zy * N1 + x];
      s1[it] = s;
    }
    __syncwarp();
    // y: s2[k][z][fy][fx]
    for (int it = lane; it < 3 * N1 * NF * NF; it += 32) {
      const int fx = it % NF, fy = (it / NF) % NF, kz = it / (NF * NF);
      T s = 0;
#pragma unroll
      for (int y = 0; y < N1; ++y) s += pm.m[fy][y] * s1[(kz * N1 + y) * NF + fx];
      s2[it] = s;
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < NPL; ++q) {
      if (node[q] < 0) continue;
      const int l = lane + 32 * q, fyx = l % (NF * NF), fz = l / (NF * NF);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        T s = 0;
#pragma unroll
        for (int z = 0; z < N1; ++z) s += pm.m[fz][z] * s2[(k * N1 + z) * NF * NF + fyx];
        T *dst = fine + 3 * (size_t)node[q] + k;
        if (plain) *dst += w[q] * s;
        else atomicAdd(dst, w[q] * s);
      }
    }
    __syncwarp();
  }
}

// coarse displacement at the coarse nodes from the fine one (nested
// Lagrange spaces: evaluation of the fine field at the coarse support points)
template <typename T>
__global__ void interpolate_kernel(int n_coarse_nodes, int ncn, const int *__restrict__ icell,
                                   const double *__restrict__ iw, const int *__restrict__ fine_cn,
                                   const T *__restrict__ fine_u, T *coarse_u) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n_coarse_nodes; i += gridDim.x * blockDim.x) {
    const int node = i / 3, k = i % 3;
    const int fc = icell[node];
    const double *w = iw + (size_t)node * ncn;
    double s = 0;
    for (int a = 0; a < ncn; ++a) s += w[a] * (double)fine_u[3 * (size_t)(fine_cn[(size_t)fc * ncn + a] & NODE_MASK) + k];
    coarse_u[i] = T(s);
  }
}

// ------------------------------------------------------- residual (FP64)
// internal force per cell, -int tau : grad_x N dV (mf_elasticity.h:2760-2843
// rhs part), evaluated in the reference configuration:
//   H[c][f] = -sum_d tau[c][d] (J_ref^-1 F^-1)[f][d] JxW_ref
// MODE 0: scatter into R; MODE 1: grad[cell] = lambda . (cell vector)
template <int P, int Q, int MODE>
__global__ void __launch_bounds__(128) internal_force_kernel(const int *__restrict__ cell_nodes, int n_cells,
                                                              const int *__restrict__ cells, int plain,
                                                              const double *__restrict__ X, const double *__restrict__ u,
                                                              const double *__restrict__ mu_cell, double nu, int formulation,
                                                              double *R, const double *__restrict__ lam, double *grad,
                                                              TabT<P, Q, double> tab, Tab<P, Q> wtab) {
  using S = SFR<P, Q, double>;
  constexpr int N1 = P + 1, NN = S::NN, NQ = S::NQ, QPL = S::QPL, RPL = S::RPL, XR = S::XR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  double *slab = (double *)smem_raw + warp * S::SZ;
  for (int ic = blockIdx.x * wpb + warp; ic < n_cells; ic += gridDim.x * wpb) {
    const int cell = cells ? __ldg(cells + ic) : ic;
    const int *cn = cell_nodes + (size_t)cell * NN;
    int ck[RPL][N1];
    double vx[RPL][N1], vu[RPL][N1];
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = lane + 32 * r;
      const int comp = row < XR ? row / (N1 * N1) : 0, kj = row % (N1 * N1);
#pragma unroll
      for (int i = 0; i < N1; ++i) {
        if (row < XR) {
          const int packed = cn[kj * N1 + i];
          ck[r][i] = packed;
          const size_t dof = 3 * (size_t)(packed & NODE_MASK) + comp;
          vx[r][i] = X[dof];
          vu[r][i] = u[dof];
        } else {
          ck[r][i] = 0; vx[r][i] = 0; vu[r][i] = 0;
        }
      }
    }
    double GX[QPL][3][3], GU[QPL][3][3], H[QPL][3][3];
    S::eval(tab, vx, slab, lane, GX);
    S::eval(tab, vu, slab, lane, GU);
    const double mu = mu_cell[cell];
    const double lambda = (2.0 * mu * nu) / (1.0 - 2.0 * nu);
    const double kappa = (2.0 * mu * (1.0 + nu)) / (3.0 * (1.0 - 2.0 * nu));
#pragma unroll
    for (int l = 0; l < QPL; ++l) {
      const int q = lane + 32 * l;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 3; ++e) H[l][c][e] = 0;
      if (q >= NQ) continue;
      const double w = wtab.w[q % Q] * wtab.w[(q / Q) % Q] * wtab.w[q / (Q * Q)];
      double Jr[3][3], Jri[3][3], F[3][3], Fi[3][3];
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int e = 0; e < 3; ++e) Jr[d][e] = GX[l][d][e];
      const double jxw = inv3(Jr, Jri) * w;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d)
          F[c][d] = GU[l][c][0] * Jri[0][d] + GU[l][c][1] * Jri[1][d] + GU[l][c][2] * Jri[2][d] + (c == d ? 1.0 : 0.0);
      const double det = inv3(F, Fi);
      double b[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
      double tau[3][3];
      if (formulation == 0) {
        // material.h:119-150: tau = (J dPsi_vol/dJ - tr(tau_bar)/3) I + tau_bar
        const double s = pow(det, -2.0 / 3.0);
        const double dPsi = (kappa / 2.0) * (det - 1.0 / det);
        double tr = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i) tr += b[i][i] * s * mu;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) tau[i][j] = b[i][j] * s * mu + (i == j ? dPsi * det - tr / 3.0 : 0.0);
      } else {
        // material.h:151-158: tau = mu b - (mu - 2 lambda ln J) I
        const double tmp = mu - 2.0 * lambda * log(det);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) tau[i][j] = mu * b[i][j] - (i == j ? tmp : 0.0);
      }
      double JF[3][3];
#pragma unroll
      for (int f = 0; f < 3; ++f)
#pragma unroll
        for (int d = 0; d < 3; ++d) JF[f][d] = Jri[f][0] * Fi[0][d] + Jri[f][1] * Fi[1][d] + Jri[f][2] * Fi[2][d];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int f = 0; f < 3; ++f)
          H[l][c][f] = -(tau[c][0] * JF[f][0] + tau[c][1] * JF[f][1] + tau[c][2] * JF[f][2]) * jxw;
    }
    double out[RPL][N1];
    S::integrate(tab, H, slab, lane, out);
    double acc = 0;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = lane + 32 * r;
      if (row >= XR) continue;
      const int comp = row / (N1 * N1);
#pragma unroll
      for (int i = 0; i < N1; ++i) {
        const size_t dof = 3 * (size_t)(ck[r][i] & NODE_MASK) + comp;
        if (MODE == 0) {
          if (plain) R[dof] += out[r][i];
          else atomicAdd(R + dof, out[r][i]);
        }
        else acc += lam[dof] * out[r][i];
      }
    }
    if (MODE == 1) {
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
      if (lane == 0) grad[cell] = acc;
    }
  }
}

int g_sms = 0;
int sms() {
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  return g_sms;
}
inline int vec_grid(size_t n) {
  const size_t b = (n + 255) / 256;
  const size_t cap = (size_t)8 * sms();
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

int reduce_blocks() { return 4 * sms(); }

lsmf_status dot_async(const void *a, const void *b, bool fp32, size_t n, double *partial, double *sc, int slot,
                      cudaStream_t st) {
  const int g = reduce_blocks();
  if (fp32) dot_partial_kernel<float, float><<<g, RED_THREADS, 0, st>>>((const float *)a, (const float *)b, n, partial);
  else dot_partial_kernel<double, double><<<g, RED_THREADS, 0, st>>>((const double *)a, (const double *)b, n, partial);
  reduce_final_kernel<<<1, 1024, 0, st>>>(partial, g, sc + slot);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

lsmf_status cg_update_async(double *x, double *g, const double *d, const double *h, size_t n, double *sc, int gh_slot,
                            double *partial, cudaStream_t st) {
  const int gr = reduce_blocks();
  cg_update_kernel<<<gr, RED_THREADS, 0, st>>>(x, g, d, h, n, sc, gh_slot, partial);
  reduce_final_kernel<<<1, 1024, 0, st>>>(partial, gr, sc + SC_RES2);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

template <typename T>
lsmf_status eig_dh_async(const T *d, T *h, const uint8_t *cmask, size_t n, double *partial, double *sc,
                         cudaStream_t st) {
  const int gr = reduce_blocks();
  eig_dh_kernel<T><<<gr, RED_THREADS, 0, st>>>(d, h, cmask, n, partial, vec_ok<T>({d, h}, cmask));
  reduce_final_kernel<<<1, 1024, 0, st>>>(partial, gr, sc + SC_DH);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status eig_dh_async<float>(const float *, float *, const uint8_t *, size_t, double *, double *,
                                         cudaStream_t);
template lsmf_status eig_dh_async<double>(const double *, double *, const uint8_t *, size_t, double *, double *,
                                          cudaStream_t);

template <typename T>
lsmf_status eig_update_precond_async(T *g, T *h, const T *invd, size_t n, double *sc, int gh_slot, int gh_new,
                                     double *hist_alpha, double *hist_res2, int k, const int *kbase, double *partial,
                                     cudaStream_t st) {
  const int gr = reduce_blocks();
  eig_update_precond_kernel<T><<<gr, RED_THREADS, 0, st>>>(g, h, invd, n, sc, gh_slot, hist_alpha, k, kbase, partial,
                                                           partial + gr, vec_ok<T>({g, h, invd}, nullptr));
  reduce2_final_kernel<<<1, 1024, 0, st>>>(partial, partial + gr, gr, hist_res2 + k, kbase, sc + gh_new);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status eig_update_precond_async<float>(float *, float *, const float *, size_t, double *, int, int,
                                                     double *, double *, int, const int *, double *, cudaStream_t);
template lsmf_status eig_update_precond_async<double>(double *, double *, const double *, size_t, double *, int, int,
                                                      double *, double *, int, const int *, double *, cudaStream_t);

template <typename T>
lsmf_status eig_dir_clear_async(T *d, T *h, size_t n, const double *sc, int gh_new, int gh_old, double *hist_beta, int k,
                                const int *kbase, cudaStream_t st) {
  const int vec = vec_ok<T>({d, h}, nullptr);
  eig_dir_clear_kernel<T><<<vec_grid(vec ? (n + Vec16<T>::W - 1) / Vec16<T>::W : n), 256, 0, st>>>(
      d, h, n, sc, gh_new, gh_old, hist_beta, k, kbase, vec);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status eig_dir_clear_async<float>(float *, float *, size_t, const double *, int, int, double *, int,
                                                const int *, cudaStream_t);
template lsmf_status eig_dir_clear_async<double>(double *, double *, size_t, const double *, int, int, double *, int,
                                                 const int *, cudaStream_t);

lsmf_status eig_advance_async(int *kbase, int by, cudaStream_t st) {
  eig_advance_kernel<<<1, 1, 0, st>>>(kbase, by);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

template <typename T>
lsmf_status eig_start_async(T *g, size_t n, double mean, cudaStream_t st) {
  eig_start_kernel<T><<<vec_grid(n), 256, 0, st>>>(g, n, mean);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status eig_start_async<float>(float *, size_t, double, cudaStream_t);
template lsmf_status eig_start_async<double>(double *, size_t, double, cudaStream_t);

lsmf_status cg_dir_async(double *d, const double *h, size_t n, const double *sc, int gh_new, int gh_old, bool first,
                         cudaStream_t st) {
  cg_dir_kernel<<<vec_grid(n), 256, 0, st>>>(d, h, n, sc, gh_new, gh_old, first ? 1 : 0);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

template <typename T>
lsmf_status neg_residual_async(T *g, const T *ax, const T *b, size_t n, cudaStream_t st) {
  residual_init_kernel<T><<<vec_grid(n), 256, 0, st>>>(g, ax, b, n);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status neg_residual_async<float>(float *, const float *, const float *, size_t, cudaStream_t);
template lsmf_status neg_residual_async<double>(double *, const double *, const double *, size_t, cudaStream_t);

template <typename T>
lsmf_status jacobi_async(T *dst, const T *invd, const T *src, double omega, size_t n, cudaStream_t st) {
  scaled_mul_kernel2<T><<<vec_grid(n), 256, 0, st>>>(dst, invd, src, T(omega), n);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status jacobi_async<float>(float *, const float *, const float *, double, size_t, cudaStream_t);
template lsmf_status jacobi_async<double>(double *, const double *, const double *, double, size_t, cudaStream_t);

template <typename TD, typename TS>
lsmf_status convert_async(TD *dst, const TS *src, size_t n, cudaStream_t st) {
  convert_kernel<TD, TS><<<vec_grid(n), 256, 0, st>>>(dst, src, n);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status convert_async<float, double>(float *, const double *, size_t, cudaStream_t);
template lsmf_status convert_async<double, float>(double *, const float *, size_t, cudaStream_t);
template lsmf_status convert_async<double, double>(double *, const double *, size_t, cudaStream_t);
template lsmf_status convert_async<float, float>(float *, const float *, size_t, cudaStream_t);

template <typename T>
lsmf_status axpy_async(T *y, double a, const T *x, size_t n, cudaStream_t st) {
  axpy_kernel<T><<<vec_grid(n), 256, 0, st>>>(y, T(a), x, n);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status axpy_async<float>(float *, double, const float *, size_t, cudaStream_t);
template lsmf_status axpy_async<double>(double *, double, const double *, size_t, cudaStream_t);

template <typename T>
lsmf_status dir_async(T *d, const T *h, double beta, size_t n, cudaStream_t st) {
  dir_kernel<T><<<vec_grid(n), 256, 0, st>>>(d, h, beta, n);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status dir_async<float>(float *, const float *, double, size_t, cudaStream_t);
template lsmf_status dir_async<double>(double *, const double *, double, size_t, cudaStream_t);

template <typename T>
lsmf_status set_indexed_async(T *v, const int *idx, int n, double val, cudaStream_t st) {
  if (n <= 0) return LSMF_OK;
  set_indexed_kernel<T><<<vec_grid(n), 256, 0, st>>>(v, idx, n, T(val));
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status set_indexed_async<float>(float *, const int *, int, double, cudaStream_t);
template lsmf_status set_indexed_async<double>(double *, const int *, int, double, cudaStream_t);

template <typename T>
lsmf_status copy_indexed_async(T *dst, const T *src, const int *idx, int n, cudaStream_t st) {
  if (n <= 0) return LSMF_OK;
  copy_indexed_kernel<T><<<vec_grid(n), 256, 0, st>>>(dst, src, idx, n);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status copy_indexed_async<double>(double *, const double *, const int *, int, cudaStream_t);

template <typename T>
lsmf_status cheb_zero_async(T *x, const T *b, const T *invd, double theta, size_t n, cudaStream_t st) {
  const int vec = vec_ok<T>({x, b, invd}, nullptr);
  cheb_zero_kernel<T><<<vec_grid(vec ? (n + Vec16<T>::W - 1) / Vec16<T>::W : n), 256, 0, st>>>(x, b, invd, 1.0 / theta,
                                                                                            n, vec);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template <typename T>
lsmf_status cheb_first_async(T *x, T *xold, const T *b, T *r, const T *invd, const uint8_t *cmask, double theta,
                             size_t n, cudaStream_t st) {
  const int vec = vec_ok<T>({x, xold, b, r, invd}, cmask);
  cheb_first_kernel<T><<<vec_grid(vec ? (n + Vec16<T>::W - 1) / Vec16<T>::W : n), 256, 0, st>>>(
      x, xold, b, r, invd, cmask, 1.0 / theta, n, vec);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template <typename T>
lsmf_status cheb_step_async(T *x, T *xold, const T *b, T *r, const T *invd, const uint8_t *cmask, double f1, double f2,
                            bool has_old, size_t n, cudaStream_t st) {
  // one thread per 16-byte vector (the grid covers the vectors, not the values)
  const int vec = vec_ok<T>({x, xold, b, r, invd}, cmask);
  cheb_step_kernel<T><<<vec_grid(vec ? (n + Vec16<T>::W - 1) / Vec16<T>::W : n), 256, 0, st>>>(
      x, xold, b, r, invd, cmask, f1, f2, has_old ? 1 : 0, n, vec);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status cheb_zero_async<float>(float *, const float *, const float *, double, size_t, cudaStream_t);
template lsmf_status cheb_zero_async<double>(double *, const double *, const double *, double, size_t, cudaStream_t);
template lsmf_status cheb_first_async<float>(float *, float *, const float *, float *, const float *, const uint8_t *,
                                             double, size_t, cudaStream_t);
template lsmf_status cheb_first_async<double>(double *, double *, const double *, double *, const double *,
                                              const uint8_t *, double, size_t, cudaStream_t);
template lsmf_status cheb_step_async<float>(float *, float *, const float *, float *, const float *, const uint8_t *,
                                            double, double, bool, size_t, cudaStream_t);
template lsmf_status cheb_step_async<double>(double *, double *, const double *, double *, const double *,
                                             const uint8_t *, double, double, bool, size_t, cudaStream_t);

template <int P, typename C>
static Prol1D<P, C> make_prol(const TransferMap &T) {
  Prol1D<P, C> pm;
  for (int f = 0; f < 2 * P + 1; ++f)
    for (int x = 0; x <= P; ++x) pm.m[f][x] = C(T.P1[f * (P + 1) + x]);
  return pm;
}

// Run f(cells, n, plain) over all cells of L (atomics), or with the colour8
// scatter once per lattice colour in the order 0..7 (plain adds).
template <typename F>
static lsmf_status over_colours(const Level &L, int scatter, F &&f) {
  // colour8 and nodesum (whose node sums serve only the vmult) both run the
  // deterministic colours here
  if (scatter != LSMF_SCATTER_ATOMIC) {
    for (int c = 0; c < 8; ++c) {
      const int n = L.colour_off[c + 1] - L.colour_off[c];
      if (n > 0) LSMF_TRY(f(L.d_colour_cells.ptr + L.colour_off[c], n, 1));
    }
    return LSMF_OK;
  }
  return f((const int *)nullptr, L.n_cells, 0);
}

template <typename T, int P>
static lsmf_status transfer_impl(bool restrict_dir, const Level &C, const TransferMap &TM, const T *b, const T *r,
                                 T *coarse_or_fine, const T *coarse_src, int scatter, cudaStream_t st) {
  constexpr int N1 = P + 1, NF = 2 * P + 1;
  const int wpb = 4;
  const Prol1D<P, T> pm = make_prol<P, T>(TM);
  if (restrict_dir) {
    constexpr int SZ = 3 * NF * NF * NF + 3 * NF * NF * N1 + 3 * NF * N1 * N1;
    const size_t smem = sizeof(T) * SZ * wpb;
    auto k = restrict_kernel<P, T>;
    LSMF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LSMF_TRY(over_colours(C, scatter, [&](const int *cells, int n, int plain) -> lsmf_status {
      int g = (n + wpb - 1) / wpb;
      if (g > 16 * sms()) g = 16 * sms();
      k<<<g, 32 * wpb, smem, st>>>(n, cells, plain, C.d_cell_nodes.ptr, TM.d_fine_nodes.ptr, TM.d_weight.ptr, b, r,
                                    coarse_or_fine, pm);
      return LSMF_OK;
    }));
  } else {
    constexpr int SZ = 3 * N1 * N1 * N1 + 3 * N1 * N1 * NF + 3 * N1 * NF * NF;
    const size_t smem = sizeof(T) * SZ * wpb;
    auto k = prolongate_kernel<P, T>;
    LSMF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LSMF_TRY(over_colours(C, scatter, [&](const int *cells, int n, int plain) -> lsmf_status {
      int g = (n + wpb - 1) / wpb;
      if (g > 16 * sms()) g = 16 * sms();
      k<<<g, 32 * wpb, smem, st>>>(n, cells, plain, C.d_cell_nodes.ptr, TM.d_fine_nodes.ptr, TM.d_weight.ptr,
                                    coarse_src, coarse_or_fine, pm);
      return LSMF_OK;
    }));
  }
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

template <typename T>
lsmf_status restrict_add_async(const Level &C, const TransferMap &TM, const T *b, const T *r, T *coarse, int scatter,
                               cudaStream_t st) {
  switch (C.p) {
    case 1: return transfer_impl<T, 1>(true, C, TM, b, r, coarse, nullptr, scatter, st);
    case 2: return transfer_impl<T, 2>(true, C, TM, b, r, coarse, nullptr, scatter, st);
    case 3: return transfer_impl<T, 3>(true, C, TM, b, r, coarse, nullptr, scatter, st);
    case 4: return transfer_impl<T, 4>(true, C, TM, b, r, coarse, nullptr, scatter, st);
  }
  return LSMF_ERR_UNSUPPORTED;
}
template <typename T>
lsmf_status prolongate_add_async(const Level &C, const TransferMap &TM, const T *coarse, T *fine, int scatter,
                                 cudaStream_t st) {
  switch (C.p) {
    case 1: return transfer_impl<T, 1>(false, C, TM, nullptr, nullptr, fine, coarse, scatter, st);
    case 2: return transfer_impl<T, 2>(false, C, TM, nullptr, nullptr, fine, coarse, scatter, st);
    case 3: return transfer_impl<T, 3>(false, C, TM, nullptr, nullptr, fine, coarse, scatter, st);
    case 4: return transfer_impl<T, 4>(false, C, TM, nullptr, nullptr, fine, coarse, scatter, st);
  }
  return LSMF_ERR_UNSUPPORTED;
}
template lsmf_status restrict_add_async<float>(const Level &, const TransferMap &, const float *, const float *, float *,
                                               int, cudaStream_t);
template lsmf_status restrict_add_async<double>(const Level &, const TransferMap &, const double *, const double *,
                                                double *, int, cudaStream_t);
template lsmf_status prolongate_add_async<float>(const Level &, const TransferMap &, const float *, float *, int,
                                                 cudaStream_t);
template lsmf_status prolongate_add_async<double>(const Level &, const TransferMap &, const double *, double *, int,
                                                  cudaStream_t);

template <typename T>
lsmf_status interpolate_async(const Level &C, const Level &F, const TransferMap &TM, const T *fine_u, T *coarse_u,
                              cudaStream_t st) {
  interpolate_kernel<T><<<vec_grid(3 * (size_t)C.n_nodes), 256, 0, st>>>(
      C.n_nodes, C.ncn(), TM.d_interp_cell.ptr, TM.d_interp_w.ptr, F.d_cell_nodes.ptr, fine_u, coarse_u);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
template lsmf_status interpolate_async<float>(const Level &, const Level &, const TransferMap &, const float *, float *,
                                              cudaStream_t);
template lsmf_status interpolate_async<double>(const Level &, const Level &, const TransferMap &, const double *,
                                               double *, cudaStream_t);

template <int P, int Q, int MODE>
static lsmf_status internal_force_impl(const Level &L, const Basis &B, const double *u, const double *mu, double nu,
                                       int formulation, double *R, const double *lam, double *grad, int scatter,
                                       cudaStream_t st) {
  using S = SFR<P, Q, double>;
  TabT<P, Q, double> t;
  Tab<P, Q> w;
  for (int k = 0; k < Q; ++k) {
    for (int i = 0; i <= P; ++i) {
      t.N[k][i] = B.N[k * (P + 1) + i];
      t.D[k][i] = B.D[k * (P + 1) + i];
      w.N[k][i] = t.N[k][i];
      w.D[k][i] = t.D[k][i];
    }
    w.w[k] = B.qw[k];
  }
  const int wpb = 4;
  const size_t smem = sizeof(double) * S::SZ * wpb;
  auto k = internal_force_kernel<P, Q, MODE>;
  LSMF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  // the cell gradient (MODE 1) writes one value per cell and needs no colours
  LSMF_TRY(over_colours(L, MODE == 0 ? scatter : LSMF_SCATTER_ATOMIC,
                        [&](const int *cells, int n, int plain) -> lsmf_status {
                          int g = (n + wpb - 1) / wpb;
                          if (g > 16 * sms()) g = 16 * sms();
                          k<<<g, 32 * wpb, smem, st>>>(L.d_cell_nodes.ptr, n, cells, plain, L.d_X.ptr, u, mu, nu,
                                                        formulation, R, lam, grad, t, w);
                          return LSMF_OK;
                        }));
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

// R += -f_int(u) (caller initialises R with the external load)
lsmf_status internal_force_async(const Level &L, const Basis &B, const double *u, const double *mu, double nu,
                                 int formulation, double *R, int scatter, cudaStream_t st) {
  switch (L.p) {
    case 1: return internal_force_impl<1, 2, 0>(L, B, u, mu, nu, formulation, R, nullptr, nullptr, scatter, st);
    case 2: return internal_force_impl<2, 3, 0>(L, B, u, mu, nu, formulation, R, nullptr, nullptr, scatter, st);
    case 3: return internal_force_impl<3, 4, 0>(L, B, u, mu, nu, formulation, R, nullptr, nullptr, scatter, st);
    case 4: return internal_force_impl<4, 5, 0>(L, B, u, mu, nu, formulation, R, nullptr, nullptr, scatter, st);
  }
  return LSMF_ERR_UNSUPPORTED;
}
// grad[c] = lambda . (-f_int of cell c)
lsmf_status adjoint_cell_grad_async(const Level &L, const Basis &B, const double *u, const double *mu, double nu,
                                    int formulation, const double *lam, double *grad, cudaStream_t st) {
  switch (L.p) {
    case 1: return internal_force_impl<1, 2, 1>(L, B, u, mu, nu, formulation, nullptr, lam, grad, LSMF_SCATTER_ATOMIC, st);
    case 2: return internal_force_impl<2, 3, 1>(L, B, u, mu, nu, formulation, nullptr, lam, grad, LSMF_SCATTER_ATOMIC, st);
    case 3: return internal_force_impl<3, 4, 1>(L, B, u, mu, nu, formulation, nullptr, lam, grad, LSMF_SCATTER_ATOMIC, st);
    case 4: return internal_force_impl<4, 5, 1>(L, B, u, mu, nu, formulation, nullptr, lam, grad, LSMF_SCATTER_ATOMIC, st);
  }
  return LSMF_ERR_UNSUPPORTED;
}

}  // namespace lsmf
