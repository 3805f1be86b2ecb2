// sm_100a kernel templates of the matrix-free tangent operator, shared by
// the per-degree / per-precision instantiation units op_p<P>_<f64|f32>.cu:
//   cache_kernel       NeoHookOperator::cache + Eulerian MatrixFree metric
//   apply_kernel       NeoHookOperator::vmult_add cell loop, basic form with
//                      the MFMask stage switches
//   apply_fast_kernel  the production vmult cell loop
//   diagonal_kernel    NeoHookOperator::compute_diagonal
// Every cell loop runs either over all cells with atomic scatter, or over
// one colour of the lattice (a list of cells no two of which share a node)
// with plain read-modify-write scatter; the host launches the 8 colours in
// order for a bit-reproducible result.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "cell_kernels.cuh"
#include "lsmf_internal.h"
#include "op_dispatch.h"
#include "pair.cuh"

namespace lsmf {

namespace {

template <typename T>
struct KArgs {
  const int *cell_nodes;
  int n_cells;
  int ncomp;
  int rec_elems;         // values per cell record
  int ref_per_cell;      // scalar caching: reference inverse Jacobian once per cell
  T *table;              // cache records (written by cache, read by apply/diag)
  const T *src;
  T *dst;
  const T *u;            // displacement (operator precision)
  const double *X;       // reference coordinates
  const double *mu;      // per cell
  double nu;
  int *flag;             // device error word
  unsigned mask;
  int wait_tries;        // try_wait calls before a bulk-copy wait gives up
  int prefetch;          // plain loads: L1 prefetch of the record (0 off, 1 this cell, 2 the next cell)
  const int *cells;      // cell list of one colour (nullptr: all n_cells cells)
  int plain;             // scatter with plain adds (colour launches) instead of atomics
  T *cellbuf;            // node-sum scatter: per-cell results [cell][local node][component]
  // fused interface exchange (SC_PEER): the neighbour part's vectors, read
  // and added to for the nodes with PEER_BIT in cell_nodes
  const T *psrc;
  T *pdst;
  const T *pu;
  int cell0;             // first cell of a contiguous chunk (cell list absent)
};

// cell of list entry i
template <typename T>
__device__ __forceinline__ int cell_of(const KArgs<T> &a, int i) { return a.cells ? __ldg(a.cells + i) : a.cell0 + i; }
template <typename T>
__device__ __forceinline__ void scatter_add(T *p, T v, bool plain) {
  if (plain) *p += v;
  else atomicAdd(p, v);
}

template <int P, int Q, typename T>
__device__ __forceinline__ void load_tables(const Tab<P, Q> &tab, T *sN, T *sD) {
  constexpr int N1 = P + 1;
  for (int i = threadIdx.x; i < Q * N1; i += blockDim.x) {
    sN[i] = T(tab.N[i / N1][i % N1]);
    sD[i] = T(tab.D[i / N1][i % N1]);
  }
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ void material(double mu_d, double nu, T &mu, T &lambda, T &kappa) {
  // material.h:82-94
  mu = T(mu_d);
  lambda = T((2.0 * mu_d * nu) / (1.0 - 2.0 * nu));
  kappa = T((2.0 * mu_d * (1.0 + nu)) / (3.0 * (1.0 - 2.0 * nu)));
}

// gather a 3-component field of a cell into V[c*NN + a]
template <int NN, typename TS, typename TD>
__device__ __forceinline__ void gather(const int *__restrict__ cn, const TS *__restrict__ vec, bool zero_constr,
                                       TD *V, int lane) {
  for (int a = lane; a < NN; a += 32) {
    const int packed = __ldg(cn + a);
    const int node = packed & NODE_MASK;
    const int cm = zero_constr ? (packed >> NODE_BITS) : 0;
    const TS *v = vec + 3 * (size_t)node;
    V[a] = (cm & 1) ? TD(0) : TD(__ldg(v));
    V[NN + a] = (cm & 2) ? TD(0) : TD(__ldg(v + 1));
    V[2 * NN + a] = (cm & 4) ? TD(0) : TD(__ldg(v + 2));
  }
  __syncwarp();
}

template <typename T>
__device__ __forceinline__ void atomic_add(T *a, T v) { atomicAdd(a, v); }

// ------------------------------------------------ bulk-copy (TMA) helpers
// One-dimensional cp.async.bulk from this GPU's global memory into the
// issuing CTA's own shared memory with mbarrier completion (no tensor map):
// each cell record is one contiguous, 16-byte aligned block of
// ncomp * Q^3 values.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ uint64_t evict_first_policy() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: try_wait suspends for a hardware time slice per call, so
// 2^22 calls are seconds; a wait that runs out reports failure instead of
// spinning forever
constexpr int WAIT_TRIES_DEFAULT = 1 << 22;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int tries = WAIT_TRIES_DEFAULT) {
  for (int i = 0; i < tries; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// device error word bits: det F <= 0 at a point (cache), a bounded wait
// ran out, a kernel found less dynamic shared memory than its layout needs
// (it returned without touching memory)
constexpr int FLAG_DETF = 1, FLAG_TIMEOUT = 2, FLAG_SMEM = 4;
// internal stage bit: gather constrained entries instead of zeroing them
constexpr unsigned MASK_INHOM = MASK_INHOM_BIT;

// ------------------------------------------------------------ cache kernel
template <int P, int Q, typename T, int VAR>
__global__ void __launch_bounds__(256) cache_kernel(KArgs<T> a, Tab<P, Q> tab) {
  using S = SF<P, Q, double>;
  constexpr int NN = S::NN, NQ = S::NQ, QPL = S::QPL;
  const int WPB = blockDim.x >> 5;
  extern __shared__ __align__(16) unsigned char smem[];
  double *sN = (double *)smem, *sD = sN + Q * (P + 1);
  load_tables<P, Q, double>(tab, sN, sD);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *slab = sD + Q * (P + 1) + warp * S::SZ;
  double *V = slab, *A = slab + S::SZ1, *B = A + S::SZ2;
  const int gw = blockIdx.x * WPB + warp, nw = gridDim.x * WPB;
  int bad = 0;
  for (int cell = gw; cell < a.n_cells; cell += nw) {
    const int *cn = a.cell_nodes + (size_t)cell * NN;
    double GX[QPL][3][3], GU[QPL][3][3];
    gather<NN>(cn, a.X, false, V, lane);
    S::eval(sN, sD, V, A, B, lane, GX);
    gather<NN>(cn, a.u, false, V, lane);
    S::eval(sN, sD, V, A, B, lane, GU);
    const double mu = a.mu[cell];
    const double lambda = (2.0 * mu * a.nu) / (1.0 - 2.0 * a.nu);
    T *rec = a.table + (size_t)cell * a.rec_elems;
#pragma unroll
    for (int l = 0; l < QPL; ++l) {
      const int q = lane + 32 * l;
      if (q >= NQ) continue;
      const double w = tab.w[q % Q] * tab.w[(q / Q) % Q] * tab.w[q / (Q * Q)];
      double Jr[3][3], Jc[3][3], Jri[3][3], Jci[3][3];
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          Jr[d][e] = GX[l][d][e];
          Jc[d][e] = GX[l][d][e] + GU[l][d][e];
        }
      inv3(Jr, Jri);
      const double dc = inv3(Jc, Jci);
      T *r = rec + q;
      // scalar_referential / tensor4_ns integrate in the reference frame
      const double jxw = variant_referential(VAR) ? det3(Jr) * w : dc * w;
#pragma unroll
      for (int i = 0; i < 9; ++i)
        r[(C_JINV + i) * NQ] = T(variant_referential(VAR) ? Jri[i / 3][i % 3] : Jci[i / 3][i % 3]);
      // tensor4 / tensor2 / tensor4_ns store their coefficients times JxW
      constexpr int CV = variant_cvar(VAR);
      const double fw = variant_folds_jxw(VAR) ? jxw : 1.0;
      if (!variant_folds_jxw(VAR)) r[C_JXW * NQ] = T(jxw);
      // F = I + Grad u (reference configuration, mf_nh_operator.h:462-476)
      double F[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d)
          F[c][d] = GU[l][c][0] * Jri[0][d] + GU[l][c][1] * Jri[1][d] + GU[l][c][2] * Jri[2][d] + (c == d ? 1.0 : 0.0);
      const double det_F = det3(F);
      if (!(det_F > 0.0)) bad = 1;
      if (VAR == VAR_SCALAR_F0 || VAR == VAR_SCALAR_F1) {
        const double c = (VAR == VAR_SCALAR_F0) ? pow(det_F, -1.0 / 3.0) : mu - 2.0 * lambda * log(det_F);
        r[C_VAR * NQ] = T(c);
        if (a.ref_per_cell) {
          // affine cell: the reference metric of the first point stands for all
          if (q == 0)
#pragma unroll
            for (int i = 0; i < 9; ++i) rec[(C_VAR + 1) * NQ + i] = T(Jri[i / 3][i % 3]);
        } else {
#pragma unroll
          for (int i = 0; i < 9; ++i) r[(C_VAR + 1 + i) * NQ] = T(Jri[i / 3][i % 3]);
        }
        continue;
      }
      const double scalar = mu - 2.0 * lambda * log(det_F);
      if (VAR == VAR_SCALAR_REF) {
        // c and the displacement values at the point (phi_reference.begin_values())
        r[C_VAR * NQ] = T(scalar);
        const int qx = q % Q, qy = (q / Q) % Q, qz = q / (Q * Q);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double v = 0;
          for (int kz = 0; kz <= P; ++kz)
            for (int jy = 0; jy <= P; ++jy)
              for (int ix = 0; ix <= P; ++ix)
                v += sN[qx * (P + 1) + ix] * sN[qy * (P + 1) + jy] * sN[qz * (P + 1) + kz] *
                     V[c * NN + (kz * (P + 1) + jy) * (P + 1) + ix];
          r[(C_VAR + 1 + c) * NQ] = T(v);
        }
        continue;
      }
      if (VAR == VAR_TENSOR4_NS) {
        // 2 lambda F^-T (x) F^-T + (mu - 2 lambda ln J) F^-T_il F^-1_jk + mu I_ik I_jl
        double Fi[3][3];
        inv3(F, Fi);
        const double lnJ = log(det_F);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
              for (int l = 0; l < 3; ++l)
                r[(CV + ((i * 3 + j) * 3 + k) * 3 + l) * NQ] =
                    T(fw * (2.0 * lambda * Fi[j][i] * Fi[l][k] + (mu - 2.0 * lambda * lnJ) * Fi[l][i] * Fi[j][k] +
                            (i == k && j == l ? mu : 0.0)));
        continue;
      }
      const double idet = 1.0 / det_F;
      double tau[6];
#pragma unroll
      for (int I = 0; I < 6; ++I) {
        const int i = sym_i(I), j = sym_j(I);
        const double b = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
        tau[I] = mu * b - (i == j ? scalar : 0.0);
      }
      if (VAR == VAR_TENSOR2) {
        r[CV * NQ] = T(fw * scalar * 2.0 * idet);
        r[(CV + 1) * NQ] = T(fw * 2.0 * lambda * idet);
#pragma unroll
        for (int I = 0; I < 6; ++I) r[(CV + 2 + I) * NQ] = T(fw * tau[I] * idet);
      } else {
#pragma unroll
        for (int I = 0; I < 6; ++I) r[(CV + I) * NQ] = T(fw * tau[I] * idet);
        // C = (2c/J) S + (2 lambda/J) I (x) I  (mf_nh_operator.h:542-546)
        const double ca = scalar * 2.0 * idet, cb = lambda * 2.0 * idet;
#pragma unroll
        for (int I = 0; I < 6; ++I)
#pragma unroll
          for (int J = 0; J < 6; ++J)
            r[(CV + 6 + I * 6 + J) * NQ] = T(fw * ((I == J ? ca : 0.0) + (I < 3 && J < 3 ? cb : 0.0)));
      }
    }
    __syncwarp();
  }
  if (bad) atomicOr(a.flag, 1);
}

// ------------------------------------------------------------ apply kernel
// FULL: all MFMask stages (the production path); otherwise stage bits of
// a.mask switch RW / SF / QD on and off like vmult<mask> for breakdowns.
template <int P, int Q, typename T, int VAR, bool FULL>
__global__ void __launch_bounds__(256) apply_kernel(KArgs<T> a, Tab<P, Q> tab) {
  using S = SF<P, Q, T>;
  constexpr int NN = S::NN, NQ = S::NQ, QPL = S::QPL;
  const int WPB = blockDim.x >> 5;
  constexpr bool SCALAR = (VAR == VAR_SCALAR_F0 || VAR == VAR_SCALAR_F1);
  extern __shared__ __align__(16) unsigned char smem[];
  T *sN = (T *)smem, *sD = sN + Q * (P + 1);
  load_tables<P, Q, T>(tab, sN, sD);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T *slab = sD + Q * (P + 1) + warp * S::SZ;
  T *V = slab, *A = slab + S::SZ1, *B = A + S::SZ2;
  const int gw = blockIdx.x * WPB + warp, nw = gridDim.x * WPB;
  const bool rw = FULL || (a.mask & LSMF_MASK_RW), sf = FULL || (a.mask & LSMF_MASK_SF),
             qd = FULL || (a.mask & LSMF_MASK_QD);
  for (int ic = gw; ic < a.n_cells; ic += nw) {
    const int cell = cell_of(a, ic);
    const int *cn = a.cell_nodes + (size_t)cell * NN;
    const T *rec = a.table + (size_t)cell * a.rec_elems;
    T G[QPL][3][3], GU[QPL][3][3];
    if (SCALAR) {
      if (rw) gather<NN>(cn, a.u, false, V, lane);   // read_dof_values_plain(u)
      if (sf) S::eval(sN, sD, V, A, B, lane, GU);
    }
    if (rw) gather<NN>(cn, a.src, !(a.mask & MASK_INHOM), V, lane);  // read_dof_values(src)
    else {
      for (int i = lane; i < 3 * NN; i += 32) V[i] = T(0);
      __syncwarp();
    }
    if (sf) S::eval(sN, sD, V, A, B, lane, G);
    else {
#pragma unroll
      for (int l = 0; l < QPL; ++l)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int e = 0; e < 3; ++e) G[l][c][e] = T(0);
    }
    T mu = 0, lambda = 0, kappa = 0;
    if (SCALAR || VAR == VAR_SCALAR_REF) material<T>(a.mu[cell], a.nu, mu, lambda, kappa);
    T H[QPL][3][3];
#pragma unroll
    for (int l = 0; l < QPL; ++l) {
      const int q = lane + 32 * l;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 3; ++e) H[l][c][e] = T(0);
      if (q >= NQ || !qd) continue;
      const T *r = rec + q;
      T Ji[3][3];
#pragma unroll
      for (int i = 0; i < 9; ++i) Ji[i / 3][i % 3] = r[(C_JINV + i) * NQ];
      const T jxw = variant_folds_jxw(VAR) ? T(1) : T(r[C_JXW * NQ]);
      T g[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[c][d] = G[l][c][0] * Ji[0][d] + G[l][c][1] * Ji[1][d] + G[l][c][2] * Ji[2][d];
      ScalarState<T> st;
      if (SCALAR) {
        T Jr[3][3];
#pragma unroll
        for (int i = 0; i < 9; ++i)
          Jr[i / 3][i % 3] = a.ref_per_cell ? rec[(C_VAR + 1) * NQ + i] : r[(C_VAR + 1 + i) * NQ];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int d = 0; d < 3; ++d)
            st.F[c][d] = GU[l][c][0] * Jr[0][d] + GU[l][c][1] * Jr[1][d] + GU[l][c][2] * Jr[2][d] + (c == d ? T(1) : T(0));
        st.det = det3(st.F);
      }
      if (VAR == VAR_SCALAR_REF) {
        collocation_F<Q>(rec, q, tab.Dc, Ji, st.F);
        st.det = det3(st.F);
      }
      T Qm[3][3];
      physics<T, VAR, NQ>(g, r, mu, lambda, kappa, st, Qm);
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          const T h = Qm[c][0] * Ji[e][0] + Qm[c][1] * Ji[e][1] + Qm[c][2] * Ji[e][2];
          H[l][c][e] = variant_folds_jxw(VAR) ? h : T(h * jxw);
        }
    }
    if (sf) {
      S::integrate(sN, sD, H, V, A, B, lane);
    } else {
      for (int i = lane; i < S::SZ2; i += 32) A[i] = T(0);
      __syncwarp();
    }
    if (rw) {
      for (int an = lane; an < NN; an += 32) {
        T o[3];
        S::integrate_node(sN, sD, A, an, o);
        const int packed = __ldg(cn + an);
        const int node = packed & NODE_MASK, cm = packed >> NODE_BITS;
        T *d = a.dst + 3 * (size_t)node;
        if (!(cm & 1)) scatter_add(d, o[0], a.plain);
        if (!(cm & 2)) scatter_add(d + 1, o[1], a.plain);
        if (!(cm & 4)) scatter_add(d + 2, o[2], a.plain);
      }
    }
    __syncwarp();
  }
}


// --------------------------------------------- apply kernel, fast path
// The production vmult cell loop.  One warp per cell; row-per-lane sum
// factorisation (SFR) with the 1D matrices as constant operands; the
// gather of the next cell (node ids, src, and u for the scalar variants) is
// prefetched into registers while the current cell is computed; with
// STAGES == 2 each warp streams its cell records through a two-stage
// shared-memory ring filled by cp.async.bulk (evict-first in L2), with
// STAGES == 0 the record is read with plain coalesced loads.  SC (scatter):
// SC_ATOMIC loops over all cells and adds with atomics; SC_COLOUR over the
// cell list of one lattice colour (a.cells, a.n_cells entries) with plain
// adds; SC_CELLBUF over all cells, storing every cell's results to
// a.cellbuf[cell][local node][component] (constrained rows as zero) for the
// node sum that follows; SC_PEER as SC_ATOMIC, with the neighbour part's
// nodes (PEER_BIT in the index map) gathered from a.psrc / a.pu and added to
// a.pdst over peer memory: the partitioned vmult's ghost update and
// compress(add) done by the cell loop itself.
constexpr int SC_ATOMIC = 0, SC_COLOUR = 1, SC_CELLBUF = 2, SC_PEER = 3;
template <int P, int Q, typename T, int VAR, int STAGES, int SC>
__global__ void __launch_bounds__(256) apply_fast_kernel(KArgs<T> a, TabT<P, Q, T> tab) {
  constexpr bool COL = SC == SC_COLOUR;
  constexpr bool SCALAR = (VAR == VAR_SCALAR_F0 || VAR == VAR_SCALAR_F1);
  // branch-free sweeps and point loop for the scalar variants (48^3 / 64^3
  // Q2: scalar -7 % FP64 / -10 % FP32, scalar_referential -4 % / -17 %;
  // tensor2 +4-6 % and tensor4 +1 %, so those keep the divergent form)
  constexpr bool CLAMP = SCALAR || VAR == VAR_SCALAR_REF;
  using S = SFR<P, Q, T, CLAMP>;
  constexpr int N1 = P + 1, NN = S::NN, NQ = S::NQ, QPL = S::QPL, RPL = S::RPL, XR = S::XR;
  // several points per lane (Q^3 > 32): the gradients stay in the slab's
  // point block and each point is read, transformed and overwritten there
  // in turn, instead of holding 2 x 9 x QPL values in registers (the FP64 Q4
  // kernel otherwise runs out of registers); the scalar variants also need
  // the displacement gradients and keep the register form
  constexpr bool PT_SMEM = !SCALAR && QPL >= 2;
  const int WPB = blockDim.x >> 5;
  extern __shared__ __align__(128) unsigned char smem[];
  const int rec_elems = a.rec_elems;
  const uint32_t rec_bytes = (uint32_t)(rec_elems * sizeof(T));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t warp_bytes = ((STAGES * (size_t)rec_bytes + 8 * (STAGES > 0 ? STAGES : 1) + S::SZ * sizeof(T) + 127) / 128) * 128;
  unsigned char *wbase = smem + warp * warp_bytes;
  constexpr int NS = STAGES > 0 ? STAGES : 1;
  T *stage[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) stage[s] = (T *)(wbase + s * rec_bytes);
  uint64_t *bar = (uint64_t *)(wbase + STAGES * rec_bytes);
  T *slab = (T *)(wbase + STAGES * rec_bytes + 8 * NS);
  const int gw = blockIdx.x * WPB + warp, nw = gridDim.x * WPB;
  // list entry -> cell
  auto cid = [&](int i) -> int { return COL ? __ldg(a.cells + i) : a.cell0 + i; };
  uint64_t pol = 0;
  if (STAGES > 0) {
    pol = evict_first_policy();
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < NS; ++s) mbar_init(&bar[s], 1);
      mbar_init_fence();
    }
    __syncwarp();
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const int c = gw + s * nw;
        if (c < a.n_cells) {
          mbar_expect_tx(&bar[s], rec_bytes);
          bulk_g2s(stage[s], a.table + (size_t)cid(c) * rec_elems, rec_bytes, &bar[s], pol);
        }
      }
    }
  }
  // gather registers of the x rows (c, k, j) owned by this lane
  int pk[RPL][N1];
  T pv[RPL][N1], pu[RPL][N1];
  auto prefetch = [&](int c) {
    const int *cn = a.cell_nodes + (size_t)cid(c) * NN;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = lane + 32 * r;
      // (CLAMP) lanes past the last row load the last row again
      if ((CLAMP && XR <= 32) || row < XR) {
        int comp, xk, xj;
        S::x_row(row < XR ? row : XR - 1, comp, xk, xj);
        const int kj = xk * N1 + xj;
#pragma unroll
        for (int i = 0; i < N1; ++i) {
          const int packed = __ldg(cn + kj * N1 + i);
          pk[r][i] = packed;
          if (SC == SC_PEER) {
            const bool pe = packed & PEER_BIT;
            const size_t dof = 3 * (size_t)(packed & PEER_NODE_MASK) + comp;
            pv[r][i] = __ldg((pe ? a.psrc : a.src) + dof);
            if (SCALAR) pu[r][i] = __ldg((pe ? a.pu : a.u) + dof);
          } else {
            const size_t dof = 3 * (size_t)(packed & NODE_MASK) + comp;
            pv[r][i] = __ldg(a.src + dof);
            if (SCALAR) pu[r][i] = __ldg(a.u + dof);
          }
        }
      }
    }
  };
  if (gw < a.n_cells) prefetch(gw);
  int it = 0;
  for (int cell = gw; cell < a.n_cells; cell += nw, ++it) {
    const int s = it % NS;
    const uint32_t parity = (it / NS) & 1;
    int ck[RPL][N1];
    T v[RPL][N1], vu[RPL][N1];
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = lane + 32 * r;
      int comp = 0, xk, xj;
      // (CLAMP: the lanes past the last row carry a copy of it; the sweeps
      // store nothing from them and the scatter skips them)
      if ((CLAMP && XR <= 32) || row < XR) S::x_row(row < XR ? row : XR - 1, comp, xk, xj);
      if (!(CLAMP && XR <= 32) && row >= XR) {
#pragma unroll
        for (int i = 0; i < N1; ++i) { ck[r][i] = 0; v[r][i] = T(0); vu[r][i] = T(0); }
        continue;
      }
#pragma unroll
      for (int i = 0; i < N1; ++i) {
        ck[r][i] = pk[r][i];
        // read_dof_values(src): constrained entries read as zero
        v[r][i] = ((pk[r][i] >> (NODE_BITS + comp)) & 1) ? T(0) : pv[r][i];
        if (SCALAR) vu[r][i] = pu[r][i];  // read_dof_values_plain(u)
      }
    }
    if (cell + nw < a.n_cells) prefetch(cell + nw);
    if (STAGES == 0 && a.prefetch) {
      // one 128-byte line of the record per lane into L1, issued before the
      // sweeps so that the point loop's loads find it there
      const int pc = a.prefetch == 2 ? cell + nw : cell;
      if (pc < a.n_cells) {
        const char *base = (const char *)(a.table + (size_t)cid(pc) * rec_elems);
        const int nbytes = rec_elems * (int)sizeof(T);
        for (int off = lane * 128; off < nbytes; off += 32 * 128)
          asm volatile("prefetch.global.L1 [%0];" ::"l"(base + off));
      }
    }
    T G[QPL][3][3], GU[QPL][3][3];
    if (SCALAR) S::eval(tab, vu, slab, lane, GU);
    if (PT_SMEM) S::eval_pt(tab, v, slab, lane);
    else S::eval(tab, v, slab, lane, G);
    const T *rec;
    if (STAGES > 0) {
      if (!mbar_wait_bounded(&bar[s], parity, a.wait_tries)) {
        if (lane == 0) atomicOr(a.flag, FLAG_TIMEOUT);
        // every copy this warp issued is still owed to a stage of its
        // shared memory: the one given up on (k = 0) and those of the next
        // NS - 1 cells.  Let each land (long bound) before the block exits,
        // so no copy writes shared memory that a later block owns.
        for (int k = 0; k < NS; ++k)
          if (cell + k * nw < a.n_cells) mbar_wait_bounded(&bar[(it + k) % NS], ((it + k) / NS) & 1);
        return;
      }
      rec = stage[s];
    } else {
      rec = a.table + (size_t)cid(cell) * rec_elems;
    }
    T mu = 0, lambda = 0, kappa = 0;
    if (SCALAR || VAR == VAR_SCALAR_REF) material<T>(a.mu[cid(cell)], a.nu, mu, lambda, kappa);
    T H[QPL][3][3];
#pragma unroll(PT_SMEM ? 1 : QPL)
    for (int l = 0; l < QPL; ++l) {
      // (CLAMP: the lanes past the last point repeat it; their H is never
      // stored)
      const int q = (CLAMP && NQ <= 32) ? (lane < NQ ? lane : NQ - 1) : lane + 32 * l;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 3; ++e) H[l][c][e] = T(0);
      if (!(CLAMP && NQ <= 32) && q >= NQ) continue;
      const T *r = rec + q;
      T Ji[3][3];
#pragma unroll
      for (int i = 0; i < 9; ++i) Ji[i / 3][i % 3] = r[(C_JINV + i) * NQ];
      const T jxw = variant_folds_jxw(VAR) ? T(1) : T(r[C_JXW * NQ]);
      T Gq[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 3; ++e) Gq[c][e] = PT_SMEM ? slab[(c * 3 + e) * S::NQP + q] : G[l][c][e];
      T g[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[c][d] = Gq[c][0] * Ji[0][d] + Gq[c][1] * Ji[1][d] + Gq[c][2] * Ji[2][d];
      ScalarState<T> st;
      if (SCALAR) {
        T Jr[3][3];
#pragma unroll
        for (int i = 0; i < 9; ++i)
          Jr[i / 3][i % 3] = a.ref_per_cell ? rec[(C_VAR + 1) * NQ + i] : r[(C_VAR + 1 + i) * NQ];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int d = 0; d < 3; ++d)
            st.F[c][d] = GU[l][c][0] * Jr[0][d] + GU[l][c][1] * Jr[1][d] + GU[l][c][2] * Jr[2][d] + (c == d ? T(1) : T(0));
        st.det = det3(st.F);
      }
      if (VAR == VAR_SCALAR_REF) {
        collocation_F<Q>(rec, q, tab.Dc, Ji, st.F);
        st.det = det3(st.F);
      }
      T Qm[3][3];
      physics<T, VAR, NQ>(g, r, mu, lambda, kappa, st, Qm);
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          const T h0 = Qm[c][0] * Ji[e][0] + Qm[c][1] * Ji[e][1] + Qm[c][2] * Ji[e][2];
          const T h = variant_folds_jxw(VAR) ? h0 : T(h0 * jxw);
          // each lane overwrites only its own points
          if (PT_SMEM) slab[(c * 3 + e) * S::NQP + q] = h;
          else H[l][c][e] = h;
        }
    }
    if (STAGES > 0) {
      __syncwarp();  // every lane is done reading stage[s]
      if (lane == 0) {
        const int next = cell + NS * nw;
        if (next < a.n_cells) {
          fence_proxy_async_smem();
          mbar_expect_tx(&bar[s], rec_bytes);
          bulk_g2s(stage[s], a.table + (size_t)cid(next) * rec_elems, rec_bytes, &bar[s], pol);
        }
      }
    }
    T out[RPL][N1];
    if (PT_SMEM) S::integrate_pt(tab, slab, lane, out);
    else S::integrate(tab, H, slab, lane, out);
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = lane + 32 * r;
      if (row < XR) {
        int comp, xk, xj;
        S::x_row(row, comp, xk, xj);
#pragma unroll
        for (int i = 0; i < N1; ++i) {
          // distribute_local_to_global: constrained rows skipped
          const bool con = (ck[r][i] >> (NODE_BITS + comp)) & 1;
          if (SC == SC_CELLBUF) {
            a.cellbuf[((size_t)cell * NN + (xk * N1 + xj) * N1 + i) * 3 + comp] = con ? T(0) : out[r][i];
          } else if (SC == SC_PEER) {
            if (!con) {
              const int k = ck[r][i];
              atomic_add(((k & PEER_BIT) ? a.pdst : a.dst) + 3 * (size_t)(k & PEER_NODE_MASK) + comp, out[r][i]);
            }
          } else if (!con) {
            T *d = a.dst + 3 * (size_t)(ck[r][i] & NODE_MASK) + comp;
            if (COL) *d += out[r][i];
            else atomic_add(d, out[r][i]);
          }
        }
      }
    }
  }
}

// ------------------------------------------------ FP32 cell-pair kernel
// The plain-load cell loop of apply_fast_kernel for FP32 operators with two
// cells per warp: list entries 2i and 2i + 1 go through the sweeps and the
// point physics together as the two halves of packed f32x2 registers
// (pair.cuh), so one issued arithmetic or shared-memory instruction serves
// both cells.  Gathers, record loads and the scatter stay per cell.  With an
// odd count the last pair repeats its first cell and scatters it once.
// per-warp shared memory of the pair kernel (8 bytes, then the slab of the
// 8-byte-entry sweep layout), used by the kernel and by its launcher
template <int P, int Q>
__host__ __device__ constexpr size_t pair_warp_bytes() {
  return ((8 + SFR<P, Q, f2>::SZ * sizeof(f2) + 127) / 128) * 128;
}

template <int P, int Q, int VAR, int SC>
__global__ void __launch_bounds__(256) apply_pair_kernel(KArgs<float> a, TabT<P, Q, f2> tab) {
  using T = f2;
  constexpr bool COL = SC == SC_COLOUR;
  constexpr bool SCALAR = (VAR == VAR_SCALAR_F0 || VAR == VAR_SCALAR_F1);
  constexpr bool CLAMP = SCALAR || VAR == VAR_SCALAR_REF;
  using S = SFR<P, Q, T, CLAMP>;
  constexpr int N1 = P + 1, NN = S::NN, NQ = S::NQ, QPL = S::QPL, RPL = S::RPL, XR = S::XR;
  constexpr bool PT_SMEM = !SCALAR && QPL >= 2;
  const int WPB = blockDim.x >> 5;
  extern __shared__ __align__(128) unsigned char smem[];
  const int rec_elems = a.rec_elems;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr size_t warp_bytes = pair_warp_bytes<P, Q>();
  {
    // the launch must provide every warp's slab; otherwise do nothing
    unsigned dyn;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if ((size_t)WPB * warp_bytes > dyn) {
      if (threadIdx.x == 0) atomicOr(a.flag, FLAG_SMEM);
      return;
    }
  }
  T *slab = (T *)(smem + warp * warp_bytes + 8);
  const int gw = blockIdx.x * WPB + warp, nw = gridDim.x * WPB;
  const int n_pairs = (a.n_cells + 1) >> 1;
  auto cid = [&](int i) -> int { return COL ? __ldg(a.cells + i) : a.cell0 + i; };
  // gather registers of the x rows (c, k, j) owned by this lane, both cells
  int pk0[RPL][N1], pk1[RPL][N1];
  float pv0[RPL][N1], pv1[RPL][N1], pu0[RPL][N1], pu1[RPL][N1];
  auto prefetch = [&](int pi) {
    const int e0 = 2 * pi, e1 = (2 * pi + 1 < a.n_cells) ? 2 * pi + 1 : 2 * pi;
    const int *cn0 = a.cell_nodes + (size_t)cid(e0) * NN, *cn1 = a.cell_nodes + (size_t)cid(e1) * NN;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = lane + 32 * r;
      if ((CLAMP && XR <= 32) || row < XR) {
        int comp, xk, xj;
        S::x_row(row < XR ? row : XR - 1, comp, xk, xj);
        const int kj = xk * N1 + xj;
#pragma unroll
        for (int i = 0; i < N1; ++i) {
          const int k0 = __ldg(cn0 + kj * N1 + i), k1 = __ldg(cn1 + kj * N1 + i);
          pk0[r][i] = k0;
          pk1[r][i] = k1;
          const size_t d0 = 3 * (size_t)(k0 & NODE_MASK) + comp, d1 = 3 * (size_t)(k1 & NODE_MASK) + comp;
          pv0[r][i] = __ldg(a.src + d0);
          pv1[r][i] = __ldg(a.src + d1);
          if (SCALAR) {
            pu0[r][i] = __ldg(a.u + d0);
            pu1[r][i] = __ldg(a.u + d1);
          }
        }
      }
    }
  };
  if (gw < n_pairs) prefetch(gw);
  for (int pi = gw; pi < n_pairs; pi += nw) {
    const int e0 = 2 * pi;
    const bool two = 2 * pi + 1 < a.n_cells;
    const int e1 = two ? e0 + 1 : e0;
    const int c0 = cid(e0), c1 = cid(e1);
    int ck0[RPL][N1], ck1[RPL][N1];
    T v[RPL][N1], vu[RPL][N1];
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = lane + 32 * r;
      int comp = 0, xk, xj;
      if ((CLAMP && XR <= 32) || row < XR) S::x_row(row < XR ? row : XR - 1, comp, xk, xj);
      if (!(CLAMP && XR <= 32) && row >= XR) {
#pragma unroll
        for (int i = 0; i < N1; ++i) { ck0[r][i] = 0; ck1[r][i] = 0; v[r][i] = T(0); vu[r][i] = T(0); }
        continue;
      }
#pragma unroll
      for (int i = 0; i < N1; ++i) {
        ck0[r][i] = pk0[r][i];
        ck1[r][i] = pk1[r][i];
        // read_dof_values(src): constrained entries read as zero
        v[r][i] = pack2(((pk0[r][i] >> (NODE_BITS + comp)) & 1) ? 0.f : pv0[r][i],
                        ((pk1[r][i] >> (NODE_BITS + comp)) & 1) ? 0.f : pv1[r][i]);
        if (SCALAR) vu[r][i] = pack2(pu0[r][i], pu1[r][i]);
      }
    }
    if (pi + nw < n_pairs) prefetch(pi + nw);
    if (a.prefetch) {
      // both records into L1 before the sweeps
      const char *b0 = (const char *)(a.table + (size_t)c0 * rec_elems);
      const char *b1 = (const char *)(a.table + (size_t)c1 * rec_elems);
      const int nbytes = rec_elems * (int)sizeof(float);
      for (int off = lane * 128; off < nbytes; off += 32 * 128) {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(b0 + off));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(b1 + off));
      }
    }
    T G[QPL][3][3], GU[QPL][3][3];
    if (SCALAR) S::eval(tab, vu, slab, lane, GU);
    if (PT_SMEM) S::eval_pt(tab, v, slab, lane);
    else S::eval(tab, v, slab, lane, G);
    const RecPair rec{a.table + (size_t)c0 * rec_elems, a.table + (size_t)c1 * rec_elems};
    T mu = 0, lambda = 0, kappa = 0;
    if (SCALAR || VAR == VAR_SCALAR_REF) {
      float m0, l0, k0, m1, l1, k1;
      material<float>(a.mu[c0], a.nu, m0, l0, k0);
      material<float>(a.mu[c1], a.nu, m1, l1, k1);
      mu = pack2(m0, m1);
      lambda = pack2(l0, l1);
      kappa = pack2(k0, k1);
    }
    T H[QPL][3][3];
#pragma unroll(PT_SMEM ? 1 : QPL)
    for (int l = 0; l < QPL; ++l) {
      const int q = (CLAMP && NQ <= 32) ? (lane < NQ ? lane : NQ - 1) : lane + 32 * l;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 3; ++e) H[l][c][e] = T(0);
      if (!(CLAMP && NQ <= 32) && q >= NQ) continue;
      const RecPair r = rec + q;
      T Ji[3][3];
#pragma unroll
      for (int i = 0; i < 9; ++i) Ji[i / 3][i % 3] = r[(C_JINV + i) * NQ];
      const T jxw = variant_folds_jxw(VAR) ? T(1) : T(r[C_JXW * NQ]);
      T Gq[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 3; ++e) Gq[c][e] = PT_SMEM ? slab[(c * 3 + e) * S::NQP + q] : G[l][c][e];
      T g[3][3];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[c][d] = Gq[c][0] * Ji[0][d] + Gq[c][1] * Ji[1][d] + Gq[c][2] * Ji[2][d];
      ScalarState<T> st;
      if (SCALAR) {
        T Jr[3][3];
#pragma unroll
        for (int i = 0; i < 9; ++i)
          Jr[i / 3][i % 3] = a.ref_per_cell ? rec[(C_VAR + 1) * NQ + i] : r[(C_VAR + 1 + i) * NQ];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int d = 0; d < 3; ++d)
            st.F[c][d] = GU[l][c][0] * Jr[0][d] + GU[l][c][1] * Jr[1][d] + GU[l][c][2] * Jr[2][d] + (c == d ? T(1) : T(0));
        st.det = det3(st.F);
      }
      if (VAR == VAR_SCALAR_REF) {
        collocation_F<Q>(rec, q, tab.Dc, Ji, st.F);
        st.det = det3(st.F);
      }
      T Qm[3][3];
      physics<T, VAR, NQ>(g, r, mu, lambda, kappa, st, Qm);
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int e = 0; e < 3; ++e) {
          const T h0 = Qm[c][0] * Ji[e][0] + Qm[c][1] * Ji[e][1] + Qm[c][2] * Ji[e][2];
          const T h = variant_folds_jxw(VAR) ? h0 : T(h0 * jxw);
          if (PT_SMEM) slab[(c * 3 + e) * S::NQP + q] = h;
          else H[l][c][e] = h;
        }
    }
    T out[RPL][N1];
    if (PT_SMEM) S::integrate_pt(tab, slab, lane, out);
    else S::integrate(tab, H, slab, lane, out);
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row = lane + 32 * r;
      if (row < XR) {
        int comp, xk, xj;
        S::x_row(row, comp, xk, xj);
#pragma unroll
        for (int i = 0; i < N1; ++i) {
          float o0, o1;
          unpack2(out[r][i], o0, o1);
          // distribute_local_to_global: constrained rows skipped
          const bool con0 = (ck0[r][i] >> (NODE_BITS + comp)) & 1, con1 = (ck1[r][i] >> (NODE_BITS + comp)) & 1;
          if (SC == SC_CELLBUF) {
            const int local = (xk * N1 + xj) * N1 + i;
            a.cellbuf[((size_t)e0 * NN + local) * 3 + comp] = con0 ? 0.f : o0;
            if (two) a.cellbuf[((size_t)e1 * NN + local) * 3 + comp] = con1 ? 0.f : o1;
          } else {
            if (!con0) {
              float *d = a.dst + 3 * (size_t)(ck0[r][i] & NODE_MASK) + comp;
              if (COL) *d += o0;
              else atomicAdd(d, o0);
            }
            if (two && !con1) {
              float *d = a.dst + 3 * (size_t)(ck1[r][i] & NODE_MASK) + comp;
              if (COL) *d += o1;
              else atomicAdd(d, o1);
            }
          }
        }
      }
    }
  }
}

// --------------------------------------------------------- diagonal kernel
// diag(a,c) = sum_q JxW n^T B_c n with n = grad_x N_a and
// B_c[d][l] = Q(e_c (x) e_l)[c][d]: identical to applying the cell operator
// to unit vectors (mf_nh_operator.h:881-899) and keeping the diagonal entry.
template <int P, int Q, typename T, int VAR>
__global__ void __launch_bounds__(128) diagonal_kernel(KArgs<T> a, Tab<P, Q> tab) {
  using S = SF<P, Q, T>;
  constexpr int N1 = P + 1, NN = S::NN, NQ = S::NQ, QPL = S::QPL;
  const int WPB = blockDim.x >> 5;
  constexpr bool SCALAR = (VAR == VAR_SCALAR_F0 || VAR == VAR_SCALAR_F1);
  constexpr int SZD = S::SZ + 36 * NQ;
  extern __shared__ __align__(16) unsigned char smem[];
  T *sN = (T *)smem, *sD = sN + Q * N1;
  load_tables<P, Q, T>(tab, sN, sD);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T *slab = sD + Q * N1 + warp * SZD;
  T *V = slab, *A = slab + S::SZ1, *B = A + S::SZ2;
  T *Bq = slab + S::SZ;  // [q][27] then [q][9] inverse Jacobian
  T *Jq = Bq + 27 * NQ;
  const int gw = blockIdx.x * WPB + warp, nw = gridDim.x * WPB;
  for (int ic = gw; ic < a.n_cells; ic += nw) {
    const int cell = cell_of(a, ic);
    const int *cn = a.cell_nodes + (size_t)cell * NN;
    const T *rec = a.table + (size_t)cell * a.rec_elems;
    T GU[QPL][3][3];
    if (SCALAR) {
      gather<NN>(cn, a.u, false, V, lane);
      S::eval(sN, sD, V, A, B, lane, GU);
    }
    T mu = 0, lambda = 0, kappa = 0;
    if (SCALAR || VAR == VAR_SCALAR_REF) material<T>(a.mu[cell], a.nu, mu, lambda, kappa);
#pragma unroll
    for (int l = 0; l < QPL; ++l) {
      const int q = lane + 32 * l;
      if (q >= NQ) continue;
      const T *r = rec + q;
      const T jxw = variant_folds_jxw(VAR) ? T(1) : T(r[C_JXW * NQ]);
      T Ji[3][3];
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        Jq[q * 9 + i] = r[(C_JINV + i) * NQ];
        Ji[i / 3][i % 3] = r[(C_JINV + i) * NQ];
      }
      ScalarState<T> st;
      if (SCALAR) {
        T Jr[3][3];
#pragma unroll
        for (int i = 0; i < 9; ++i)
          Jr[i / 3][i % 3] = a.ref_per_cell ? rec[(C_VAR + 1) * NQ + i] : r[(C_VAR + 1 + i) * NQ];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int d = 0; d < 3; ++d)
            st.F[c][d] = GU[l][c][0] * Jr[0][d] + GU[l][c][1] * Jr[1][d] + GU[l][c][2] * Jr[2][d] + (c == d ? T(1) : T(0));
        st.det = det3(st.F);
      }
      if (VAR == VAR_SCALAR_REF) {
        collocation_F<Q>(rec, q, tab.Dc, Ji, st.F);
        st.det = det3(st.F);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int ll = 0; ll < 3; ++ll) {
          T g[3][3];
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) g[i][j] = (i == c && j == ll) ? T(1) : T(0);
          T Qm[3][3];
          physics<T, VAR, NQ>(g, r, mu, lambda, kappa, st, Qm);
#pragma unroll
          for (int d = 0; d < 3; ++d)
            Bq[q * 27 + (c * 3 + d) * 3 + ll] = variant_folds_jxw(VAR) ? Qm[c][d] : T(Qm[c][d] * jxw);
        }
    }
    __syncwarp();
    for (int an = lane; an < NN; an += 32) {
      const int ix = an % N1, iy = (an / N1) % N1, iz = an / (N1 * N1);
      T o[3] = {T(0), T(0), T(0)};
      for (int q = 0; q < NQ; ++q) {
        const int qx = q % Q, qy = (q / Q) % Q, qz = q / (Q * Q);
        const T nx = sN[qx * N1 + ix], ny = sN[qy * N1 + iy], nz = sN[qz * N1 + iz];
        const T gx = sD[qx * N1 + ix] * ny * nz, gy = nx * sD[qy * N1 + iy] * nz, gz = nx * ny * sD[qz * N1 + iz];
        const T *J = Jq + q * 9;
        T n[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) n[d] = gx * J[d] + gy * J[3 + d] + gz * J[6 + d];
        const T *Bc = Bq + q * 27;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T s = 0;
#pragma unroll
          for (int d = 0; d < 3; ++d)
            s += n[d] * (Bc[(c * 3 + d) * 3 + 0] * n[0] + Bc[(c * 3 + d) * 3 + 1] * n[1] + Bc[(c * 3 + d) * 3 + 2] * n[2]);
          o[c] += s;
        }
      }
      const int packed = __ldg(cn + an);
      const int node = packed & NODE_MASK, cm = packed >> NODE_BITS;
      T *d = a.dst + 3 * (size_t)node;
      if (!(cm & 1)) scatter_add(d, o[0], a.plain);
      if (!(cm & 2)) scatter_add(d + 1, o[1], a.plain);
      if (!(cm & 4)) scatter_add(d + 2, o[2], a.plain);
    }
    __syncwarp();
  }
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

template <int P, int Q, typename T>
TabT<P, Q, T> make_tabt(const Basis &b) {
  TabT<P, Q, T> t;
  for (int k = 0; k < Q; ++k) {
    for (int i = 0; i <= P; ++i) {
      t.N[k][i] = T(b.N[k * (P + 1) + i]);
      t.D[k][i] = T(b.D[k * (P + 1) + i]);
    }
    for (int m = 0; m < Q; ++m) t.Dc[k][m] = T(b.Dc[k * Q + m]);
  }
  return t;
}

template <int P, int Q>
Tab<P, Q> make_tab(const Basis &b) {
  Tab<P, Q> t;
  for (int k = 0; k < Q; ++k) {
    for (int i = 0; i <= P; ++i) {
      t.N[k][i] = b.N[k * (P + 1) + i];
      t.D[k][i] = b.D[k * (P + 1) + i];
    }
    t.w[k] = b.qw[k];
    for (int m = 0; m < Q; ++m) t.Dc[k][m] = b.Dc[k * Q + m];
  }
  return t;
}

// grid for a persistent-style launch: a whole number of waves of the SMs
template <typename K>
int grid_for(K kernel, int threads, size_t smem, int n_items_per_block_total) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  if (per_sm < 1) per_sm = 1;
  int g = num_sms() * per_sm;
  if (g > n_items_per_block_total) g = n_items_per_block_total;
  return g < 1 ? 1 : g;
}

// warps per block such that the per-warp slabs fit in ~200 KB of shared memory
inline int warps_for(size_t slab_bytes, int max_warps) {
  int w = max_warps;
  while (w > 1 && slab_bytes * w > 200 * 1024) w >>= 1;
  return w;
}
// largest warp count (<= max_warps) whose slabs fit in budget bytes
inline int warps_for_budget(size_t warp_bytes, int max_warps, size_t budget) {
  int w = max_warps;
  while (w > 0 && warp_bytes * w > budget) --w;
  return w;
}

int variant_of(const lsmf_op *op) {
  if (op->caching == LSMF_CACHE_TENSOR4) return VAR_TENSOR4;
  if (op->caching == LSMF_CACHE_TENSOR2) return VAR_TENSOR2;
  if (op->caching == LSMF_CACHE_SCALAR_REFERENTIAL) return VAR_SCALAR_REF;
  if (op->caching == LSMF_CACHE_TENSOR4_NS) return VAR_TENSOR4_NS;
  return op->formulation == 0 ? VAR_SCALAR_F0 : VAR_SCALAR_F1;
}

template <typename T>
KArgs<T> make_args(const lsmf_op *op) {
  const Level &L = op->L();
  KArgs<T> a;
  a.cell_nodes = L.d_cell_nodes.ptr;
  a.n_cells = L.n_cells;
  a.ncomp = op->ncomp;
  a.rec_elems = op->rec_elems;
  a.ref_per_cell = op->ref_per_cell ? 1 : 0;
  a.table = (T *)op->d_table.ptr;
  a.src = nullptr;
  a.dst = nullptr;
  a.u = (const T *)op->d_u;
  a.X = L.d_X.ptr;
  a.mu = op->d_mu.ptr;
  a.nu = op->nu;
  a.flag = op->d_flag.ptr;
  a.mask = LSMF_MASK_DEFAULT;
  a.wait_tries = op->wait_tries >= 0 ? op->wait_tries : WAIT_TRIES_DEFAULT;
  a.cells = nullptr;
  a.plain = 0;
  a.cellbuf = nullptr;
  a.prefetch = op->prefetch;
  a.psrc = nullptr;
  a.pdst = nullptr;
  a.pu = nullptr;
  a.cell0 = 0;
  return a;
}

template <typename T>
void set_range(KArgs<T> &a, const CellRange &r) {
  if (r.cells) {
    a.cells = r.cells;
    a.n_cells = r.n_list;
  }
  a.plain = r.plain ? 1 : 0;
  a.cellbuf = (T *)r.cellbuf;
  if (r.count >= 0) {
    a.cell0 = r.first;
    a.n_cells = r.count;
  }
  if (r.peer_nodes) {
    a.cell_nodes = r.peer_nodes;
    a.psrc = (const T *)r.peer_src;
    a.pdst = (T *)r.peer_dst;
    a.pu = (const T *)r.peer_u;
  }
}

template <int P, int Q, typename T, int VAR>
lsmf_status run_cache(lsmf_op *op) {
  auto a = make_args<T>(op);
  const Tab<P, Q> tab = make_tab<P, Q>(op->mesh->basis);
  using S = SF<P, Q, double>;
  const int w = warps_for(sizeof(double) * S::SZ, 8);
  const size_t smem = sizeof(double) * (S::TAB + w * S::SZ);
  auto k = cache_kernel<P, Q, T, VAR>;
  LSMF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int g = grid_for(k, 32 * w, smem, (a.n_cells + w - 1) / w);
  k<<<g, 32 * w, smem, op->stream>>>(a, tab);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

template <int P, int Q, typename T, int VAR>
lsmf_status run_apply(const lsmf_op *op, T *dst, const T *src, unsigned mask, CellRange range) {
  auto a = make_args<T>(op);
  cudaStream_t stream = range.stream ? range.stream : op->stream;
  a.src = src;
  a.dst = dst;
  a.mask = mask;
  set_range(a, range);
  if (a.n_cells == 0) return LSMF_OK;
  // L1 prefetch of each cell's record before its sweeps (plain-load
  // kernels): measured on B200 at 64^3 Q2 and 48^3 Q4 it shortens every
  // plain-load kernel (Q4 tensor4 FP64 1.37 -> 1.19 ms, Q2 tensor2 FP32
  // -6 %) except the FP64 scalar variant (+1 %), which keeps it off
  if (op->prefetch < 0) a.prefetch = ((VAR == VAR_SCALAR_F0 || VAR == VAR_SCALAR_F1) && sizeof(T) == 8) ? 0 : 1;
  const Tab<P, Q> tab = make_tab<P, Q>(op->mesh->basis);
  using S = SF<P, Q, T>;
  const int w = warps_for(sizeof(T) * S::SZ, 8);
  const size_t smem = sizeof(T) * (S::TAB + w * S::SZ);
  const bool full = (mask & (LSMF_MASK_RW | LSMF_MASK_SF | LSMF_MASK_QD)) ==
                        (LSMF_MASK_RW | LSMF_MASK_SF | LSMF_MASK_QD) &&
                    !(mask & MASK_INHOM);
  using SR = SFR<P, Q, T>;
  const size_t rec_bytes = (size_t)op->rec_elems * sizeof(T);
  const TabT<P, Q, T> tabt = make_tabt<P, Q, T>(op->mesh->basis);
  auto wbytes = [&](int st) { return ((st * rec_bytes + 8 * (st > 0 ? st : 1) + SR::SZ * sizeof(T) + 127) / 128) * 128; };
  // defaults measured on B200 (ring depth x record prefetch x warps per
  // block swept for Q2 / Q3 / Q4 at 64^3 / 48^3 / 48^3 cells): at Q1 / Q2
  // the variants that stream a large record per point (tensor4, tensor4_ns)
  // and scalar_referential (whose collocation gradient reads the record out
  // of order) want the one-stage bulk-copy ring while a record fits in
  // 24 KB; from Q3 on, plain loads with the L1 record prefetch are faster
  // (Q3 FP32 tensor4 0.409 -> 0.337 ms, tensor4_ns 0.661 -> 0.449 ms,
  // scalar_referential FP32 -6 % / FP64 -15 %), as they are for the larger
  // records (Q3 FP64 tensor4, Q4) and for tensor2 and scalar (latency / FP64
  // bound)
  const bool ring_variant = VAR == VAR_TENSOR4 || VAR == VAR_TENSOR4_NS || VAR == VAR_SCALAR_REF;
  int stages = op->stages >= 0 ? op->stages : ((ring_variant && P <= 2 && rec_bytes <= 24 * 1024) ? 1 : 0);
  // a level small enough that every warp gets at most one cell (a coarse
  // multigrid level) gains nothing from the ring, which can only prefetch
  // a warp's next cell: plain loads (15^3-cell FP64 coarse Chebyshev solve
  // 10.9 -> 9.9 ms per V-cycle, FP32 unchanged)
  if (op->stages < 0 && a.n_cells <= 32 * num_sms()) stages = 0;
  // warps per block, swept 2 / 4 / 8 for every variant and precision at
  // 64^3 Q2: 8 for the FP64 tensor2 and scalar kernels (scalar 0.478 ->
  // 0.466 ms, formulation 0 0.497 -> 0.482 ms), 2 for FP64
  // scalar_referential (0.467 -> 0.452 ms), 4 otherwise (the others within
  // 1 % of each other)
  constexpr bool fp64 = sizeof(T) == 8;
  const int max_warps =
      op->max_warps > 0 ? op->max_warps
      : (fp64 && (VAR == VAR_TENSOR2 || VAR == VAR_SCALAR_F1 || VAR == VAR_SCALAR_F0)) ? 8
      : (fp64 && VAR == VAR_SCALAR_REF) ? 2
                                        : 4;
  if (rec_bytes % 16 != 0) stages = 0;
  // fewer stages when the ring would leave fewer than 4 warps per block
  while (stages > 0 && warps_for_budget(wbytes(stages), 8, 220 * 1024) < 4) --stages;
  const bool col = a.cells != nullptr;
  const bool cellbuf = a.cellbuf != nullptr;
  if (cellbuf && !(full && !op->basic)) {
    set_error("the node-sum scatter serves the full vmult cell loop only");
    return LSMF_ERR_INVALID_ARG;
  }
  const bool peer = range.peer_nodes != nullptr;
  if (peer && (!full || op->basic || col || cellbuf || sizeof(T) != 8)) {
    set_error("the fused interface exchange serves the full FP64 vmult cell loop with atomic scatter only");
    return LSMF_ERR_INVALID_ARG;
  }
  // the colour, cell-buffer and peer launches are built with at most one stage
  if ((col || cellbuf || peer) && stages > 1) stages = 1;
  if constexpr (std::is_same<T, float>::value) {
    // automatic choice, measured on B200 (FP32 vmult at 96^3 Q1, 64^3 Q2,
    // 48^3 Q3 / Q4 and the 15^3 -> 30^3 / 60^3 Q2 V-cycles), pairs where
    // they were faster: Q1 tensor2 (-2 %) and scalar (-8 %); Q2 tensor2
    // (-9 %, V-cycle -5 %), scalar (-8 %, V-cycle -7 %) and
    // scalar_referential (-11 %); Q4 scalar_referential (-10 %).  Every Q3
    // variant (+5-13 %), the record-heavy tensor4 (Q2 +27 %) and tensor4_ns
    // (+8 %), whose loops are bound by load latency and lose half their warps
    // to the pair kernel's registers, and formulation 0 (+12 %, 159
    // registers) stay one cell per warp.
    constexpr bool pair_variant = (P == 1 && (VAR == VAR_TENSOR2 || VAR == VAR_SCALAR_F1)) ||
                                  (P == 2 && (VAR == VAR_TENSOR2 || VAR == VAR_SCALAR_F1 || VAR == VAR_SCALAR_REF)) ||
                                  (P == 4 && VAR == VAR_SCALAR_REF);
    if (full && !op->basic && (op->pairs > 0 || (op->pairs < 0 && pair_variant))) {
      // FP32 cell pairs (plain loads; the ring is not used)
      const size_t wb = pair_warp_bytes<P, Q>();
      const int w = warps_for_budget(wb, max_warps < 8 ? max_warps : 8, 220 * 1024);
      const size_t smem_p = w * wb;
      const TabT<P, Q, f2> tabp = make_tabt<P, Q, f2>(op->mesh->basis);
      const int n_pairs = (a.n_cells + 1) / 2;
      auto go = [&](auto k) -> lsmf_status {
        LSMF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_p));
        const int g = grid_for(k, 32 * w, smem_p, (n_pairs + w - 1) / w);
        k<<<g, 32 * w, smem_p, stream>>>(a, tabp);
        return LSMF_OK;
      };
      if (col) return go(apply_pair_kernel<P, Q, VAR, SC_COLOUR>);
      if (cellbuf) return go(apply_pair_kernel<P, Q, VAR, SC_CELLBUF>);
      return go(apply_pair_kernel<P, Q, VAR, SC_ATOMIC>);
    }
  }
  if (full && !op->basic) {
    // at most 8 warps per block (the kernel's launch bound is 256 threads);
    // smaller blocks let several blocks share an SM
    const int w = warps_for_budget(wbytes(stages), max_warps < 8 ? max_warps : 8, 220 * 1024);
    const size_t smem_t = w * wbytes(stages);
    lsmf_status st = LSMF_OK;
    auto go = [&](auto k) -> lsmf_status {
      LSMF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_t));
      const int g = grid_for(k, 32 * w, smem_t, (a.n_cells + w - 1) / w);
      k<<<g, 32 * w, smem_t, stream>>>(a, tabt);
      return LSMF_OK;
    };
    if (col) {
      st = stages == 0 ? go(apply_fast_kernel<P, Q, T, VAR, 0, SC_COLOUR>)
                       : go(apply_fast_kernel<P, Q, T, VAR, 1, SC_COLOUR>);
    } else if (cellbuf) {
      st = stages == 0 ? go(apply_fast_kernel<P, Q, T, VAR, 0, SC_CELLBUF>)
                       : go(apply_fast_kernel<P, Q, T, VAR, 1, SC_CELLBUF>);
    } else if (peer) {
      if constexpr (sizeof(T) == 8)
        st = stages == 0 ? go(apply_fast_kernel<P, Q, T, VAR, 0, SC_PEER>)
                         : go(apply_fast_kernel<P, Q, T, VAR, 1, SC_PEER>);
    } else {
      switch (stages) {
        case 0: st = go(apply_fast_kernel<P, Q, T, VAR, 0, SC_ATOMIC>); break;
        case 1: st = go(apply_fast_kernel<P, Q, T, VAR, 1, SC_ATOMIC>); break;
        case 2: st = go(apply_fast_kernel<P, Q, T, VAR, 2, SC_ATOMIC>); break;
        default: st = go(apply_fast_kernel<P, Q, T, VAR, 3, SC_ATOMIC>); break;
      }
    }
    if (st != LSMF_OK) return st;
  } else if (full) {
    auto k = apply_kernel<P, Q, T, VAR, true>;
    LSMF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int g = grid_for(k, 32 * w, smem, (a.n_cells + w - 1) / w);
    k<<<g, 32 * w, smem, stream>>>(a, tab);
  } else {
    auto k = apply_kernel<P, Q, T, VAR, false>;
    LSMF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int g = grid_for(k, 32 * w, smem, (a.n_cells + w - 1) / w);
    k<<<g, 32 * w, smem, stream>>>(a, tab);
  }
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

template <int P, int Q, typename T, int VAR>
lsmf_status run_diag(lsmf_op *op, T *diag, CellRange range) {
  auto a = make_args<T>(op);
  a.dst = diag;
  set_range(a, range);
  if (a.n_cells == 0) return LSMF_OK;
  const Tab<P, Q> tab = make_tab<P, Q>(op->mesh->basis);
  using S = SF<P, Q, T>;
  const int w = warps_for(sizeof(T) * (S::SZ + 36 * S::NQ), 4);
  const size_t smem = sizeof(T) * (S::TAB + w * (S::SZ + 36 * S::NQ));
  auto k = diagonal_kernel<P, Q, T, VAR>;
  LSMF_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int g = grid_for(k, 32 * w, smem, (a.n_cells + w - 1) / w);
  k<<<g, 32 * w, smem, op->stream>>>(a, tab);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}

#define LSMF_DISPATCH_VAR(v, ...)                                                     \
  [&]() -> lsmf_status {                                                              \
    switch (v) {                                                                      \
      case VAR_TENSOR4: { constexpr int V_ = VAR_TENSOR4; return __VA_ARGS__; }       \
      case VAR_TENSOR2: { constexpr int V_ = VAR_TENSOR2; return __VA_ARGS__; }       \
      case VAR_SCALAR_F1: { constexpr int V_ = VAR_SCALAR_F1; return __VA_ARGS__; }   \
      case VAR_SCALAR_REF: { constexpr int V_ = VAR_SCALAR_REF; return __VA_ARGS__; } \
      case VAR_TENSOR4_NS: { constexpr int V_ = VAR_TENSOR4_NS; return __VA_ARGS__; } \
      default: { constexpr int V_ = VAR_SCALAR_F0; return __VA_ARGS__; }             \
    }                                                                                 \
  }()

// the entry points of one (degree, precision) pair, Q = P + 1 Gauss points
template <int P, typename T>
struct DegreeOps {
  static constexpr int Q = P + 1;
  static lsmf_status cache(lsmf_op *op) {
    return LSMF_DISPATCH_VAR(variant_of(op), (run_cache<P, Q, T, V_>(op)));
  }
  static lsmf_status apply(const lsmf_op *op, void *dst, const void *src, unsigned mask, CellRange range) {
    return LSMF_DISPATCH_VAR(variant_of(op), (run_apply<P, Q, T, V_>(op, (T *)dst, (const T *)src, mask, range)));
  }
  static lsmf_status diag(lsmf_op *op, void *d, CellRange range) {
    return LSMF_DISPATCH_VAR(variant_of(op), (run_diag<P, Q, T, V_>(op, (T *)d, range)));
  }
  static const OpsTable &table() {
    static const OpsTable t = {&cache, &apply, &diag};
    return t;
  }
};

}  // namespace
}  // namespace lsmf
