// Device building blocks of the cell kernels: warp-cooperative sum
// factorisation and the quadrature-point physics of the Neo-Hookean tangent.
//
// Execution model: one warp owns one cell at a time.  Lanes stride over the
// work items of each tensor-product sweep; intermediate tensors live in a
// per-warp shared-memory slab, so only __syncwarp() separates the sweeps.
// Quadrature point q belongs to lane q % 32 (QPL = ceil(Q^3/32) points per
// lane), so everything per quadrature point stays in registers.
#pragma once
#include <cuda_runtime.h>

#include "lsmf_internal.h"

namespace lsmf {

enum Variant {
  VAR_TENSOR4 = 0, VAR_TENSOR2 = 1, VAR_SCALAR_F1 = 2, VAR_SCALAR_F0 = 3,
  VAR_SCALAR_REF = 4,  // scalar_referential
  VAR_TENSOR4_NS = 5   // tensor4_ns (dP/dF)
};
__host__ __device__ constexpr bool variant_referential(int v) { return v == VAR_SCALAR_REF || v == VAR_TENSOR4_NS; }

// Record layout per cell: [comp][qp], ncomp * Q^3 values, the record padded
// at its end to a multiple of 16 bytes.  The first 9 components are the
// inverse Jacobian (row-major) of the frame the variant integrates in:
// Eulerian for tensor4 / tensor2 / scalar, reference for scalar_referential
// and tensor4_ns.  The point result of tensor4, tensor2 and tensor4_ns is
// linear in their cached coefficients, so those are stored multiplied by
// JxW and follow from component 9: tensor4 JxW tau/J (6) + JxW C (36);
// tensor2 JxW c1, JxW c2, JxW tau/J (6); tensor4_ns JxW dP/dF (81).  The
// scalar variants keep JxW as component 9, then: scalar c + reference
// inverse Jacobian (9); scalar_referential c + u at the point (3).
constexpr int C_JINV = 0, C_JXW = 9, C_VAR = 10;
__host__ __device__ constexpr bool variant_folds_jxw(int v) {
  return v == VAR_TENSOR4 || v == VAR_TENSOR2 || v == VAR_TENSOR4_NS;
}
// first coefficient component
__host__ __device__ constexpr int variant_cvar(int v) { return variant_folds_jxw(v) ? C_JXW : C_VAR; }
__host__ __device__ constexpr int variant_ncomp(int v) {
  return v == VAR_TENSOR4 ? 51 : v == VAR_TENSOR2 ? 17 : v == VAR_SCALAR_REF ? 14 : v == VAR_TENSOR4_NS ? 90 : 20;
}

template <int P, int Q>
struct Tab {
  double N[Q][P + 1], D[Q][P + 1], w[Q];
  double Dc[Q][Q];  // collocation derivative on the Gauss points
};

// 1D tables in the arithmetic type, passed by value as a kernel parameter:
// with compile-time indices every entry is a constant-bank operand of the
// FMA, so the sweeps below load no shape values from memory.
template <int P, int Q, typename T>
struct TabT {
  T N[Q][P + 1], D[Q][P + 1];
  T Dc[Q][Q];  // collocation derivative on the Gauss points
};

// scalar_referential: F = I + Grad u from the displacement stored at the
// points of the cell record (collocation derivative, the
// FEEvaluationImplCollocation step of mf_nh_operator.h:1271-1300) and the
// reference inverse Jacobian
// (R: the record, a pointer or an accessor with operator[] and + offset)
template <int Q, typename T, typename DC, typename R>
__device__ __forceinline__ void collocation_F(const R &rec, int q, const DC &Dc, const T Ji[3][3], T F[3][3]) {
  constexpr int NQ = Q * Q * Q;
  const int qx = q % Q, qy = (q / Q) % Q, qz = q / (Q * Q);
  T G[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const auto u = rec + (C_VAR + 1 + c) * NQ;
    T gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int m = 0; m < Q; ++m) {
      gx += T(Dc[qx][m]) * u[(qz * Q + qy) * Q + m];
      gy += T(Dc[qy][m]) * u[(qz * Q + m) * Q + qx];
      gz += T(Dc[qz][m]) * u[(m * Q + qy) * Q + qx];
    }
    G[c][0] = gx; G[c][1] = gy; G[c][2] = gz;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d)
      F[c][d] = G[c][0] * Ji[0][d] + G[c][1] * Ji[1][d] + G[c][2] * Ji[2][d] + (c == d ? T(1) : T(0));
}

// Shared-memory layout of the row sweeps, chosen per (degree, element size)
// by a wavefront count of every warp access of the sweeps (32 banks of 4
// bytes; 8-byte words served per half warp) so that the transposes between
// sweeps are free of bank conflicts where the unpadded tensors allow it:
//   X0..X2: order in which the x sweep (and the gather / scatter) enumerates
//           its rows (c, k, j) over the lanes, fastest first (ids 0 = c,
//           1 = k, 2 = j);
//   Y0..Y2: the same for the y sweep rows (0 = c, 1 = k, 2 = qx);
//   Z0..Z2: the same for the z sweep rows (0 = c, 1 = qy, 2 = qx);
//   AC, AK, AJ, AQ: strides of the x-sweep output A[c][k][j][qx] (and of
//           the y-sweep output of integrate);
//   BC, BK, BY, BX: strides of the y-sweep output B[c][k][qy][qx] (and of
//           the z-sweep output of integrate);
//   NQP:    stride of the 9 per-point blocks (c, e) of the point tensor.
template <int P, int ES>
struct SFRLayout {  // generic: the natural orders, no padding
  static constexpr int N1 = P + 1;
  static constexpr int X0 = 2, X1 = 1, X2 = 0, Y0 = 2, Y1 = 1, Y2 = 0, Z0 = 2, Z1 = 1, Z2 = 0;
  static constexpr int AC = N1 * N1 * N1, AK = N1 * N1, AJ = N1, AQ = 1;
  static constexpr int BC = N1 * N1 * N1, BK = N1 * N1, BY = N1, BX = 1;
  static constexpr int NQP = N1 * N1 * N1;
};
// Q1 / Q2 with 8-byte (FP64) and 4-byte (FP32) entries.  Wavefronts per
// cell of the sweeps and point accesses, natural -> chosen: Q2 FP64 306 ->
// 192 and Q2 FP32 162 -> 96 (both conflict-free), Q1 FP64 122 -> 110.  For
// Q3 / Q4 the best orders with unpadded A / B save under 10 % of the
// wavefronts and measured slower (FP32 Q4 0.73 -> 1.08 ms), so they keep the
// natural layout.
template <int P, int Y0_, int Y1_, int Y2_, int Z0_, int Z1_, int Z2_, int NQP_>
struct SFRLayoutYZ : SFRLayout<P, 0> {
  static constexpr int Y0 = Y0_, Y1 = Y1_, Y2 = Y2_, Z0 = Z0_, Z1 = Z1_, Z2 = Z2_, NQP = NQP_;
};
template <> struct SFRLayout<1, 8> : SFRLayoutYZ<1, 0, 1, 2, 0, 1, 2, 9> {};
template <> struct SFRLayout<1, 4> : SFRLayoutYZ<1, 0, 1, 2, 0, 1, 2, 8> {};
template <> struct SFRLayout<2, 8> : SFRLayoutYZ<2, 1, 0, 2, 0, 2, 1, 41> {};
// FP32 Q2: x rows with the component fastest (the three components of a node
// are gathered by neighbouring lanes), A[j][c][k][qx], B[k][c][qx][qy]
template <> struct SFRLayout<2, 4> : SFRLayoutYZ<2, 0, 1, 2, 0, 1, 2, 29> {
  static constexpr int X0 = 0, X1 = 1, X2 = 2;
  static constexpr int AC = 9, AK = 3, AJ = 27, AQ = 1;
  static constexpr int BC = 9, BK = 27, BY = 1, BX = 3;
};
// Q4 FP32: conflict-free sweeps with reordered intermediate tensors
// (A[qx][c][k][j], B[qy][qx][c][k]).  The conflict-free orders found for Q3
// and for Q4 FP64 measured slower for tensor4 (FP64 Q4 1.36 -> 1.98 ms), so
// those keep the natural layout.
template <> struct SFRLayout<4, 4> : SFRLayoutYZ<4, 1, 0, 2, 0, 2, 1, 153> {
  static constexpr int AC = 25, AK = 5, AJ = 1, AQ = 75;
  static constexpr int BC = 5, BK = 1, BY = 75, BX = 15;
};

// row -> its three indices (by id) for an enumeration (I0 fastest, I2
// slowest) over index ranges D[id]
template <int I0, int I1, int I2, int DA, int DB, int DC>
__device__ __forceinline__ void decode_row(int row, int idx[3]) {
  constexpr int D[3] = {DA, DB, DC};
  idx[I0] = row % D[I0];
  idx[I1] = (row / D[I0]) % D[I1];
  idx[I2] = row / (D[I0] * D[I1]);
}

// Visit the rows lane, lane + 32, ... of a sweep with NR rows: f(row, act).
// CLAMP with NR <= 32: every lane takes one row, lanes past the end repeat
// the last row (act = false: they compute, but store nothing), so the sweep
// has no divergent branch.
template <int NR, bool CLAMP, typename F>
__device__ __forceinline__ void rows_of_lane(int lane, F &&f) {
  if constexpr (CLAMP && NR <= 32) {
    f(lane < NR ? lane : NR - 1, lane < NR);
  } else {
    for (int row = lane; row < NR; row += 32) f(row, true);
  }
}

// Sum factorisation with one 1D line per lane ("row" sweeps).  Each sweep
// maps lane -> row of the tensor it produces and unrolls the 1D contraction
// completely; shared memory only carries the transposes between sweeps.
//   eval:      src rows (c,k,j) in registers -> A (x) -> B (y) -> G (z) ->
//              per-point gradient registers
//   integrate: per-point H -> Z (z) -> Y (y) -> per-row nodal values (x)
// Slab layout (elements of T): [9*NQ points][2*NA][3*NB].
// CLAMP: with at most 32 rows / points per sweep, the lanes past the end
// repeat the last row or point and only their stores are skipped (no
// divergent branches; measured faster for the scalar variants, whose
// kernels carry the most registers, and slower for tensor2)
template <int P, int Q, typename T, bool CLAMP = false>
struct SFR {
  using LY = SFRLayout<P, (int)sizeof(T)>;
  static constexpr int N1 = P + 1, NN = N1 * N1 * N1, NQ = Q * Q * Q;
  static constexpr int NQP = (Q == P + 1) ? LY::NQP : NQ;  // point-block stride
  static constexpr int QPL = (NQ + 31) / 32;
  static constexpr int XR = 3 * N1 * N1;      // x rows (c,k,j)
  static constexpr int YR = 3 * N1 * Q;       // y rows (c,k,qx)
  static constexpr int ZR = 3 * Q * Q;        // z rows (c,qy,qx)
  static constexpr int RPL = (XR + 31) / 32;  // x rows per lane
  static constexpr int NA = 3 * N1 * N1 * Q;
  static constexpr int NB = 3 * N1 * Q * Q;
  static constexpr int SZP = 9 * NQP;
  static constexpr int SZ = SZP + 2 * NA + 3 * NB;

  // v[r][i]: value of component c at node (i, j, k) for x row r = lane + 32 r;
  // the reference gradients are left in the point block of the slab,
  // Pt[(c * 3 + e) * NQP + q]
  // x row (component c, node line (k, j)) of a lane: row -> (c, k, j)
  static __device__ __forceinline__ void x_row(int row, int &c, int &k, int &j) {
    int ix[3];
    decode_row<LY::X0, LY::X1, LY::X2, 3, N1, N1>(row, ix);
    c = ix[0]; k = ix[1]; j = ix[2];
  }
  static __device__ __forceinline__ int a_at(int c, int k, int j, int qx) {
    return c * LY::AC + k * LY::AK + j * LY::AJ + qx * LY::AQ;
  }
  static __device__ __forceinline__ int b_at(int c, int k, int qy, int qx) {
    return c * LY::BC + k * LY::BK + qy * LY::BY + qx * LY::BX;
  }

  static __device__ __forceinline__ void eval_pt(const TabT<P, Q, T> &t, const T v[RPL][N1], T *slab, int lane) {
    T *Pt = slab, *A = slab + SZP, *B = A + 2 * NA;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row0 = lane + 32 * r;
      if ((CLAMP && XR <= 32) || row0 < XR) {
        const bool act = row0 < XR;
        int c, k, j;
        x_row(act ? row0 : XR - 1, c, k, j);
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          T s0 = 0, s1 = 0;
#pragma unroll
          for (int i = 0; i < N1; ++i) {
            s0 += t.N[qx][i] * v[r][i];
            s1 += t.D[qx][i] * v[r][i];
          }
          if (act) {
            A[a_at(c, k, j, qx)] = s0;
            A[NA + a_at(c, k, j, qx)] = s1;
          }
        }
      }
    }
    __syncwarp();
    rows_of_lane<YR, CLAMP>(lane, [&](int row, bool act) {
      int ix[3];
      decode_row<LY::Y0, LY::Y1, LY::Y2, 3, N1, Q>(row, ix);
      const int c = ix[0], k = ix[1], qx = ix[2];
      T a0[N1], a1[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        a0[j] = A[a_at(c, k, j, qx)];
        a1[j] = A[NA + a_at(c, k, j, qx)];
      }
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        T s00 = 0, s01 = 0, s10 = 0;
#pragma unroll
        for (int j = 0; j < N1; ++j) {
          s00 += t.N[qy][j] * a0[j];
          s01 += t.D[qy][j] * a0[j];
          s10 += t.N[qy][j] * a1[j];
        }
        const int b = b_at(c, k, qy, qx);
        if (act) {
          B[b] = s00;
          B[NB + b] = s01;
          B[2 * NB + b] = s10;
        }
      }
    });
    __syncwarp();
    rows_of_lane<ZR, CLAMP>(lane, [&](int row, bool act) {
      int ix[3];
      decode_row<LY::Z0, LY::Z1, LY::Z2, 3, Q, Q>(row, ix);
      const int qyx = ix[1] * Q + ix[2], c = ix[0];
      T b00[N1], b01[N1], b10[N1];
#pragma unroll
      for (int k = 0; k < N1; ++k) {
        const int b = b_at(c, k, ix[1], ix[2]);
        b00[k] = B[b];
        b01[k] = B[NB + b];
        b10[k] = B[2 * NB + b];
      }
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) {
        T gx = 0, gy = 0, gz = 0;
#pragma unroll
        for (int k = 0; k < N1; ++k) {
          gx += t.N[qz][k] * b10[k];
          gy += t.N[qz][k] * b01[k];
          gz += t.D[qz][k] * b00[k];
        }
        const int q = qz * Q * Q + qyx;
        if (act) {
          Pt[(c * 3 + 0) * NQP + q] = gx;
          Pt[(c * 3 + 1) * NQP + q] = gy;
          Pt[(c * 3 + 2) * NQP + q] = gz;
        }
      }
    });
    __syncwarp();
  }

  // eval_pt, then the gradients of the points lane + 32 l into registers
  static __device__ __forceinline__ void eval(const TabT<P, Q, T> &t, const T v[RPL][N1], T *slab, int lane,
                                              T G[QPL][3][3]) {
    eval_pt(t, v, slab, lane);
    const T *Pt = slab;
#pragma unroll
    for (int l = 0; l < QPL; ++l) {
      // lanes past the last point read the last point (no divergent branch)
      const int q = (CLAMP && NQ <= 32) ? (lane < NQ ? lane : NQ - 1) : lane + 32 * l;
      if ((CLAMP && NQ <= 32) || q < NQ) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int e = 0; e < 3; ++e) G[l][c][e] = Pt[(c * 3 + e) * NQP + q];
      }
    }
    __syncwarp();
  }

  // per-point H -> out[r][i] for x row r (component c, node (i, j, k))
  static __device__ __forceinline__ void integrate(const TabT<P, Q, T> &t, const T H[QPL][3][3], T *slab, int lane,
                                                   T out[RPL][N1]) {
    T *Pt = slab;
#pragma unroll
    for (int l = 0; l < QPL; ++l) {
      const int q = lane + 32 * l;
      if (q < NQ) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int e = 0; e < 3; ++e) Pt[(c * 3 + e) * NQP + q] = H[l][c][e];
      }
    }
    integrate_pt(t, slab, lane, out);
  }

  // the same with H already in the point block of the slab
  static __device__ __forceinline__ void integrate_pt(const TabT<P, Q, T> &t, T *slab, int lane, T out[RPL][N1]) {
    T *Pt = slab, *Y = slab + SZP, *Z = Y + 2 * NA;
    __syncwarp();
    rows_of_lane<ZR, CLAMP>(lane, [&](int row, bool act) {
      int ix[3];
      decode_row<LY::Z0, LY::Z1, LY::Z2, 3, Q, Q>(row, ix);
      const int qyx = ix[1] * Q + ix[2], c = ix[0];
      T hx[Q], hy[Q], hz[Q];
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) {
        const int q = qz * Q * Q + qyx;
        hx[qz] = Pt[(c * 3 + 0) * NQP + q];
        hy[qz] = Pt[(c * 3 + 1) * NQP + q];
        hz[qz] = Pt[(c * 3 + 2) * NQP + q];
      }
#pragma unroll
      for (int k = 0; k < N1; ++k) {
        T sx = 0, sy = 0, sz = 0;
#pragma unroll
        for (int qz = 0; qz < Q; ++qz) {
          sx += t.N[qz][k] * hx[qz];
          sy += t.N[qz][k] * hy[qz];
          sz += t.D[qz][k] * hz[qz];
        }
        const int z = b_at(c, k, ix[1], ix[2]);
        if (act) {
          Z[z] = sx;
          Z[NB + z] = sy;
          Z[2 * NB + z] = sz;
        }
      }
    });
    __syncwarp();
    rows_of_lane<YR, CLAMP>(lane, [&](int row, bool act) {
      int ix[3];
      decode_row<LY::Y0, LY::Y1, LY::Y2, 3, N1, Q>(row, ix);
      const int c = ix[0], k = ix[1], qx = ix[2];
      T zx[Q], zy[Q], zz[Q];
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        const int z = b_at(c, k, qy, qx);
        zx[qy] = Z[z];
        zy[qy] = Z[NB + z];
        zz[qy] = Z[2 * NB + z];
      }
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        T sx = 0, so = 0;
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) {
          sx += t.N[qy][j] * zx[qy];
          so += t.D[qy][j] * zy[qy] + t.N[qy][j] * zz[qy];
        }
        const int y = a_at(c, k, j, qx);
        if (act) {
          Y[y] = sx;
          Y[NA + y] = so;
        }
      }
    });
    __syncwarp();
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int row0 = lane + 32 * r;
      // lanes past the last row compute the last row (their out is unused)
      if ((CLAMP && XR <= 32) || row0 < XR) {
        int c, k, j;
        x_row(row0 < XR ? row0 : XR - 1, c, k, j);
        T yx[Q], yo[Q];
#pragma unroll
        for (int qx = 0; qx < Q; ++qx) {
          yx[qx] = Y[a_at(c, k, j, qx)];
          yo[qx] = Y[NA + a_at(c, k, j, qx)];
        }
#pragma unroll
        for (int i = 0; i < N1; ++i) {
          T s = 0;
#pragma unroll
          for (int qx = 0; qx < Q; ++qx) s += t.D[qx][i] * yx[qx] + t.N[qx][i] * yo[qx];
          out[r][i] = s;
        }
      }
    }
    __syncwarp();
  }
};

template <int P, int Q, typename T>
struct SF {
  static constexpr int N1 = P + 1, NN = N1 * N1 * N1, NQ = Q * Q * Q;
  static constexpr int QPL = (NQ + 31) / 32;   // quadrature points per lane
  static constexpr int NPL = (NN + 31) / 32;   // nodes per lane
  static constexpr int NA = 3 * N1 * N1 * Q;   // x-sweep outputs per field
  static constexpr int NB = 3 * N1 * Q * Q;    // y-sweep outputs per field
  static constexpr int SZ1 = (3 * NN > 9 * NQ) ? 3 * NN : 9 * NQ;
  static constexpr int SZ2 = 2 * NA;
  static constexpr int SZ3 = 3 * NB;
  static constexpr int SZ = SZ1 + SZ2 + SZ3;   // per-warp slab (elements of T)
  static constexpr int TAB = 2 * Q * N1;        // sN + sD

  // nodal values V[c][k][j][i] (c*NN + node) -> G[i][c][e] at the owned points
  static __device__ __forceinline__ void eval(const T *__restrict__ sN, const T *__restrict__ sD,
                                              const T *V, T *A, T *B, int lane, T G[QPL][3][3]) {
    for (int it = lane; it < NA; it += 32) {
      const int qx = it % Q, r = it / Q;
      const T *v = V + r * N1;
      T s0 = 0, s1 = 0;
#pragma unroll
      for (int i = 0; i < N1; ++i) {
        const T x = v[i];
        s0 += sN[qx * N1 + i] * x;
        s1 += sD[qx * N1 + i] * x;
      }
      A[it] = s0;
      A[NA + it] = s1;
    }
    __syncwarp();
    for (int it = lane; it < NB; it += 32) {
      const int qx = it % Q, qy = (it / Q) % Q, ck = it / (Q * Q);
      T s00 = 0, s01 = 0, s10 = 0;
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        const T a0 = A[(ck * N1 + j) * Q + qx], a1 = A[NA + (ck * N1 + j) * Q + qx];
        const T nn = sN[qy * N1 + j], dd = sD[qy * N1 + j];
        s00 += nn * a0;
        s01 += dd * a0;
        s10 += nn * a1;
      }
      B[it] = s00;
      B[NB + it] = s01;
      B[2 * NB + it] = s10;
    }
    __syncwarp();
#pragma unroll
    for (int l = 0; l < QPL; ++l) {
      const int q = lane + 32 * l;
      if (q < NQ) {
        const int qx = q % Q, qy = (q / Q) % Q, qz = q / (Q * Q);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          T gx = 0, gy = 0, gz = 0;
#pragma unroll
          for (int k = 0; k < N1; ++k) {
            const int b = ((c * N1 + k) * Q + qy) * Q + qx;
            const T nn = sN[qz * N1 + k];
            gx += nn * B[2 * NB + b];
            gy += nn * B[NB + b];
            gz += sD[qz * N1 + k] * B[b];
          }
          G[l][c][0] = gx;
          G[l][c][1] = gy;
          G[l][c][2] = gz;
        }
      }
    }
    __syncwarp();
  }

  // H[i][c][e] at owned points -> nodal values out[c][node] in smem Yout
  // (= the V region), the transpose of eval().
  static __device__ __forceinline__ void integrate(const T *__restrict__ sN, const T *__restrict__ sD,
                                                   const T H[QPL][3][3], T *Hs, T *Y, T *Z, int lane) {
#pragma unroll
    for (int l = 0; l < QPL; ++l) {
      const int q = lane + 32 * l;
      if (q < NQ) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int e = 0; e < 3; ++e) Hs[(c * 3 + e) * NQ + q] = H[l][c][e];
      }
    }
    __syncwarp();
    // z: Z[c][k][qy][qx] for the three gradient directions
    for (int it = lane; it < NB; it += 32) {
      const int qx = it % Q, qy = (it / Q) % Q, ck = it / (Q * Q);
      const int c = ck / N1, k = ck % N1;
      T sx = 0, sy = 0, sz = 0;
#pragma unroll
      for (int qz = 0; qz < Q; ++qz) {
        const int q = (qz * Q + qy) * Q + qx;
        const T nn = sN[qz * N1 + k];
        sx += nn * Hs[(c * 3 + 0) * NQ + q];
        sy += nn * Hs[(c * 3 + 1) * NQ + q];
        sz += sD[qz * N1 + k] * Hs[(c * 3 + 2) * NQ + q];
      }
      Z[it] = sx;
      Z[NB + it] = sy;
      Z[2 * NB + it] = sz;
    }
    __syncwarp();
    // y: Yx[c][k][j][qx], Yo[c][k][j][qx]
    for (int it = lane; it < NA; it += 32) {
      const int qx = it % Q, j = (it / Q) % N1, ck = it / (Q * N1);
      T sx = 0, so = 0;
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        const int z = (ck * Q + qy) * Q + qx;
        const T nn = sN[qy * N1 + j];
        sx += nn * Z[z];
        so += sD[qy * N1 + j] * Z[NB + z] + nn * Z[2 * NB + z];
      }
      Y[it] = sx;
      Y[NA + it] = so;
    }
    __syncwarp();
  }

  // final x sweep for node a = (i, j, k): 3 component values
  static __device__ __forceinline__ void integrate_node(const T *__restrict__ sN, const T *__restrict__ sD,
                                                        const T *Y, int a, T out[3]) {
    const int i = a % N1, jk = a / N1;  // jk = k*N1 + j
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int base = ((c * N1 * N1) + jk) * Q;
      T s = 0;
#pragma unroll
      for (int qx = 0; qx < Q; ++qx) s += sD[qx * N1 + i] * Y[base + qx] + sN[qx * N1 + i] * Y[NA + base + qx];
      out[c] = s;
    }
  }
};

// --------------------------------------------------------------- physics
// symmetric storage (0,0),(1,1),(2,2),(0,1),(0,2),(1,2)
__device__ __forceinline__ int sym_i(int I) { return I < 3 ? I : (I == 5 ? 1 : 0); }
__device__ __forceinline__ int sym_j(int I) { return I < 3 ? I : (I == 3 ? 1 : 2); }

template <typename T>
__device__ __forceinline__ T det3(const T F[3][3]) {
  return F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) - F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
         F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
}
template <typename T>
__device__ __forceinline__ T inv3(const T J[3][3], T Ji[3][3]) {
  const T d = det3(J);
  const T id = T(1) / d;
  Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
  Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
  Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
  Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  return d;
}

// Per-point state of the scalar variants (computed from the displacement).
template <typename T>
struct ScalarState {
  T F[3][3];
  T det;
};

// Q(g) of do_operation_on_cell (mf_nh_operator.h:922-1499) for the point
// whose record is rec[comp * NQ] (rec already offset by q; a pointer, or an
// accessor with operator[] such as the record pair of two cells); for the
// variants that fold JxW into their coefficients Q(g) comes out times JxW.
template <typename T, int VAR, int NQ, typename R>
__device__ __forceinline__ void physics(const T g[3][3], const R &rec, T mu, T lambda, T kappa,
                                        const ScalarState<T> &st, T Qm[3][3]) {
  constexpr int CV = variant_cvar(VAR);
  T s[6];
#pragma unroll
  for (int I = 0; I < 6; ++I) s[I] = T(0.5) * (g[sym_i(I)][sym_j(I)] + g[sym_j(I)][sym_i(I)]);
  const T tr = s[0] + s[1] + s[2];
  if (VAR == VAR_TENSOR4) {
    // g * (tau/J) + C : sym(g)     (mf_nh_operator.h:1425-1440)
    T Ts[6];
#pragma unroll
    for (int I = 0; I < 6; ++I) Ts[I] = rec[(CV + I) * NQ];
    T cs[6];
#pragma unroll
    for (int I = 0; I < 6; ++I) {
      T a = 0;
#pragma unroll
      for (int J = 0; J < 6; ++J) a += rec[(CV + 6 + I * 6 + J) * NQ] * s[J];
      cs[I] = a;
    }
    const T T00 = Ts[0], T11 = Ts[1], T22 = Ts[2], T01 = Ts[3], T02 = Ts[4], T12 = Ts[5];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      Qm[i][0] = g[i][0] * T00 + g[i][1] * T01 + g[i][2] * T02;
      Qm[i][1] = g[i][0] * T01 + g[i][1] * T11 + g[i][2] * T12;
      Qm[i][2] = g[i][0] * T02 + g[i][1] * T12 + g[i][2] * T22;
    }
    Qm[0][0] += cs[0]; Qm[1][1] += cs[1]; Qm[2][2] += cs[2];
    Qm[0][1] += cs[3]; Qm[1][0] += cs[3];
    Qm[0][2] += cs[4]; Qm[2][0] += cs[4];
    Qm[1][2] += cs[5]; Qm[2][1] += cs[5];
  } else if (VAR == VAR_TENSOR2) {
    // c1 sym(g) + c2 tr(g) I + g * (tau/J)   (mf_nh_operator.h:1401-1424)
    const T c1 = rec[CV * NQ], c2 = rec[(CV + 1) * NQ];
    const T T00 = rec[(CV + 2) * NQ], T11 = rec[(CV + 3) * NQ], T22 = rec[(CV + 4) * NQ];
    const T T01 = rec[(CV + 5) * NQ], T02 = rec[(CV + 6) * NQ], T12 = rec[(CV + 7) * NQ];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      Qm[i][0] = g[i][0] * T00 + g[i][1] * T01 + g[i][2] * T02;
      Qm[i][1] = g[i][0] * T01 + g[i][1] * T11 + g[i][2] * T12;
      Qm[i][2] = g[i][0] * T02 + g[i][1] * T12 + g[i][2] * T22;
    }
#pragma unroll
    for (int I = 0; I < 6; ++I) {
      const int i = sym_i(I), j = sym_j(I);
      const T v = c1 * s[I] + (I < 3 ? c2 * tr : T(0));
      Qm[i][j] += v;
      if (i != j) Qm[j][i] += v;
    }
  } else if (VAR == VAR_TENSOR4_NS) {
    // out_ij = A_ijkl Grad v_kl (double_contract<2,0,3,1>, mf_nh_operator.h:1441-1455)
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        T a = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int l = 0; l < 3; ++l) a += rec[(CV + ((i * 3 + j) * 3 + k) * 3 + l) * NQ] * g[k][l];
        Qm[i][j] = a;
      }
  } else if (VAR == VAR_SCALAR_REF) {
    // mf_nh_operator.h:1255-1400: g = Grad v; grad_x v = Grad v F^-1; the
    // scalar-variant physics; submitted as (jc + grad_x v tau) F^-T
    const T c = rec[C_VAR * NQ];
    T Fi[3][3];
    inv3(st.F, Fi);
    T gx[3][3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int e = 0; e < 3; ++e) gx[d][e] = g[d][0] * Fi[0][e] + g[d][1] * Fi[1][e] + g[d][2] * Fi[2][e];
    T tau[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T b = st.F[i][0] * st.F[j][0] + st.F[i][1] * st.F[j][1] + st.F[i][2] * st.F[j][2];
        tau[i][j] = mu * b - (i == j ? c : T(0));
      }
    const T trx = gx[0][0] + gx[1][1] + gx[2][2];
    T qd[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        T v = c * (gx[i][j] + gx[j][i]);
        if (i == j) v += T(2) * lambda * trx;
        v += gx[i][0] * tau[0][j] + gx[i][1] * tau[1][j] + gx[i][2] * tau[2][j];
        qd[i][j] = v;
      }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Qm[i][j] = qd[i][0] * Fi[j][0] + qd[i][1] * Fi[j][1] + qd[i][2] * Fi[j][2];
  } else if (VAR == VAR_SCALAR_F1) {
    // mf_nh_operator.h:1182-1254: tau = mu b - c I, jc = 2c sym + 2 lambda tr I
    const T c = rec[C_VAR * NQ];
    T jc[6];
#pragma unroll
    for (int I = 0; I < 6; ++I) jc[I] = T(2) * c * s[I] + (I < 3 ? T(2) * lambda * tr : T(0));
    T tau[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T b = st.F[i][0] * st.F[j][0] + st.F[i][1] * st.F[j][1] + st.F[i][2] * st.F[j][2];
        tau[i][j] = mu * b - (i == j ? c : T(0));
      }
    const T idet = T(1) / st.det;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        T geo = g[i][0] * tau[0][j] + g[i][1] * tau[1][j] + g[i][2] * tau[2][j];
        Qm[i][j] = geo;
      }
#pragma unroll
    for (int I = 0; I < 6; ++I) {
      const int i = sym_i(I), j = sym_j(I);
      Qm[i][j] += jc[I];
      if (i != j) Qm[j][i] += jc[I];
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Qm[i][j] *= idet;
  } else {
    // formulation 0 (vol/iso split), mf_nh_operator.h:1001-1181
    const T Jm13 = rec[C_VAR * NQ];
    const T det_F = st.det;
    T bbar[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j)
        bbar[i][j] = (st.F[i][0] * st.F[j][0] + st.F[i][1] * st.F[j][1] + st.F[i][2] * st.F[j][2]) * Jm13 * Jm13;
    const T c_1 = T(0.5) * mu;
    T tau_bar[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) tau_bar[i][j] = bbar[i][j] * (T(2) * c_1);
    const T tr_tau_bar = tau_bar[0][0] + tau_bar[1][1] + tau_bar[2][2];
    const T trd = tr_tau_bar * T(1.0 / 3.0);
    const T dPsi = (kappa / T(2)) * (det_F - T(1) / det_F);
    const T dPsi_J = dPsi * det_F;
    const T d2Psi = (kappa / T(2)) * (T(1) + T(1) / (det_F * det_F));
    T sym[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) sym[i][j] = T(0.5) * (g[i][j] + g[j][i]);
    T tis = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) tis += (tau_bar[i][j] - (i == j ? trd : T(0))) * sym[i][j];
    const T volI = det_F * (dPsi + det_F * d2Psi) * tr;
    const T two3 = T(2.0 / 3.0);
    const T idet = T(1) / det_F;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T tau_iso = tau_bar[i][j] - (i == j ? trd : T(0));
        T v = sym[i][j] * (-dPsi_J * T(2));
        if (i == j) v += volI;
        v += (two3 * tr_tau_bar) * (sym[i][j] - (i == j ? tr * T(1.0 / 3.0) : T(0)));
        v -= (two3 * tr) * tau_iso;
        if (i == j) v -= two3 * tis;
        Qm[i][j] = v;
      }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const T tau_0j = tau_bar[0][j] + (0 == j ? dPsi_J - trd : T(0));
        const T tau_1j = tau_bar[1][j] + (1 == j ? dPsi_J - trd : T(0));
        const T tau_2j = tau_bar[2][j] + (2 == j ? dPsi_J - trd : T(0));
        const T geo = g[i][0] * tau_0j + g[i][1] * tau_1j + g[i][2] * tau_2j;
        Qm[i][j] = (Qm[i][j] + geo) * idet;
      }
  }
}

}  // namespace lsmf
