// CPU oracle (test infrastructure only): per-cell kernels templated on the
// polynomial degree P and the 1D Gauss point count Q.
#pragma once
#include <cmath>
#include <stdexcept>
#include <vector>

#include "oracle.h"

#define DISPATCH_PQ(p, q, ...)                                          \
  do {                                                                  \
    if ((p) == 1 && (q) == 2) { constexpr int P_ = 1, Q_ = 2; __VA_ARGS__ }    \
    else if ((p) == 2 && (q) == 3) { constexpr int P_ = 2, Q_ = 3; __VA_ARGS__ } \
    else if ((p) == 3 && (q) == 4) { constexpr int P_ = 3, Q_ = 4; __VA_ARGS__ } \
    else if ((p) == 4 && (q) == 5) { constexpr int P_ = 4, Q_ = 5; __VA_ARGS__ } \
    else throw std::runtime_error("unsupported (degree, n_q_points_1d)"); \
  } while (0)

namespace orc {

template <typename T>
inline T det3(const T J[3][3]) {
  return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
         J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
         J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}
template <typename T>
inline T inv3(const T J[3][3], T Ji[3][3]) {
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

// symmetric storage order (0,0),(1,1),(2,2),(0,1),(0,2),(1,2)
static const int SYM_I[6] = {0, 1, 2, 0, 0, 1};
static const int SYM_J[6] = {0, 1, 2, 1, 2, 2};

// Fill the 6x6 matrix M with out_I = sum_J M[I][J] s_J representing
// C = a * S + b * I (x) I acting on a symmetric s given by its 6 tensor
// components (mf_nh_operator.h:542-546: C = (2c/J) S + (2 lambda/J) IxI).
template <typename T>
inline void tensor4_from_scalars(T a, T b, T *M) {
  for (int I = 0; I < 6; ++I)
    for (int J = 0; J < 6; ++J) {
      T v = T(0);
      if (I == J) v += a;
      if (I < 3 && J < 3) v += b;
      M[I * 6 + J] = v;
    }
}

template <int P, int Q, typename Number>
struct CellOps {
  static constexpr int N1 = P + 1, NN = N1 * N1 * N1, NQ = Q * Q * Q;
  struct Tables { double N[Q][N1], D[Q][N1], w[NQ]; };

  static void tables(const Basis1D &b, Tables &t) {
    for (int k = 0; k < Q; ++k)
      for (int i = 0; i < N1; ++i) { t.N[k][i] = b.N[k * N1 + i]; t.D[k][i] = b.D[k * N1 + i]; }
    for (int qz = 0; qz < Q; ++qz)
      for (int qy = 0; qy < Q; ++qy)
        for (int qx = 0; qx < Q; ++qx)
          t.w[(qz * Q + qy) * Q + qx] = b.qw[qx] * b.qw[qy] * b.qw[qz];
  }

  // G[c][e][q] = d v_c / d xi_e at quadrature point q, from nodal values
  // in[c*NN + a] (FEEvaluation::evaluate(gradients), sum factorised).
  template <typename T>
  static void grad(const Tables &t, const T *in, T G[3][3][NQ]) {
    for (int c = 0; c < 3; ++c) {
      const T *v = in + c * NN;
      T A0[N1][N1][Q], A1[N1][N1][Q];
      for (int k = 0; k < N1; ++k)
        for (int j = 0; j < N1; ++j)
          for (int qx = 0; qx < Q; ++qx) {
            T s0 = 0, s1 = 0;
            for (int i = 0; i < N1; ++i) {
              const T x = v[(k * N1 + j) * N1 + i];
              s0 += T(t.N[qx][i]) * x; s1 += T(t.D[qx][i]) * x;
            }
            A0[k][j][qx] = s0; A1[k][j][qx] = s1;
          }
      T B00[N1][Q][Q], B01[N1][Q][Q], B10[N1][Q][Q];
      for (int k = 0; k < N1; ++k)
        for (int qy = 0; qy < Q; ++qy)
          for (int qx = 0; qx < Q; ++qx) {
            T s00 = 0, s01 = 0, s10 = 0;
            for (int j = 0; j < N1; ++j) {
              s00 += T(t.N[qy][j]) * A0[k][j][qx];
              s01 += T(t.D[qy][j]) * A0[k][j][qx];
              s10 += T(t.N[qy][j]) * A1[k][j][qx];
            }
            B00[k][qy][qx] = s00; B01[k][qy][qx] = s01; B10[k][qy][qx] = s10;
          }
      for (int qz = 0; qz < Q; ++qz)
        for (int qy = 0; qy < Q; ++qy)
          for (int qx = 0; qx < Q; ++qx) {
            T gx = 0, gy = 0, gz = 0;
            for (int k = 0; k < N1; ++k) {
              gx += T(t.N[qz][k]) * B10[k][qy][qx];
              gy += T(t.N[qz][k]) * B01[k][qy][qx];
              gz += T(t.D[qz][k]) * B00[k][qy][qx];
            }
            const int q = (qz * Q + qy) * Q + qx;
            G[c][0][q] = gx; G[c][1][q] = gy; G[c][2][q] = gz;
          }
    }
  }

  // out[c*NN + a] = sum_q sum_e dN_a/dxi_e(q) H[c][e][q]
  // (FEEvaluation::integrate(gradients), the transpose of grad()).
  template <typename T>
  static void integrate(const Tables &t, const T H[3][3][NQ], T *out) {
    for (int c = 0; c < 3; ++c) {
      T Zx[N1][Q][Q], Zy[N1][Q][Q], Zz[N1][Q][Q];
      for (int k = 0; k < N1; ++k)
        for (int qy = 0; qy < Q; ++qy)
          for (int qx = 0; qx < Q; ++qx) {
            T sx = 0, sy = 0, sz = 0;
            for (int qz = 0; qz < Q; ++qz) {
              const int q = (qz * Q + qy) * Q + qx;
              sx += T(t.N[qz][k]) * H[c][0][q];
              sy += T(t.N[qz][k]) * H[c][1][q];
              sz += T(t.D[qz][k]) * H[c][2][q];
            }
            Zx[k][qy][qx] = sx; Zy[k][qy][qx] = sy; Zz[k][qy][qx] = sz;
          }
      T Yx[N1][N1][Q], Yo[N1][N1][Q];
      for (int k = 0; k < N1; ++k)
        for (int j = 0; j < N1; ++j)
          for (int qx = 0; qx < Q; ++qx) {
            T sx = 0, so = 0;
            for (int qy = 0; qy < Q; ++qy) {
              sx += T(t.N[qy][j]) * Zx[k][qy][qx];
              so += T(t.D[qy][j]) * Zy[k][qy][qx] + T(t.N[qy][j]) * Zz[k][qy][qx];
            }
            Yx[k][j][qx] = sx; Yo[k][j][qx] = so;
          }
      for (int k = 0; k < N1; ++k)
        for (int j = 0; j < N1; ++j)
          for (int i = 0; i < N1; ++i) {
            T s = 0;
            for (int qx = 0; qx < Q; ++qx)
              s += T(t.D[qx][i]) * Yx[k][j][qx] + T(t.N[qx][i]) * Yo[k][j][qx];
            out[c * NN + (k * N1 + j) * N1 + i] = s;
          }
    }
  }

  static void gather(const Operator<Number> &op, int cell, const Number *vec,
                     bool zero_constrained, Number *loc) {
    const int *nodes = &op.mesh->cell_nodes[(size_t)cell * NN];
    for (int a = 0; a < NN; ++a)
      for (int c = 0; c < 3; ++c) {
        const size_t dof = 3 * (size_t)nodes[a] + c;
        loc[c * NN + a] = (zero_constrained && op.cmask[dof]) ? Number(0) : vec[dof];
      }
  }
  static void scatter(const Operator<Number> &op, int cell, const Number *loc, Number *vec) {
    const int *nodes = &op.mesh->cell_nodes[(size_t)cell * NN];
    for (int a = 0; a < NN; ++a)
      for (int c = 0; c < 3; ++c) {
        const size_t dof = 3 * (size_t)nodes[a] + c;
        if (!op.cmask[dof]) vec[dof] += loc[c * NN + a];
      }
  }

  // ---- quadrature-point physics of do_operation_on_cell (f1/f0 branches)
  // g: gradient of src in the current configuration.  Q out is what
  // FEEvaluation::submit_gradient receives.
  static void qp_physics(const Operator<Number> &op, int cell, size_t qi,
                         const Number g[3][3], const Number *Gu_ref /*3x3 grad u*/,
                         Number Qm[3][3]) {
    const int caching = op.caching;
    Number s[6];
    for (int I = 0; I < 6; ++I) s[I] = Number(0.5) * (g[SYM_I[I]][SYM_J[I]] + g[SYM_J[I]][SYM_I[I]]);
    if (caching == CACHE_TENSOR4) {
      // mf_nh_operator.h:1425-1440: out = g * (tau/J) + C : sym(g)
      const Number *T = &op.c_t2[6 * qi];
      const Number *M = &op.c_t4[36 * qi];
      Number Ts[3][3];
      for (int I = 0; I < 6; ++I) Ts[SYM_I[I]][SYM_J[I]] = Ts[SYM_J[I]][SYM_I[I]] = T[I];
      Number cs[6];
      for (int I = 0; I < 6; ++I) {
        Number a = 0;
        for (int J = 0; J < 6; ++J) a += M[I * 6 + J] * s[J];
        cs[I] = a;
      }
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          Number a = 0;
          for (int k = 0; k < 3; ++k) a += g[i][k] * Ts[k][j];
          Qm[i][j] = a;
        }
      for (int I = 0; I < 6; ++I) {
        Qm[SYM_I[I]][SYM_J[I]] += cs[I];
        if (SYM_I[I] != SYM_J[I]) Qm[SYM_J[I]][SYM_I[I]] += cs[I];
      }
      return;
    }
    if (caching == CACHE_TENSOR2) {
      // mf_nh_operator.h:1401-1424: c1 sym(g) + c2 tr(g) I + g * (tau/J)
      const Number c1 = op.c_scalar[qi], c2 = op.c_second[qi];
      const Number *T = &op.c_t2[6 * qi];
      Number Ts[3][3];
      for (int I = 0; I < 6; ++I) Ts[SYM_I[I]][SYM_J[I]] = Ts[SYM_J[I]][SYM_I[I]] = T[I];
      const Number tr = s[0] + s[1] + s[2];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          Number a = 0;
          for (int k = 0; k < 3; ++k) a += g[i][k] * Ts[k][j];
          Number sij = Number(0.5) * (g[i][j] + g[j][i]);
          Qm[i][j] = c1 * sij + (i == j ? c2 * tr : Number(0)) + a;
        }
      return;
    }
    if (caching == CACHE_TENSOR4_NS) {
      // out_ij = A_ijkl Grad v_kl (double_contract<2,0,3,1>, :1441-1455)
      const Number *A = &op.c_t4ns[81 * qi];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          Number a = 0;
          for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) a += A[((i * 3 + j) * 3 + k) * 3 + l] * g[k][l];
          Qm[i][j] = a;
        }
      return;
    }
    // scalar caching: F from grad u in the reference configuration
    const double mu = op.mu_cell[cell];
    const Material mat(mu, op.nu, op.formulation);
    Number F[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) F[i][j] = Gu_ref[i * 3 + j] + (i == j ? Number(1) : Number(0));
    const Number det_F = det3(F);
    Number tau[3][3], jc[3][3];
    const Number tr = s[0] + s[1] + s[2];
    if (op.formulation == 1) {
      // mf_nh_operator.h:1182-1254
      const Number c = op.c_scalar[qi];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          Number b = 0;
          for (int k = 0; k < 3; ++k) b += F[i][k] * F[j][k];
          tau[i][j] = Number(mu) * b - (i == j ? c : Number(0));
          Number sij = Number(0.5) * (g[i][j] + g[j][i]);
          jc[i][j] = Number(2.0) * c * sij + (i == j ? Number(2.0) * Number(mat.lambda) * tr : Number(0));
        }
    } else {
      // formulation 0, mf_nh_operator.h:1001-1181
      const Number kappa = Number(mat.kappa), c_1 = Number(mat.c1);
      const Number Jm13 = op.c_scalar[qi];  // det_F^{-1/dim}
      Number Fb[3][3], bbar[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Fb[i][j] = F[i][j] * Jm13;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          Number b = 0;
          for (int k = 0; k < 3; ++k) b += Fb[i][k] * Fb[j][k];
          bbar[i][j] = b;
        }
      Number tau_bar[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) tau_bar[i][j] = bbar[i][j] * (Number(2.0) * c_1);
      const Number tr_tau_bar = tau_bar[0][0] + tau_bar[1][1] + tau_bar[2][2];
      const Number tr_tau_bar_dim = tr_tau_bar * Number(1.0 / 3.0);
      const Number dPsi = (kappa / Number(2.0)) * (det_F - Number(1.0) / det_F);
      const Number dPsi_J = dPsi * det_F;
      const Number d2Psi = (kappa / Number(2.0)) * (Number(1.0) + Number(1.0) / (det_F * det_F));
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          tau[i][j] = tau_bar[i][j] + (i == j ? dPsi_J - tr_tau_bar_dim : Number(0));
      Number tau_iso[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) tau_iso[i][j] = tau_bar[i][j] - (i == j ? tr_tau_bar_dim : Number(0));
      Number sym[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) sym[i][j] = Number(0.5) * (g[i][j] + g[j][i]);
      Number tau_iso_src = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) tau_iso_src += tau_iso[i][j] * sym[i][j];
      const Number volI = det_F * (dPsi + det_F * d2Psi) * tr;
      const Number two_over_dim = Number(2.0 / 3.0);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          Number dev = sym[i][j] - (i == j ? tr * Number(1.0 / 3.0) : Number(0));
          Number v = sym[i][j] * (-dPsi_J * Number(2.0));
          if (i == j) v += volI;
          v += (two_over_dim * tr_tau_bar) * dev;
          v -= (two_over_dim * tr) * tau_iso[i][j];
          if (i == j) v -= two_over_dim * tau_iso_src;
          jc[i][j] = v;
        }
    }
    const Number inv_det_F = Number(1.0) / det_F;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        Number geo = 0;
        for (int k = 0; k < 3; ++k) geo += g[i][k] * tau[k][j];
        Qm[i][j] = (jc[i][j] + geo) * inv_det_F;
      }
  }

  // scalar_referential (mf_nh_operator.h:1255-1400): g = Grad v in the
  // reference configuration; grad_x v = Grad v F^-1, tau and jc as in the
  // scalar variant, submitted as (jc + grad_x v tau) F^-T (no 1/J: the
  // integration is over the reference configuration)
  static void qp_physics_sr(const Operator<Number> &op, int cell, size_t qi, const Number g[3][3],
                            const Number *Gu_ref, Number Qm[3][3]) {
    const double mu = op.mu_cell[cell];
    const Material mat(mu, op.nu, 1);
    Number F[3][3], Fi[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) F[i][j] = Gu_ref[i * 3 + j] + (i == j ? Number(1) : Number(0));
    inv3(F, Fi);
    Number gx[3][3];
    for (int d = 0; d < 3; ++d)
      for (int e = 0; e < 3; ++e) {
        Number a = 0;
        for (int f = 0; f < 3; ++f) a += g[d][f] * Fi[f][e];
        gx[d][e] = a;
      }
    const Number c = op.c_scalar[qi];
    Number tau[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        Number b = 0;
        for (int k = 0; k < 3; ++k) b += F[i][k] * F[j][k];
        tau[i][j] = Number(mu) * b - (i == j ? c : Number(0));
      }
    const Number tr = gx[0][0] + gx[1][1] + gx[2][2];
    Number qd[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        Number v = Number(2.0) * c * Number(0.5) * (gx[i][j] + gx[j][i]);
        if (i == j) v += Number(2.0) * Number(mat.lambda) * tr;
        for (int k = 0; k < 3; ++k) v += gx[i][k] * tau[k][j];
        qd[i][j] = v;
      }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        Number a = 0;
        for (int k = 0; k < 3; ++k) a += qd[i][k] * Fi[j][k];  // queued * F^-T
        Qm[i][j] = a;
      }
  }

  // Cell operator on a local (component-blocked) vector; metric and cache
  // must be available (mf_nh_operator.h:922-1499).
  static void cell_apply_tables(const Tables &t, const Operator<Number> &op, int cell,
                                const Number *in, Number *out) {
    Number G[3][3][NQ], H[3][3][NQ];
    grad(t, in, G);
    Number Gu[3][3][NQ];
    const bool need_u = op.caching == CACHE_SCALAR || op.caching == CACHE_SCALAR_REFERENTIAL;
    if (need_u) {
      Number uloc[3 * NN];
      gather(op, cell, op.u.data(), false, uloc);  // read_dof_values_plain(u)
      grad(t, uloc, Gu);
    }
    const bool ref = op.referential();
    for (int q = 0; q < NQ; ++q) {
      const size_t qi = (size_t)cell * NQ + q;
      const Number *Ji = ref ? &op.jinv_ref[9 * qi] : &op.jinv_cur[9 * qi];
      Number g[3][3];
      for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d) {
          Number a = 0;
          for (int e = 0; e < 3; ++e) a += G[c][e][q] * Ji[e * 3 + d];
          g[c][d] = a;
        }
      Number gu[9];
      if (need_u) {
        const Number *Jr = &op.jinv_ref[9 * qi];
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) {
            Number a = 0;
            for (int e = 0; e < 3; ++e) a += Gu[c][e][q] * Jr[e * 3 + d];
            gu[c * 3 + d] = a;
          }
      }
      Number Qm[3][3];
      if (op.caching == CACHE_SCALAR_REFERENTIAL) qp_physics_sr(op, cell, qi, g, gu, Qm);
      else qp_physics(op, cell, qi, g, gu, Qm);
      const Number jxw = ref ? op.jxw_ref[qi] : op.jxw_cur[qi];
      for (int c = 0; c < 3; ++c)
        for (int e = 0; e < 3; ++e) {
          Number a = 0;
          for (int d = 0; d < 3; ++d) a += Qm[c][d] * Ji[e * 3 + d];
          H[c][e][q] = a * jxw;
        }
    }
    integrate(t, H, out);
  }

  static void cell_apply(const Operator<Number> &op, int cell, const Number *in, Number *out) {
    Tables t; tables(*op.basis, t);
    cell_apply_tables(t, op, cell, in, out);
  }

  static void colours(const Mesh &m, std::vector<std::vector<int>> &col) {
    col.assign(8, {});
    for (int c = 0; c < m.n_cells; ++c) {
      int k = (m.cell_ijk[3 * c] & 1) + 2 * (m.cell_ijk[3 * c + 1] & 1) + 4 * (m.cell_ijk[3 * c + 2] & 1);
      col[k].push_back(c);
    }
  }

  static void apply_all(const Operator<Number> &op, Number *dst, const Number *src,
                        bool zero_constrained = true) {
    Tables t; tables(*op.basis, t);
    std::vector<std::vector<int>> col; colours(*op.mesh, col);
    for (int k = 0; k < 8; ++k) {
      const std::vector<int> &cells = col[k];
      const long n = (long)cells.size();
#pragma omp parallel for schedule(static)
      for (long ii = 0; ii < n; ++ii) {
        const int cell = cells[ii];
        Number in[3 * NN], out[3 * NN];
        gather(op, cell, src, zero_constrained, in);   // read_dof_values(src)
        cell_apply_tables(t, op, cell, in, out);
        scatter(op, cell, out, dst);       // distribute_local_to_global
      }
    }
  }

  static void diagonal_all(const Operator<Number> &op, Number *diag) {
    Tables t; tables(*op.basis, t);
    std::vector<std::vector<int>> col; colours(*op.mesh, col);
    for (int k = 0; k < 8; ++k) {
      const std::vector<int> &cells = col[k];
      const long n = (long)cells.size();
#pragma omp parallel for schedule(static)
      for (long ii = 0; ii < n; ++ii) {
        const int cell = cells[ii];
        Number in[3 * NN], out[3 * NN], dl[3 * NN];
        for (int i = 0; i < 3 * NN; ++i) {
          for (int j = 0; j < 3 * NN; ++j) in[j] = Number(0);
          in[i] = Number(1);
          cell_apply_tables(t, op, cell, in, out);
          dl[i] = out[i];
        }
        scatter(op, cell, dl, diag);
      }
    }
  }

  // cache(): reference-configuration loop over u (mf_nh_operator.h:447-592),
  // together with the reference (StaticMappingQ1) and Eulerian
  // (MappingQEulerian(p, u)) metric of MatrixFree (mf_elasticity.h:1821-1831,
  // 1949-1951).  Metric arithmetic is double, stored as Number.
  static int cache_all(Operator<Number> &op) {
    Tables t; tables(*op.basis, t);
    const Mesh &m = *op.mesh;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int cell = 0; cell < m.n_cells; ++cell) {
      const int *nodes = &m.cell_nodes[(size_t)cell * NN];
      double xl[3 * NN], ul[3 * NN];
      for (int a = 0; a < NN; ++a)
        for (int c = 0; c < 3; ++c) {
          xl[c * NN + a] = m.X[3 * (size_t)nodes[a] + c];
          ul[c * NN + a] = (double)op.u[3 * (size_t)nodes[a] + c];
        }
      double GX[3][3][NQ], GU[3][3][NQ];
      grad(t, xl, GX);
      grad(t, ul, GU);
      // displacement gradient for the cache in Number precision
      Number uN[3 * NN];
      for (int i = 0; i < 3 * NN; ++i) uN[i] = op.u[3 * (size_t)nodes[i % NN] + i / NN];
      Number GUN[3][3][NQ];
      grad(t, uN, GUN);
      const double mu = op.mu_cell[cell];
      const Material mat(mu, op.nu, op.formulation);
      for (int q = 0; q < NQ; ++q) {
        const size_t qi = (size_t)cell * NQ + q;
        double Jr[3][3], Jc[3][3], Jri[3][3], Jci[3][3];
        for (int d = 0; d < 3; ++d)
          for (int e = 0; e < 3; ++e) {
            Jr[d][e] = GX[d][e][q];
            Jc[d][e] = GX[d][e][q] + GU[d][e][q];
          }
        const double dr = inv3(Jr, Jri), dc = inv3(Jc, Jci);
        for (int i = 0; i < 9; ++i) {
          op.jinv_ref[9 * qi + i] = Number(Jri[i / 3][i % 3]);
          op.jinv_cur[9 * qi + i] = Number(Jci[i / 3][i % 3]);
        }
        op.jxw_ref[qi] = Number(dr * t.w[q]);
        op.jxw_cur[qi] = Number(dc * t.w[q]);
        // F = I + Grad u in Number precision (phi_reference.get_gradient)
        Number Jrn[3][3];
        for (int d = 0; d < 3; ++d)
          for (int e = 0; e < 3; ++e) Jrn[d][e] = Number(Jri[d][e]);
        Number F[3][3];
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) {
            Number a = 0;
            for (int e = 0; e < 3; ++e) a += GUN[c][e][q] * Jrn[e][d];
            F[c][d] = a + (c == d ? Number(1) : Number(0));
          }
        const Number det_F = det3(F);
        if (!(det_F > Number(0))) { bad = 1; continue; }
        if (op.formulation == 0) {
          op.c_scalar[qi] = std::pow(det_F, Number(-1.0 / 3.0));
          continue;
        }
        const Number scalar = Number(mat.mu) - Number(2.0) * Number(mat.lambda) * std::log(det_F);
        if (op.caching == CACHE_SCALAR) { op.c_scalar[qi] = scalar; continue; }
        if (op.caching == CACHE_SCALAR_REFERENTIAL) {
          // c and the displacement values at the point (phi_reference.begin_values())
          op.c_scalar[qi] = scalar;
          const int qx = q % Q, qy = (q / Q) % Q, qz = q / (Q * Q);
          for (int c = 0; c < 3; ++c) {
            Number v = 0;
            for (int kz = 0; kz < N1; ++kz)
              for (int jy = 0; jy < N1; ++jy)
                for (int ix = 0; ix < N1; ++ix)
                  v += Number(t.N[qx][ix] * t.N[qy][jy] * t.N[qz][kz]) * uN[c * NN + (kz * N1 + jy) * N1 + ix];
            op.c_second[3 * qi + c] = v;
          }
          continue;
        }
        if (op.caching == CACHE_TENSOR4_NS) {
          // 2 lambda F^-T (x) F^-T + (mu - 2 lambda ln J) F^-T_il F^-1_jk + mu I_ik I_jl
          Number Fi[3][3];
          inv3(F, Fi);
          const Number lnJ = std::log(det_F);
          for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
              for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l)
                  op.c_t4ns[81 * qi + ((i * 3 + j) * 3 + k) * 3 + l] =
                      Number(2.0) * Number(mat.lambda) * Fi[j][i] * Fi[l][k] +
                      (Number(mat.mu) - Number(2.0) * Number(mat.lambda) * lnJ) * Fi[l][i] * Fi[j][k] +
                      (i == k && j == l ? Number(mat.mu) : Number(0));
          continue;
        }
        Number tau[6];
        for (int I = 0; I < 6; ++I) {
          const int i = SYM_I[I], j = SYM_J[I];
          Number b = 0;
          for (int k = 0; k < 3; ++k) b += F[i][k] * F[j][k];
          tau[I] = Number(mat.mu) * b - (i == j ? scalar : Number(0));
        }
        if (op.caching == CACHE_TENSOR2) {
          op.c_scalar[qi] = scalar * Number(2.0) / det_F;
          op.c_second[qi] = Number(2.0) * Number(mat.lambda) / det_F;
          for (int I = 0; I < 6; ++I) op.c_t2[6 * qi + I] = tau[I] / det_F;
        } else {
          for (int I = 0; I < 6; ++I) op.c_t2[6 * qi + I] = tau[I] / det_F;
          tensor4_from_scalars(scalar * Number(2.0) / det_F,
                               Number(mat.lambda) * Number(2.0) / det_F, &op.c_t4[36 * qi]);
        }
      }
    }
    return bad;
  }
};

}  // namespace orc
