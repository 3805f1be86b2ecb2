// CPU oracle (test infrastructure only): FP64 residual with Neumann load
// (mf_elasticity.h:2708-2922) and the independent matrix-based single-cell
// tangent used by tests/mf_neo_hook_operator*.cc.
#include <cmath>
#include <cstring>

#include "oracle.h"
#include "oracle_cell.h"

namespace orc {

// material.h:119-163 get_tau.  b_bar only used by formulation 0.
static void get_tau(const Material &mat, double det_F, const double bbar[3][3],
                    const double b[3][3], double tau[3][3]) {
  if (mat.formulation == 0) {
    const double dPsi = (mat.kappa / 2.0) * (det_F - 1.0 / det_F);
    const double tmp = dPsi * det_F;
    double tau_bar[3][3], tr = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) tau_bar[i][j] = bbar[i][j] * (2.0 * mat.c1);
    for (int d = 0; d < 3; ++d) tr += tau_bar[d][d];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) tau[i][j] = tau_bar[i][j] + (i == j ? tmp - tr / 3.0 : 0.0);
  } else {
    const double tmp = mat.mu - 2.0 * mat.lambda * std::log(det_F);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) tau[i][j] = mat.mu * b[i][j] - (i == j ? tmp : 0.0);
  }
}

// material.h:171-250 act_Jc on a symmetric tensor src.
static void act_Jc(const Material &mat, double det_F, const double bbar[3][3],
                   const double src[3][3], double res[3][3]) {
  double tr = src[0][0] + src[1][1] + src[2][2];
  if (mat.formulation == 0) {
    const double dPsi = (mat.kappa / 2.0) * (det_F - 1.0 / det_F);
    const double d2Psi = (mat.kappa / 2.0) * (1.0 + 1.0 / (det_F * det_F));
    double dev[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) dev[i][j] = src[i][j] - (i == j ? tr / 3.0 : 0.0);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) res[i][j] = src[i][j] * (-det_F * (2.0 * dPsi));
    const double tmp = det_F * (dPsi + det_F * d2Psi) * tr;
    for (int i = 0; i < 3; ++i) res[i][i] += tmp;
    const double tr_tau_bar = (bbar[0][0] + bbar[1][1] + bbar[2][2]) * 2.0 * mat.c1;
    double tau_iso[3][3];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) tau_iso[i][j] = bbar[i][j] * (2.0 * mat.c1) - (i == j ? tr_tau_bar / 3.0 : 0.0);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) res[i][j] += ((2.0 / 3.0) * tr_tau_bar) * dev[i][j];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) res[i][j] -= ((2.0 / 3.0) * tr) * tau_iso[i][j];
    double tis = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) tis += tau_iso[i][j] * src[i][j];
    for (int i = 0; i < 3; ++i) res[i][i] -= (2.0 / 3.0) * tis;
  } else {
    const double f = 2.0 * (mat.mu - 2.0 * mat.lambda * std::log(det_F));
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) res[i][j] = f * src[i][j];
    for (int i = 0; i < 3; ++i) res[i][i] += 2.0 * mat.lambda * tr;
  }
}

// Kinematics at a quadrature point: F, det F, F^{-1}, b and b_bar.
struct Kin {
  double F[3][3], Fi[3][3], b[3][3], bbar[3][3], det;
};
static void kinematics(const double gradu[3][3], Kin &k) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) k.F[i][j] = gradu[i][j] + (i == j ? 1.0 : 0.0);
  k.det = inv3(k.F, k.Fi);
  const double s = std::pow(k.det, -1.0 / 3.0);  // F_iso = J^{-1/3} F
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double b = 0;
      for (int l = 0; l < 3; ++l) b += k.F[i][l] * k.F[j][l];
      k.b[i][j] = b;
      k.bbar[i][j] = b * s * s;
    }
}

template <int P, int Q>
static double residual_impl(const Mesh &m, const Basis1D &bas, const std::vector<double> &mu,
                            double nu, int formulation, const double *u,
                            const std::vector<Neumann> &neu, double time,
                            const std::vector<uint8_t> &cmask, double *R) {
  using CO = CellOps<P, Q, double>;
  constexpr int NN = CO::NN, NQ = CO::NQ, N1 = CO::N1;
  typename CO::Tables t; CO::tables(bas, t);
  std::memset(R, 0, sizeof(double) * m.n_dofs());
  std::vector<std::vector<int>> col; CO::colours(m, col);
  for (int kk = 0; kk < 8; ++kk) {
    const std::vector<int> &cells = col[kk];
    const long n = (long)cells.size();
#pragma omp parallel for schedule(static)
    for (long ii = 0; ii < n; ++ii) {
      const int cell = cells[ii];
      const int *nodes = &m.cell_nodes[(size_t)cell * NN];
      double xl[3 * NN], ul[3 * NN];
      for (int a = 0; a < NN; ++a)
        for (int c = 0; c < 3; ++c) {
          xl[c * NN + a] = m.X[3 * (size_t)nodes[a] + c];
          ul[c * NN + a] = u[3 * (size_t)nodes[a] + c];
        }
      double GX[3][3][NQ], GU[3][3][NQ], H[3][3][NQ];
      CO::grad(t, xl, GX);
      CO::grad(t, ul, GU);
      const Material mat(mu[cell], nu, formulation);
      for (int q = 0; q < NQ; ++q) {
        double Jr[3][3], Jri[3][3], gu[3][3];
        for (int d = 0; d < 3; ++d)
          for (int e = 0; e < 3; ++e) Jr[d][e] = GX[d][e][q];
        const double jxw = inv3(Jr, Jri) * t.w[q];
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) {
            double a = 0;
            for (int e = 0; e < 3; ++e) a += GU[c][e][q] * Jri[e][d];
            gu[c][d] = a;
          }
        Kin k; kinematics(gu, k);
        double tau[3][3]; get_tau(mat, k.det, k.bbar, k.b, tau);
        // grad_x N = Grad_xi N . Jri . F^{-1};  R -= tau : grad_x N JxW
        double JF[3][3];
        for (int f = 0; f < 3; ++f)
          for (int d = 0; d < 3; ++d) {
            double a = 0;
            for (int e = 0; e < 3; ++e) a += Jri[f][e] * k.Fi[e][d];
            JF[f][d] = a;
          }
        for (int c = 0; c < 3; ++c)
          for (int f = 0; f < 3; ++f) {
            double a = 0;
            for (int d = 0; d < 3; ++d) a += tau[c][d] * JF[f][d];
            H[c][f][q] = -a * jxw;
          }
      }
      double out[3 * NN];
      CO::integrate(t, H, out);
      // Neumann faces of this cell (mf_elasticity.h:2859-2892)
      for (size_t f3 = 0; f3 < m.bfaces.size(); f3 += 3) {
        if (m.bfaces[f3] != cell) continue;
        const int face = m.bfaces[f3 + 1], id = m.bfaces[f3 + 2];
        for (const auto &nm : neu) {
          if (nm.id != id) continue;
          const int nd = face / 2;            // normal direction
          const double xi_n = (face & 1) ? 1.0 : 0.0;
          double vn[N1], dn[N1];
          bas.eval(xi_n, vn, dn);
          const int ta = (nd == 0) ? 1 : 0, tb = (nd == 2) ? 1 : 2;  // tangential dirs
          for (int qb = 0; qb < Q; ++qb)
            for (int qa = 0; qa < Q; ++qa) {
              double xi[3];
              xi[nd] = xi_n; xi[ta] = bas.qpts[qa]; xi[tb] = bas.qpts[qb];
              double v[3][N1], dv[3][N1];
              for (int d = 0; d < 3; ++d) bas.eval(xi[d], v[d], dv[d]);
              double tA[3] = {0, 0, 0}, tB[3] = {0, 0, 0};
              double Nv[NN];
              for (int kz = 0; kz < N1; ++kz)
                for (int jy = 0; jy < N1; ++jy)
                  for (int ix = 0; ix < N1; ++ix) {
                    const int a = (kz * N1 + jy) * N1 + ix;
                    const int li[3] = {ix, jy, kz};
                    Nv[a] = v[0][ix] * v[1][jy] * v[2][kz];
                    double ga = 1, gb = 1;
                    for (int d = 0; d < 3; ++d) {
                      ga *= (d == ta) ? dv[d][li[d]] : v[d][li[d]];
                      gb *= (d == tb) ? dv[d][li[d]] : v[d][li[d]];
                    }
                    for (int c = 0; c < 3; ++c) {
                      tA[c] += xl[c * NN + a] * ga;
                      tB[c] += xl[c * NN + a] * gb;
                    }
                  }
              const double cr[3] = {tA[1] * tB[2] - tA[2] * tB[1], tA[2] * tB[0] - tA[0] * tB[2],
                                    tA[0] * tB[1] - tA[1] * tB[0]};
              const double jxw = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) *
                                 bas.qw[qa] * bas.qw[qb];
              for (int a = 0; a < NN; ++a)
                for (int c = 0; c < 3; ++c)
                  out[c * NN + a] += Nv[a] * (nm.a[c] + nm.b[c] * time) * jxw;
            }
        }
      }
      for (int a = 0; a < NN; ++a)
        for (int c = 0; c < 3; ++c) R[3 * (size_t)nodes[a] + c] += out[c * NN + a];
    }
  }
  // constraints.set_zero(system_rhs), ||R|| (mf_elasticity.h:2917-2921)
  double nrm = 0;
  for (size_t i = 0; i < (size_t)m.n_dofs(); ++i) {
    if (cmask[i]) R[i] = 0.0;
    nrm += R[i] * R[i];
  }
  return std::sqrt(nrm);
}

// d tau / d mu at a fixed deformation: get_tau (material.h:119-163)
// differentiated in the shear modulus, with lambda = 2 mu nu / (1 - 2 nu) and
// kappa = 2 mu (1 + nu) / (3 (1 - 2 nu)) (material.h:82-94) moving with it.
//   formulation 1: tau = mu b - (mu - 2 lambda ln J) I
//                  dtau/dmu = b - (1 - 2 lambda' ln J) I,  lambda' = 2 nu / (1 - 2 nu)
//   formulation 0: tau = (J dPsi_vol/dJ - tr(tau_bar) / 3) I + tau_bar,
//                  tau_bar = 2 c_1 b_bar = mu b_bar, dPsi_vol/dJ = kappa/2 (J - 1/J)
//                  dtau/dmu = (J kappa'/2 (J - 1/J) - tr(b_bar) / 3) I + b_bar
static void dtau_dmu(const Material &mat, double det_F, const double bbar[3][3], const double b[3][3],
                     double out[3][3]) {
  const double nu = mat.nu;
  if (mat.formulation == 0) {
    const double dkappa = 2.0 * (1.0 + nu) / (3.0 * (1.0 - 2.0 * nu));
    const double vol = det_F * (dkappa / 2.0) * (det_F - 1.0 / det_F);
    const double tr = bbar[0][0] + bbar[1][1] + bbar[2][2];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out[i][j] = bbar[i][j] + (i == j ? vol - tr / 3.0 : 0.0);
  } else {
    const double dlambda = 2.0 * nu / (1.0 - 2.0 * nu);
    const double d = 1.0 - 2.0 * dlambda * std::log(det_F);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out[i][j] = b[i][j] - (i == j ? d : 0.0);
  }
}

// g[c] = mu_c * lambda . dR_c/dmu_c for every cell c, where R_c is the cell's
// internal-force part of the residual (mf_elasticity.h:2736-2804),
// dR_c/dmu = -int dtau/dmu : grad_x N dV: the derivative of the residual with
// respect to log mu_c, contracted with the adjoint vector.
template <int P, int Q>
static void dresidual_dlogmu_impl(const Mesh &m, const Basis1D &bas, const std::vector<double> &mu, double nu,
                                  int formulation, const double *u, const double *lam, double *g) {
  using CO = CellOps<P, Q, double>;
  constexpr int NN = CO::NN, NQ = CO::NQ;
  typename CO::Tables t; CO::tables(bas, t);
#pragma omp parallel for schedule(static)
  for (int cell = 0; cell < m.n_cells; ++cell) {
    const int *nodes = &m.cell_nodes[(size_t)cell * NN];
    double xl[3 * NN], ul[3 * NN];
    for (int a = 0; a < NN; ++a)
      for (int c = 0; c < 3; ++c) {
        xl[c * NN + a] = m.X[3 * (size_t)nodes[a] + c];
        ul[c * NN + a] = u[3 * (size_t)nodes[a] + c];
      }
    double GX[3][3][NQ], GU[3][3][NQ], H[3][3][NQ];
    CO::grad(t, xl, GX);
    CO::grad(t, ul, GU);
    const Material mat(mu[cell], nu, formulation);
    for (int q = 0; q < NQ; ++q) {
      double Jr[3][3], Jri[3][3], gu[3][3];
      for (int d = 0; d < 3; ++d)
        for (int e = 0; e < 3; ++e) Jr[d][e] = GX[d][e][q];
      const double jxw = inv3(Jr, Jri) * t.w[q];
      for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d) {
          double a = 0;
          for (int e = 0; e < 3; ++e) a += GU[c][e][q] * Jri[e][d];
          gu[c][d] = a;
        }
      Kin k; kinematics(gu, k);
      double dt[3][3]; dtau_dmu(mat, k.det, k.bbar, k.b, dt);
      for (int c = 0; c < 3; ++c)
        for (int f = 0; f < 3; ++f) {
          double a = 0;
          for (int d = 0; d < 3; ++d) {
            double jf = 0;
            for (int e = 0; e < 3; ++e) jf += Jri[f][e] * k.Fi[e][d];
            a += dt[c][d] * jf;
          }
          H[c][f][q] = -a * jxw;
        }
    }
    double out[3 * NN];
    CO::integrate(t, H, out);
    double s = 0;
    for (int a = 0; a < NN; ++a)
      for (int c = 0; c < 3; ++c) s += lam[3 * (size_t)nodes[a] + c] * out[c * NN + a];
    g[cell] = mu[cell] * s;
  }
}

void dresidual_dlogmu_dot(const Mesh &m, const Basis1D &b, const std::vector<double> &mu, double nu,
                          int formulation, const double *u, const double *lam, double *g) {
  DISPATCH_PQ(m.p, b.q, { dresidual_dlogmu_impl<P_, Q_>(m, b, mu, nu, formulation, u, lam, g); });
}

double residual(const Mesh &m, const Basis1D &b, const std::vector<double> &mu, double nu,
                int formulation, const double *u, const std::vector<Neumann> &neu,
                double time, const std::vector<uint8_t> &cmask, double *R) {
  double r = 0;
  DISPATCH_PQ(m.p, b.q, { r = residual_impl<P_, Q_>(m, b, mu, nu, formulation, u, neu, time, cmask, R); });
  return r;
}

template <int P, int Q>
static void element_matrix_impl(const Mesh &m, const Basis1D &bas, int cell, const Material &mat,
                                const double *u, std::vector<double> &K) {
  using CO = CellOps<P, Q, double>;
  constexpr int NN = CO::NN, NQ = CO::NQ, N1 = CO::N1;
  constexpr int ND = 3 * NN;
  typename CO::Tables t; CO::tables(bas, t);
  K.assign((size_t)ND * ND, 0.0);
  const int *nodes = &m.cell_nodes[(size_t)cell * NN];
  double xl[3 * NN], ul[3 * NN];
  for (int a = 0; a < NN; ++a)
    for (int c = 0; c < 3; ++c) {
      xl[c * NN + a] = m.X[3 * (size_t)nodes[a] + c];
      ul[c * NN + a] = u[3 * (size_t)nodes[a] + c];
    }
  double GX[3][3][NQ], GU[3][3][NQ];
  CO::grad(t, xl, GX);
  CO::grad(t, ul, GU);
  for (int qz = 0; qz < Q; ++qz)
    for (int qy = 0; qy < Q; ++qy)
      for (int qx = 0; qx < Q; ++qx) {
        const int q = (qz * Q + qy) * Q + qx;
        double Jr[3][3], Jri[3][3], gu[3][3];
        for (int d = 0; d < 3; ++d)
          for (int e = 0; e < 3; ++e) Jr[d][e] = GX[d][e][q];
        const double JxW = inv3(Jr, Jri) * t.w[q];
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) {
            double a = 0;
            for (int e = 0; e < 3; ++e) a += GU[c][e][q] * Jri[e][d];
            gu[c][d] = a;
          }
        Kin k; kinematics(gu, k);
        double tau[3][3]; get_tau(mat, k.det, k.bbar, k.b, tau);
        // grad_Nx[i] = fe_values.gradient(i, q) * F_inv, as 3 components of
        // the row of component c_i
        std::vector<double> gN(NN * 3);
        for (int kz = 0; kz < N1; ++kz)
          for (int jy = 0; jy < N1; ++jy)
            for (int ix = 0; ix < N1; ++ix) {
              const int a = (kz * N1 + jy) * N1 + ix;
              const double gxi[3] = {t.D[qx][ix] * t.N[qy][jy] * t.N[qz][kz],
                                     t.N[qx][ix] * t.D[qy][jy] * t.N[qz][kz],
                                     t.N[qx][ix] * t.N[qy][jy] * t.D[qz][kz]};
              double gX[3];
              for (int e = 0; e < 3; ++e) {
                double s = 0;
                for (int f = 0; f < 3; ++f) s += gxi[f] * Jri[f][e];
                gX[e] = s;
              }
              for (int d = 0; d < 3; ++d) {
                double s = 0;
                for (int e = 0; e < 3; ++e) s += gX[e] * k.Fi[e][d];
                gN[a * 3 + d] = s;
              }
            }
        for (int j = 0; j < ND; ++j) {
          const int cj = j / NN, aj = j % NN;
          double Gj[3][3] = {}, Sj[3][3];
          for (int d = 0; d < 3; ++d) Gj[cj][d] = gN[aj * 3 + d];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) Sj[a][b] = 0.5 * (Gj[a][b] + Gj[b][a]);
          double JcS[3][3]; act_Jc(mat, k.det, k.bbar, Sj, JcS);
          double geo[3][3];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
              double s = 0;
              for (int l = 0; l < 3; ++l) s += Gj[a][l] * tau[l][b];
              geo[a][b] = s;
            }
          for (int i = 0; i < ND; ++i) {
            const int ci = i / NN, ai = i % NN;
            double v = 0;
            for (int d = 0; d < 3; ++d) {
              const double gi = gN[ai * 3 + d];
              const double si_cd = 0.5 * gi;  // sym(e_ci (x) g)_{ci,d} part
              // sym(Gi) : JcS = sum_ab Si_ab JcS_ab with Si = sym(e_ci (x) gi)
              v += si_cd * (JcS[ci][d] + JcS[d][ci]);
              v += gi * geo[ci][d];
            }
            K[(size_t)i * ND + j] += v * JxW;
          }
        }
      }
}

void element_matrix(const Mesh &m, const Basis1D &b, int cell, const Material &mat,
                    const double *u, std::vector<double> &K) {
  DISPATCH_PQ(m.p, b.q, { element_matrix_impl<P_, Q_>(m, b, cell, mat, u, K); });
}

}  // namespace orc
