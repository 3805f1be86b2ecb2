// CPU oracle (test infrastructure only): CG, Chebyshev smoother with CG-
// Lanczos eigenvalue estimate, matrix-free level transfer, V-cycle and the
// load-stepping Newton driver of mf_elasticity.h.
#include "solver.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "oracle_cell.h"

namespace orc {

// ------------------------------------------------------------- helpers
template <typename T>
static double dot(const std::vector<T> &a, const std::vector<T> &b) {
  double s = 0;
  const long n = (long)a.size();
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long i = 0; i < n; ++i) s += (double)a[i] * (double)b[i];
  return s;
}
template <typename T>
static double norm2(const std::vector<T> &a) { return std::sqrt(dot(a, a)); }

// Eigenvalues of a symmetric tridiagonal matrix by bisection on Sturm
// sequences (used for the CG-Lanczos estimate; SolverCG::compute_eigs_and_cond).
static double tridiag_eig(const std::vector<double> &d, const std::vector<double> &e, bool want_max) {
  const int n = (int)d.size();
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < n; ++i) {
    double r = (i > 0 ? std::fabs(e[i - 1]) : 0) + (i < n - 1 ? std::fabs(e[i]) : 0);
    lo = std::min(lo, d[i] - r); hi = std::max(hi, d[i] + r);
  }
  auto count_below = [&](double x) {
    int cnt = 0; double q = 1.0;
    for (int i = 0; i < n; ++i) {
      double ee = (i > 0) ? e[i - 1] * e[i - 1] : 0.0;
      q = d[i] - x - (i > 0 ? ee / q : 0.0);
      if (q == 0.0) q = -1e-300;
      if (q < 0) ++cnt;
    }
    return cnt;
  };
  const int k = want_max ? n - 1 : 0;  // index of wanted eigenvalue
  double a = lo, b = hi;
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (a + b);
    if (count_below(mid) > k) b = mid; else a = mid;
    if (b - a <= 1e-15 * std::max(std::fabs(a), std::fabs(b))) break;
  }
  return 0.5 * (a + b);
}

// ------------------------------------------------------------------ CG
// deal.II SolverCG as used by mf_elasticity.h:3175-3180 / Chebyshev's
// eigenvalue estimate: g = Ax - b, d = -P g, convergence on ||g||_2.
template <typename T, typename Amul, typename Prec>
static int cg_solve(Amul A, Prec Pm, std::vector<T> &x, const std::vector<T> &b,
                    int max_it, double abs_tol, double rel_red, bool *converged,
                    std::vector<double> *diag_T, std::vector<double> *off_T, double *final_res) {
  const size_t n = b.size();
  std::vector<T> g(n), h(n), d(n);
  A(g, x);
  for (size_t i = 0; i < n; ++i) g[i] -= b[i];
  double res = norm2(g), res0 = res;
  double tol = std::max(abs_tol, rel_red * res0);
  int it = 0;
  if (converged) *converged = false;
  if (res <= tol) { if (converged) *converged = true; if (final_res) *final_res = res; return 0; }
  Pm(h, g);
  for (size_t i = 0; i < n; ++i) d[i] = -h[i];
  double gh = dot(g, h), beta = 0, old_alpha = 0;
  while (true) {
    ++it;
    A(h, d);
    double alpha = dot(d, h);
    alpha = gh / alpha;
    for (size_t i = 0; i < n; ++i) { x[i] += T(alpha) * d[i]; g[i] += T(alpha) * h[i]; }
    res = norm2(g);
    if (diag_T) {
      if (it > 1) { diag_T->push_back(1.0 / alpha + beta / old_alpha); off_T->push_back(std::sqrt(beta) / old_alpha); }
      else diag_T->push_back(1.0 / alpha);
    }
    if (res <= tol) { if (converged) *converged = true; break; }
    if (it >= max_it) break;
    Pm(h, g);
    beta = gh;
    gh = dot(g, h);
    beta = gh / beta;
    for (size_t i = 0; i < n; ++i) d[i] = T(beta) * d[i] - h[i];
    old_alpha = alpha;
  }
  if (final_res) *final_res = res;
  return it;
}

// -------------------------------------------------------------- transfer
void Transfer::build(const Mesh &coarse, const Mesh &fine, const Basis1D &b) {
  const int p = coarse.p, n1 = p + 1, nf1 = 2 * p + 1;
  P1.assign(nf1 * n1, 0.0);
  for (int f = 0; f < nf1; ++f) {
    int child = f / p, loc = f - child * p;
    if (child > 1) { child = 1; loc = p; }
    double xi = 0.5 * (child + (loc == p ? 1.0 : b.nodes[loc]));
    b.eval(xi, &P1[f * n1], nullptr);
  }
  n_coarse_cells = coarse.n_cells;
  nfb = nf1 * nf1 * nf1;
  fine_nodes.resize((size_t)coarse.n_cells * nfb);
  std::vector<int> mult(fine.n_nodes, 0);
  for (int c = 0; c < coarse.n_cells; ++c) {
    const int i = coarse.cell_ijk[3 * c], j = coarse.cell_ijk[3 * c + 1], k = coarse.cell_ijk[3 * c + 2];
    int idx = 0;
    for (int fz = 0; fz < nf1; ++fz)
      for (int fy = 0; fy < nf1; ++fy)
        for (int fx = 0; fx < nf1; ++fx) {
          size_t L = ((size_t)(2 * k * p + fz) * fine.nn[1] + (2 * j * p + fy)) * fine.nn[0] + (2 * i * p + fx);
          int node = fine.lattice_to_node[L];
          fine_nodes[(size_t)c * nfb + idx++] = node;
          mult[node]++;
        }
  }
  weight.resize(fine.n_nodes);
  for (int n = 0; n < fine.n_nodes; ++n) weight[n] = mult[n] ? 1.0 / mult[n] : 0.0;
}

// prolongation (MGTransferMatrixFree::prolongate): coarse Dirichlet entries
// are zeroed before the cell-wise interpolation, fine values weighted by the
// inverse multiplicity so that shared nodes receive exactly one value.
template <typename T>
void Transfer::prolongate_add(const Mesh &coarse, const std::vector<uint8_t> &ccmask,
                              const T *src, T *dst) const {
  const int p = coarse.p, n1 = p + 1, nf1 = 2 * p + 1, ncn = coarse.ncn();
  for (int c = 0; c < coarse.n_cells; ++c) {
    const int *cn = &coarse.cell_nodes[(size_t)c * ncn];
    for (int comp = 0; comp < 3; ++comp) {
      std::vector<double> v(ncn), a(nf1 * n1 * n1), bb(nf1 * nf1 * n1), out(nfb);
      for (int l = 0; l < ncn; ++l) {
        size_t dof = 3 * (size_t)cn[l] + comp;
        v[l] = ccmask[dof] ? 0.0 : (double)src[dof];
      }
      for (int z = 0; z < n1; ++z)
        for (int y = 0; y < n1; ++y)
          for (int fx = 0; fx < nf1; ++fx) {
            double s = 0;
            for (int x = 0; x < n1; ++x) s += P1[fx * n1 + x] * v[(z * n1 + y) * n1 + x];
            a[(z * n1 + y) * nf1 + fx] = s;
          }
      for (int z = 0; z < n1; ++z)
        for (int fy = 0; fy < nf1; ++fy)
          for (int fx = 0; fx < nf1; ++fx) {
            double s = 0;
            for (int y = 0; y < n1; ++y) s += P1[fy * n1 + y] * a[(z * n1 + y) * nf1 + fx];
            bb[(z * nf1 + fy) * nf1 + fx] = s;
          }
      for (int fz = 0; fz < nf1; ++fz)
        for (int fy = 0; fy < nf1; ++fy)
          for (int fx = 0; fx < nf1; ++fx) {
            double s = 0;
            for (int z = 0; z < n1; ++z) s += P1[fz * n1 + z] * bb[(z * nf1 + fy) * nf1 + fx];
            out[(fz * nf1 + fy) * nf1 + fx] = s;
          }
      for (int l = 0; l < nfb; ++l) {
        const int node = fine_nodes[(size_t)c * nfb + l];
        dst[3 * (size_t)node + comp] += T(weight[node] * out[l]);
      }
    }
  }
}

// restriction = transpose of prolongation, coarse Dirichlet entries zeroed
// (MGTransferMatrixFree::restrict_and_add).
template <typename T>
void Transfer::restrict_add(const Mesh &coarse, const std::vector<uint8_t> &ccmask,
                            const T *src, T *dst) const {
  const int p = coarse.p, n1 = p + 1, nf1 = 2 * p + 1, ncn = coarse.ncn();
  for (int c = 0; c < coarse.n_cells; ++c) {
    const int *cn = &coarse.cell_nodes[(size_t)c * ncn];
    for (int comp = 0; comp < 3; ++comp) {
      std::vector<double> in(nfb), bb(nf1 * nf1 * n1), a(nf1 * n1 * n1), v(ncn);
      for (int l = 0; l < nfb; ++l) {
        const int node = fine_nodes[(size_t)c * nfb + l];
        in[l] = weight[node] * (double)src[3 * (size_t)node + comp];
      }
      for (int z = 0; z < n1; ++z)
        for (int fy = 0; fy < nf1; ++fy)
          for (int fx = 0; fx < nf1; ++fx) {
            double s = 0;
            for (int fz = 0; fz < nf1; ++fz) s += P1[fz * n1 + z] * in[(fz * nf1 + fy) * nf1 + fx];
            bb[(z * nf1 + fy) * nf1 + fx] = s;
          }
      for (int z = 0; z < n1; ++z)
        for (int y = 0; y < n1; ++y)
          for (int fx = 0; fx < nf1; ++fx) {
            double s = 0;
            for (int fy = 0; fy < nf1; ++fy) s += P1[fy * n1 + y] * bb[(z * nf1 + fy) * nf1 + fx];
            a[(z * n1 + y) * nf1 + fx] = s;
          }
      for (int z = 0; z < n1; ++z)
        for (int y = 0; y < n1; ++y)
          for (int x = 0; x < n1; ++x) {
            double s = 0;
            for (int fx = 0; fx < nf1; ++fx) s += P1[fx * n1 + x] * a[(z * n1 + y) * nf1 + fx];
            v[(z * n1 + y) * n1 + x] = s;
          }
      for (int l = 0; l < ncn; ++l) {
        size_t dof = 3 * (size_t)cn[l] + comp;
        if (!ccmask[dof]) dst[dof] += T(v[l]);
      }
    }
  }
}

// nodal injection of the fine displacement onto the coarse nodes: for
// nested Lagrange spaces interpolate_to_mg (mf_elasticity.h:1929-1942)
// evaluates the fine function at the coarse support points.
template <typename T>
void Transfer::interpolate(const Mesh &coarse, const Mesh &fine, const T *fine_u, T *coarse_u) const {
  // coarse node with lattice index I sits at fine lattice index 2I only for
  // the element vertices; interior GL nodes are evaluated through the fine
  // cell containing them.
  const int p = coarse.p, n1 = p + 1;
  Basis1D b; b.init(p, p + 1);
  const int ncn = coarse.ncn();
  for (int c = 0; c < coarse.n_cells; ++c) {
    const int i = coarse.cell_ijk[3 * c], j = coarse.cell_ijk[3 * c + 1], k = coarse.cell_ijk[3 * c + 2];
    for (int lz = 0; lz < n1; ++lz)
      for (int ly = 0; ly < n1; ++ly)
        for (int lx = 0; lx < n1; ++lx) {
          const int cnode = coarse.cell_nodes[(size_t)c * ncn + (lz * n1 + ly) * n1 + lx];
          // position inside coarse cell in [0,1], mapped to fine child
          int li[3] = {lx, ly, lz}, ci[3] = {i, j, k}, child[3];
          double xf[3];
          for (int d = 0; d < 3; ++d) {
            double xi = b.nodes[li[d]];
            double s = 2.0 * xi;
            child[d] = std::min(1, (int)std::floor(s));
            xf[d] = s - child[d];
          }
          int fi = 2 * ci[0] + child[0], fj = 2 * ci[1] + child[1], fk = 2 * ci[2] + child[2];
          int fcell = fine.cell_of_lattice[((size_t)fk * fine.nc[1] + fj) * fine.nc[0] + fi];
          double vx[5], vy[5], vz[5];
          b.eval(xf[0], vx, nullptr); b.eval(xf[1], vy, nullptr); b.eval(xf[2], vz, nullptr);
          for (int comp = 0; comp < 3; ++comp) {
            double s = 0;
            for (int z = 0; z < n1; ++z)
              for (int y = 0; y < n1; ++y)
                for (int x = 0; x < n1; ++x) {
                  const int fn = fine.cell_nodes[(size_t)fcell * ncn + (z * n1 + y) * n1 + x];
                  s += vx[x] * vy[y] * vz[z] * (double)fine_u[3 * (size_t)fn + comp];
                }
            coarse_u[3 * (size_t)cnode + comp] = T(s);
          }
        }
  }
}

template void Transfer::prolongate_add<float>(const Mesh &, const std::vector<uint8_t> &, const float *, float *) const;
template void Transfer::prolongate_add<double>(const Mesh &, const std::vector<uint8_t> &, const double *, double *) const;
template void Transfer::restrict_add<float>(const Mesh &, const std::vector<uint8_t> &, const float *, float *) const;
template void Transfer::restrict_add<double>(const Mesh &, const std::vector<uint8_t> &, const double *, double *) const;
template void Transfer::interpolate<float>(const Mesh &, const Mesh &, const float *, float *) const;
template void Transfer::interpolate<double>(const Mesh &, const Mesh &, const double *, double *) const;

// ------------------------------------------------------------ Chebyshev
// deal.II PreconditionChebyshev (configured in mf_elasticity.h:2079-2113):
// eigenvalue estimate by CG with the inverse diagonal from a period-11
// start vector, lambda_max * 1.2, smoothing range or (coarse "solver"
// mode) a degree chosen for the requested reduction.
template <typename T>
void Chebyshev<T>::setup(const Operator<T> &A, const std::vector<T> &inv_diag_, int degree_,
                         double range_, int eig_its) {
  op = &A; inv_diag = inv_diag_;
  const size_t n = inv_diag.size();
  std::vector<T> x(n, T(0)), rhs(n);
  for (size_t i = 0; i < n; ++i) rhs[i] = T(i % 11);
  double mean = 0; for (size_t i = 0; i < n; ++i) mean += (double)rhs[i];
  mean /= (double)n;
  for (size_t i = 0; i < n; ++i) rhs[i] = T((double)rhs[i] - mean);
  std::vector<double> dT, oT;
  bool conv;
  auto Am = [&](std::vector<T> &dst, const std::vector<T> &src) { A.vmult(dst.data(), src.data()); };
  auto Pm = [&](std::vector<T> &dst, const std::vector<T> &src) {
    for (size_t i = 0; i < n; ++i) dst[i] = inv_diag[i] * src[i];
  };
  const double abs_tol = std::sqrt((double)std::numeric_limits<T>::epsilon());
  cg_solve(Am, Pm, x, rhs, eig_its, abs_tol, 1e-10, &conv, &dT, &oT, nullptr);
  double mn = 1, mx = 1;
  if (!dT.empty()) {
    mn = tridiag_eig(dT, oT, false);
    mx = tridiag_eig(dT, oT, true);
  }
  eig_min = mn; eig_max = mx;
  const double max_eigenvalue = 1.2 * mx;
  const double alpha = (range_ > 1.0) ? max_eigenvalue / range_ : std::min(0.9 * max_eigenvalue, mn);
  degree = degree_;
  if (degree_ <= 0) {
    const double actual_range = max_eigenvalue / alpha;
    const double sigma = (1. - std::sqrt(1. / actual_range)) / (1. + std::sqrt(1. / actual_range));
    const double eps = range_;
    degree = 1 + (int)(std::log(1. / eps + std::sqrt(1. / eps / eps - 1.)) / std::log(1. / sigma));
  }
  theta = 0.5 * (max_eigenvalue + alpha);
  delta = 0.5 * (max_eigenvalue - alpha);
}

// Chebyshev iteration x_{k+1} = x_k + rho_k rho_{k-1} (x_k - x_{k-1})
//   + 2 rho_k / delta * D^{-1} (b - A x_k); zero_start = vmult(), else step().
template <typename T>
void Chebyshev<T>::run(std::vector<T> &x, const std::vector<T> &b, bool zero_start) const {
  const size_t n = b.size();
  std::vector<T> r(n), xold(n), tmp(n);
  // vmult(): x_1 = D^-1 b / theta; step(): x_1 = x_0 + D^-1 (b - A x_0) / theta;
  // then degree - 1 recurrence steps, each with one matrix-vector product
  const int mv = degree - 1;
  if (zero_start) {
    for (size_t i = 0; i < n; ++i) { x[i] = T(inv_diag[i] * b[i] / theta); xold[i] = T(0); }
  } else {
    op->vmult(r.data(), x.data());
    for (size_t i = 0; i < n; ++i) {
      xold[i] = x[i];
      x[i] = T((double)x[i] + (double)inv_diag[i] * ((double)b[i] - (double)r[i]) / theta);
    }
  }
  if (degree < 2 || std::fabs(delta) < 1e-40) return;
  double rhok = delta / theta;
  const double sigma = theta / delta;
  for (int k = 0; k < mv; ++k) {
    op->vmult(r.data(), x.data());
    const double rhokp = 1. / (2. * sigma - rhok);
    const double f1 = rhokp * rhok, f2 = 2. * rhokp / delta;
    rhok = rhokp;
    for (size_t i = 0; i < n; ++i) {
      const double xn = (double)x[i] + f1 * ((double)x[i] - (double)xold[i]) +
                        f2 * (double)inv_diag[i] * ((double)b[i] - (double)r[i]);
      xold[i] = x[i];
      x[i] = T(xn);
    }
  }
}

template struct Chebyshev<float>;
template struct Chebyshev<double>;

// ------------------------------------------------------------------ GMG
template <typename T>
void GMG<T>::vcycle(int l, std::vector<T> &x, const std::vector<T> &b) const {
  const Level &L = levels[l];
  if (l == 0 && coarse_cg) {
    const size_t n = b.size();
    std::fill(x.begin(), x.end(), T(0));
    auto Am = [&](std::vector<T> &dst, const std::vector<T> &src) { L.op.vmult(dst.data(), src.data()); };
    auto Pm = [&](std::vector<T> &dst, const std::vector<T> &src) { L.cheb.run(dst, src, true); };
    const int max_it = std::max((int)n, 100);
    cg_solve(Am, Pm, x, b, max_it, 1e-10, 1e-3, nullptr, nullptr, nullptr, nullptr);
    return;
  }
  if (l == 0) { L.cheb.run(x, b, true); return; }   // MGCoarseGridApplySmoother
  L.cheb.run(x, b, true);                           // pre-smoothing: apply()
  std::vector<T> t(b.size());
  L.op.vmult(t.data(), x.data());
  for (size_t i = 0; i < b.size(); ++i) t[i] = b[i] - t[i];
  const Level &C = levels[l - 1];
  std::vector<T> bc(C.mesh.n_dofs(), T(0)), xc(C.mesh.n_dofs(), T(0));
  L.transfer.restrict_add(C.mesh, C.cmask, t.data(), bc.data());
  vcycle(l - 1, xc, bc);
  std::vector<T> corr(b.size(), T(0));
  L.transfer.prolongate_add(C.mesh, C.cmask, xc.data(), corr.data());
  for (size_t i = 0; i < b.size(); ++i) x[i] += corr[i];
  L.cheb.run(x, b, false);                          // post-smoothing: smooth()
}

template <typename T>
void GMG<T>::vmult(std::vector<double> &dst, const std::vector<double> &src) const {
  const int top = (int)levels.size() - 1;
  std::vector<T> b(src.size()), x(src.size(), T(0));
  for (size_t i = 0; i < src.size(); ++i) b[i] = T(src[i]);  // copy_to_mg
  vcycle(top, x, b);
  for (size_t i = 0; i < src.size(); ++i) dst[i] = (double)x[i];  // copy_from_mg
}

template struct GMG<float>;
template struct GMG<double>;

// --------------------------------------------------------- output point
bool point_value(const Mesh &m, const Basis1D &b, const double *u, const double pt[3], double out[3]) {
  const int p = m.p, n1 = p + 1, ncn = m.ncn();
  const double tol = 1e-10;
  for (int c = 0; c < m.n_cells; ++c) {
    const int *nodes = &m.cell_nodes[(size_t)c * ncn];
    // bounding box test
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int a = 0; a < ncn; ++a)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], m.X[3 * (size_t)nodes[a] + d]);
        hi[d] = std::max(hi[d], m.X[3 * (size_t)nodes[a] + d]);
      }
    bool inside = true;
    for (int d = 0; d < 3; ++d) {
      double h = (hi[d] - lo[d]) * 1e-9 + 1e-300;
      if (pt[d] < lo[d] - h || pt[d] > hi[d] + h) inside = false;
    }
    if (!inside) continue;
    double xi[3] = {0.5, 0.5, 0.5};
    for (int it = 0; it < 50; ++it) {
      double v[3][5], dv[3][5];
      for (int d = 0; d < 3; ++d) b.eval(xi[d], v[d], dv[d]);
      double x[3] = {0, 0, 0}, J[3][3] = {};
      for (int z = 0; z < n1; ++z)
        for (int y = 0; y < n1; ++y)
          for (int xx = 0; xx < n1; ++xx) {
            const double *X = &m.X[3 * (size_t)nodes[(z * n1 + y) * n1 + xx]];
            const double N = v[0][xx] * v[1][y] * v[2][z];
            const double g[3] = {dv[0][xx] * v[1][y] * v[2][z], v[0][xx] * dv[1][y] * v[2][z],
                                 v[0][xx] * v[1][y] * dv[2][z]};
            for (int d = 0; d < 3; ++d) {
              x[d] += N * X[d];
              for (int e = 0; e < 3; ++e) J[d][e] += X[d] * g[e];
            }
          }
      double Ji[3][3]; inv3(J, Ji);
      double dxi[3];
      for (int d = 0; d < 3; ++d) {
        dxi[d] = 0;
        for (int e = 0; e < 3; ++e) dxi[d] += Ji[d][e] * (pt[e] - x[e]);
      }
      for (int d = 0; d < 3; ++d) xi[d] += dxi[d];
      if (std::fabs(dxi[0]) + std::fabs(dxi[1]) + std::fabs(dxi[2]) < 1e-14) break;
    }
    if (xi[0] < -tol || xi[0] > 1 + tol || xi[1] < -tol || xi[1] > 1 + tol || xi[2] < -tol || xi[2] > 1 + tol)
      continue;
    double v[3][5];
    for (int d = 0; d < 3; ++d) b.eval(std::min(1.0, std::max(0.0, xi[d])), v[d], nullptr);
    out[0] = out[1] = out[2] = 0;
    for (int z = 0; z < n1; ++z)
      for (int y = 0; y < n1; ++y)
        for (int xx = 0; xx < n1; ++xx) {
          const int node = nodes[(z * n1 + y) * n1 + xx];
          const double N = v[0][xx] * v[1][y] * v[2][z];
          for (int d = 0; d < 3; ++d) out[d] += N * u[3 * (size_t)node + d];
        }
    return true;
  }
  return false;
}

// Per-cell values on level l from a fine per-cell field: mean over the fine
// cells inside each level cell (the coarse-level material of a per-cell mu).
std::vector<double> coarsen_cell_field(const std::vector<Mesh> &meshes, int l, const std::vector<double> &fine) {
  const Mesh &F = meshes.back(), &L = meshes[l];
  const int sh = (int)meshes.size() - 1 - l;
  std::vector<double> out(L.n_cells, 1.0);
  for (int c = 0; c < L.n_cells; ++c) {
    const int i0 = L.cell_ijk[3 * c] << sh, j0 = L.cell_ijk[3 * c + 1] << sh, k0 = L.cell_ijk[3 * c + 2] << sh;
    double s = 0; int n = 0;
    for (int k = k0; k < k0 + (1 << sh); ++k)
      for (int j = j0; j < j0 + (1 << sh); ++j)
        for (int i = i0; i < i0 + (1 << sh); ++i) {
          const int fc = F.cell_of_lattice[((size_t)k * F.nc[1] + j) * F.nc[0] + i];
          if (fc >= 0) { s += fine[fc]; ++n; }
        }
    if (n) out[c] = s / n;
  }
  return out;
}

// --------------------------------------------------------------- Newton
// Solid::run / solve_nonlinear_timestep / check_convergence /
// solve_linear_system (mf_elasticity.h:1187-1235, 2245-2559, 3012-3214).
template <typename LT>
void setup_gmg(const NewtonParams &prm, const std::vector<Mesh> &meshes, const Basis1D &bas,
                      const std::vector<std::vector<uint8_t>> &lmask,
                      const std::vector<std::vector<double>> &lmu,
                      const std::vector<double> &u_fine, GMG<LT> &gmg, bool first) {
  const int nl = (int)meshes.size();
  if (first) {
    gmg.levels.clear();
    gmg.levels.resize(nl);
    for (int l = 0; l < nl; ++l) {
      auto &L = gmg.levels[l];
      L.mesh = meshes[l];
      L.cmask = lmask[l];
      L.op.initialize(&L.mesh, &bas, prm.caching, prm.formulation);
      L.op.set_material(lmu[l], prm.nu);
      L.op.set_constraints(L.cmask);
      if (l > 0) L.transfer.build(gmg.levels[l - 1].mesh, L.mesh, bas);
    }
  }
  // interpolate_to_mg in level precision
  std::vector<std::vector<LT>> lu(nl);
  lu[nl - 1].resize(u_fine.size());
  for (size_t i = 0; i < u_fine.size(); ++i) lu[nl - 1][i] = LT(u_fine[i]);
  for (int l = nl - 1; l > 0; --l) {
    lu[l - 1].assign(meshes[l - 1].n_dofs(), LT(0));
    gmg.levels[l].transfer.interpolate(gmg.levels[l - 1].mesh, gmg.levels[l].mesh, lu[l].data(), lu[l - 1].data());
  }
  for (int l = 0; l < nl; ++l) {
    auto &L = gmg.levels[l];
    L.op.cache(lu[l].data());
    L.op.compute_diagonal();
    gmg.coarse_cg = !prm.coarse_chebyshev;
    if (l == 0 && prm.coarse_chebyshev)
      L.cheb.setup(L.op, L.op.inv_diag, 0, 1e-3,
                   prm.coarse_accurate_eig ? L.mesh.n_dofs() : prm.cheb_eig_its);
    else
      L.cheb.setup(L.op, L.op.inv_diag, prm.cheb_degree, prm.smoothing_range, prm.cheb_eig_its);
  }
}

int newton_run(const NewtonParams &prm, NewtonResult &res) {
  Basis1D bas; bas.init(prm.mesh.p, prm.mesh.q);
  const int nl = prm.mesh.n_refinements + 1;
  std::vector<Mesh> meshes(nl);
  for (int l = 0; l < nl; ++l) build_mesh(prm.mesh, l, meshes[l]);
  const Mesh &m = meshes[nl - 1];
  res.n_cells = m.n_cells; res.n_dofs = m.n_dofs();
  res.volume = mesh_volume(m, bas);
  // per-cell shear modulus on every level (children inherit the parent's)
  std::vector<double> mu_f = prm.mu_fine;
  if (mu_f.empty()) mu_f.assign(m.n_cells, prm.mu);
  std::vector<std::vector<double>> lmu(nl);
  for (int l = 0; l < nl; ++l) lmu[l] = coarsen_cell_field(meshes, l, mu_f);
  std::vector<std::vector<uint8_t>> lmask(nl);
  for (int l = 0; l < nl; ++l) constrained_dofs(meshes[l], prm.dirichlet, lmask[l]);
  const std::vector<uint8_t> &cmask = lmask[nl - 1];
  // inhomogeneous constraint values (applied as the increment of a load step)
  std::vector<double> gvals(m.n_dofs(), 0.0);
  bool inhom = false;
  {
    std::vector<uint8_t> one;
    for (size_t s = 0; s < prm.dirichlet.size(); ++s) {
      constrained_dofs(m, {prm.dirichlet[s]}, one);
      for (size_t i = 0; i < one.size(); ++i)
        if (one[i]) { gvals[i] = prm.dirichlet_value[s][i % 3]; if (gvals[i] != 0) inhom = true; }
    }
  }
  const size_t n = m.n_dofs();
  std::vector<double> u_n(n, 0.0), du(n, 0.0), u_tot(n), R(n), dx(n);
  Operator<double> op;
  op.initialize(&m, &bas, prm.caching, prm.formulation);
  op.set_material(lmu[nl - 1], prm.nu);
  op.set_constraints(cmask);
  GMG<float> gmg_f; GMG<double> gmg_d;
  double time = 0.0;
  time += prm.dt;
  res.steps.clear();
  while (time <= prm.end_time) {
    std::fill(du.begin(), du.end(), 0.0);
    double err_res = 0, err_res0 = 0, err_upd = 0, err_upd0 = 0, err_upd_norm = 0;
    int it = 0; bool conv = false;
    StepResult sr;
    for (; it < prm.max_nr; ++it) {
      for (size_t i = 0; i < n; ++i) u_tot[i] = u_n[i] + du[i];
      err_res = residual(m, bas, lmu[nl - 1], prm.nu, prm.formulation, u_tot.data(), prm.neumann, time, cmask, R.data());
      if (op.cache(u_tot.data())) return 2;   // det F <= 0
      if (it == 0 && inhom) {
        // rhs -= K g over constrained columns (AffineConstraints with an
        // inhomogeneity, mf_elasticity.h:2910-2915)
        std::vector<double> Kg(n, 0.0), gz(n);
        op.apply_inhomogeneous(Kg.data(), gvals.data());
        double s = 0;
        for (size_t i = 0; i < n; ++i) { if (!cmask[i]) R[i] -= Kg[i]; else R[i] = 0; s += R[i] * R[i]; }
        err_res = std::sqrt(s);
      }
      if (it == 0) err_res0 = err_res;
      const double rel_res = err_res0 != 0 ? err_res / err_res0 : err_res;
      sr.rel_res.push_back(rel_res);
      sr.rel_upd.push_back(err_upd_norm);
      if (it > 2) {
        if (err_res <= prm.tol_f_abs || err_upd <= prm.tol_u_abs) conv = true;
        if (rel_res <= prm.tol_f && err_upd_norm <= prm.tol_u) conv = true;
        if (conv) break;
      }
      // setup + linear solve
      const double tol = prm.tol_lin * err_res;
      const int max_it = prm.max_it_mult * (int)n;
      std::fill(dx.begin(), dx.end(), 0.0);
      auto Am = [&](std::vector<double> &d, const std::vector<double> &s) { op.vmult(d.data(), s.data()); };
      int lin_it = 0; bool lconv = false;
      if (prm.precond == 2) {
        if (prm.level_fp32) setup_gmg<float>(prm, meshes, bas, lmask, lmu, u_tot, gmg_f, it <= 1);
        else setup_gmg<double>(prm, meshes, bas, lmask, lmu, u_tot, gmg_d, it <= 1);
        auto Pm = [&](std::vector<double> &d, const std::vector<double> &s) {
          if (prm.level_fp32) gmg_f.vmult(d, s); else gmg_d.vmult(d, s);
        };
        lin_it = cg_solve(Am, Pm, dx, R, max_it, tol, 0.0, &lconv, nullptr, nullptr, nullptr);
      } else if (prm.precond == 1) {
        op.compute_diagonal();
        auto Pm = [&](std::vector<double> &d, const std::vector<double> &s) {
          for (size_t i = 0; i < n; ++i) d[i] = prm.relaxation * op.inv_diag[i] * s[i];
        };
        lin_it = cg_solve(Am, Pm, dx, R, max_it, tol, 0.0, &lconv, nullptr, nullptr, nullptr);
      } else {
        auto Pm = [&](std::vector<double> &d, const std::vector<double> &s) { d = s; };
        lin_it = cg_solve(Am, Pm, dx, R, max_it, tol, 0.0, &lconv, nullptr, nullptr, nullptr);
      }
      if (!lconv) return 3;
      sr.cg_iterations.push_back(lin_it);
      double s = 0;
      for (size_t i = 0; i < n; ++i) { if (cmask[i]) dx[i] = 0; s += dx[i] * dx[i]; }
      err_upd = std::sqrt(s);
      for (size_t i = 0; i < n; ++i) if (cmask[i] && it == 0) dx[i] = gvals[i];
      if (it == 0) err_upd0 = err_upd;
      err_upd_norm = err_upd0 != 0 ? err_upd / err_upd0 : err_upd;
      for (size_t i = 0; i < n; ++i) du[i] += dx[i];
    }
    sr.newton_iterations = it;
    sr.converged = conv;
    sr.time = time;
    for (size_t i = 0; i < n; ++i) u_n[i] += du[i];
    if (prm.has_output_point) point_value(m, bas, u_n.data(), prm.output_point, sr.point_u);
    res.steps.push_back(sr);
    if (!conv) { res.u = u_n; return 4; }
    time += prm.dt;
  }
  res.u = u_n;
  return 0;
}

// Gradient of J(u(theta)) = 1/2 sum over the dofs on boundary `obj_id` of
// (u - u_target)^2 with respect to theta_c = log mu_c (no reference
// counterpart: the check of the device adjoint).  Forward: the load-stepping
// Newton solve with mu = exp(theta).  Adjoint: K(u) lambda = dJ/du (the
// symmetric tangent at the converged u, Dirichlet rows identity with zero
// right-hand side) by CG with the FP64 V-cycle to 1e-13 of ||dJ/du||.
// Gradient: dJ/dtheta_c = lambda . dR/dtheta_c, since R(u, theta) = 0 gives
// du/dtheta = K^-1 dR/dtheta.
int adjoint_run(const NewtonParams &prm_in, const std::vector<double> &log_mu, const std::vector<double> &target,
                int obj_id, double &J, std::vector<double> &grad, std::vector<double> &u) {
  NewtonParams prm = prm_in;
  Basis1D bas; bas.init(prm.mesh.p, prm.mesh.q);
  const int nl = prm.mesh.n_refinements + 1;
  std::vector<Mesh> meshes(nl);
  for (int l = 0; l < nl; ++l) build_mesh(prm.mesh, l, meshes[l]);
  const Mesh &m = meshes[nl - 1];
  if ((int)log_mu.size() != m.n_cells || (int)target.size() != m.n_dofs()) return 5;
  prm.mu_fine.resize(m.n_cells);
  for (int c = 0; c < m.n_cells; ++c) prm.mu_fine[c] = std::exp(log_mu[c]);
  NewtonResult res;
  const int rc = newton_run(prm, res);
  if (rc) return rc;
  u = res.u;
  std::vector<std::vector<double>> lmu(nl);
  for (int l = 0; l < nl; ++l) lmu[l] = coarsen_cell_field(meshes, l, prm.mu_fine);
  std::vector<std::vector<uint8_t>> lmask(nl);
  for (int l = 0; l < nl; ++l) constrained_dofs(meshes[l], prm.dirichlet, lmask[l]);
  const std::vector<uint8_t> &cmask = lmask[nl - 1];
  std::vector<uint8_t> obj;
  constrained_dofs(m, {DirichletSpec{obj_id, 7}}, obj);
  const size_t n = m.n_dofs();
  std::vector<double> rhs(n, 0.0), lam(n, 0.0);
  J = 0;
  for (size_t i = 0; i < n; ++i)
    if (obj[i]) {
      const double r = u[i] - target[i];
      J += 0.5 * r * r;
      if (!cmask[i]) rhs[i] = r;
    }
  Operator<double> op;
  op.initialize(&m, &bas, prm.caching, prm.formulation);
  op.set_material(lmu[nl - 1], prm.nu);
  op.set_constraints(cmask);
  if (op.cache(u.data())) return 2;
  GMG<double> gmg;
  setup_gmg<double>(prm, meshes, bas, lmask, lmu, u, gmg, true);
  auto Am = [&](std::vector<double> &d, const std::vector<double> &s) { op.vmult(d.data(), s.data()); };
  auto Pm = [&](std::vector<double> &d, const std::vector<double> &s) { gmg.vmult(d, s); };
  const double nr = norm2(rhs);
  bool conv = true;
  if (nr > 0) cg_solve(Am, Pm, lam, rhs, 100000, 1e-13 * nr, 0.0, &conv, nullptr, nullptr, nullptr);
  if (!conv) return 3;
  grad.assign(m.n_cells, 0.0);
  dresidual_dlogmu_dot(m, bas, lmu[nl - 1], prm.nu, prm.formulation, u.data(), lam.data(), grad.data());
  return 0;
}

}  // namespace orc

namespace orc {
template void setup_gmg<float>(const NewtonParams &, const std::vector<Mesh> &, const Basis1D &,
                               const std::vector<std::vector<uint8_t>> &, const std::vector<std::vector<double>> &,
                               const std::vector<double> &, GMG<float> &, bool);
template void setup_gmg<double>(const NewtonParams &, const std::vector<Mesh> &, const Basis1D &,
                                const std::vector<std::vector<uint8_t>> &, const std::vector<std::vector<double>> &,
                                const std::vector<double> &, GMG<double> &, bool);
}  // namespace orc
