// Problem object: .prm driven mesh, loads, operators and the device
// load-stepping Newton driver (Solid::run, solve_nonlinear_timestep,
// check_convergence, solve_linear_system of mf_elasticity.h:1187-1235,
// 2245-2559, 3012-3214), plus the adjoint gradient with respect to a
// per-cell log shear modulus.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "problem_internal.h"

namespace lsmf {

namespace {

uint64_t splitmix64(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uniform01(uint64_t &s) { return (splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

// Seeded non-overlapping spherical voids inside the box; coarse cells whose
// centre lies in a sphere are removed (a conforming hex mesh whose coarsest
// level already resolves the voids).
std::vector<uint8_t> void_mask(const ProblemParams &P) {
  const int nx = P.box_cells[0], ny = P.box_cells[1], nz = P.box_cells[2];
  std::vector<uint8_t> act((size_t)nx * ny * nz, 1);
  uint64_t s = (uint64_t)P.void_seed * 0x2545F4914F6CDD1Dull + 1;
  std::vector<std::array<double, 3>> c;
  const double r = P.void_radius;
  int tries = 0;
  while ((int)c.size() < P.void_count && tries < 100000) {
    ++tries;
    std::array<double, 3> p;
    for (int d = 0; d < 3; ++d) {
      const double L = P.box_hi[d] - P.box_lo[d];
      p[d] = P.box_lo[d] + r + uniform01(s) * (L - 2 * r);
    }
    bool ok = true;
    for (const auto &q : c) {
      const double dd = std::sqrt((p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) +
                                  (p[2] - q[2]) * (p[2] - q[2]));
      if (dd < 2.0 * r * 1.25) ok = false;
    }
    if (ok) c.push_back(p);
  }
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const double x[3] = {P.box_lo[0] + (i + 0.5) * (P.box_hi[0] - P.box_lo[0]) / nx,
                             P.box_lo[1] + (j + 0.5) * (P.box_hi[1] - P.box_lo[1]) / ny,
                             P.box_lo[2] + (k + 0.5) * (P.box_hi[2] - P.box_lo[2]) / nz};
        for (const auto &q : c)
          if ((x[0] - q[0]) * (x[0] - q[0]) + (x[1] - q[1]) * (x[1] - q[1]) + (x[2] - q[2]) * (x[2] - q[2]) < r * r)
            act[((size_t)k * ny + j) * nx + i] = 0;
      }
  return act;
}

void face_local_nodes(int p, int f, std::vector<int> &out) {
  out.clear();
  const int n1 = p + 1;
  for (int c = 0; c <= p; ++c)
    for (int b = 0; b <= p; ++b)
      for (int a = 0; a <= p; ++a) {
        const bool on = (f == 0 && a == 0) || (f == 1 && a == p) || (f == 2 && b == 0) || (f == 3 && b == p) ||
                        (f == 4 && c == 0) || (f == 5 && c == p);
        if (on) out.push_back((c * n1 + b) * n1 + a);
      }
}

// external (dead) load: sum over Neumann faces of N_a T(x, t) JxW with the
// face quadrature QGauss<2>(q) (mf_elasticity.h:2859-2892)
void neumann_load(const lsmf_problem &pb, double t, std::vector<double> &f) {
  const Level &L = *pb.mesh->levels.back();
  const Basis &B = pb.mesh->basis;
  const int p = L.p, q = L.q, n1 = p + 1, ncn = L.ncn();
  f.assign(L.n_dofs(), 0.0);
  std::vector<double> v[3], dv[3];
  for (int d = 0; d < 3; ++d) { v[d].resize(n1); dv[d].resize(n1); }
  for (size_t k = 0; k < L.bfaces.size(); k += 3) {
    const int cell = L.bfaces[k], face = L.bfaces[k + 1], id = L.bfaces[k + 2];
    for (const BCExpr &nm : pb.prm.neumann) {
      if (nm.id != id) continue;
      const int nd = face / 2, ta = nd == 0 ? 1 : 0, tb = nd == 2 ? 1 : 2;
      const int *nodes = &L.cell_nodes[(size_t)cell * ncn];
      for (int qb = 0; qb < q; ++qb)
        for (int qa = 0; qa < q; ++qa) {
          double xi[3];
          xi[nd] = (face & 1) ? 1.0 : 0.0;
          xi[ta] = B.qpts[qa];
          xi[tb] = B.qpts[qb];
          for (int d = 0; d < 3; ++d) B.eval(xi[d], v[d].data(), dv[d].data());
          double x[3] = {0, 0, 0}, tA[3] = {0, 0, 0}, tB[3] = {0, 0, 0};
          std::vector<double> Nv(ncn);
          for (int c = 0; c <= p; ++c)
            for (int b = 0; b <= p; ++b)
              for (int a = 0; a <= p; ++a) {
                const int ln = (c * n1 + b) * n1 + a;
                const int li[3] = {a, b, c};
                const double *X = &L.X[3 * (size_t)nodes[ln]];
                Nv[ln] = v[0][a] * v[1][b] * v[2][c];
                double ga = 1, gb = 1;
                for (int d = 0; d < 3; ++d) {
                  ga *= d == ta ? dv[d][li[d]] : v[d][li[d]];
                  gb *= d == tb ? dv[d][li[d]] : v[d][li[d]];
                }
                for (int d = 0; d < 3; ++d) {
                  x[d] += Nv[ln] * X[d];
                  tA[d] += ga * X[d];
                  tB[d] += gb * X[d];
                }
              }
          const double cr[3] = {tA[1] * tB[2] - tA[2] * tB[1], tA[2] * tB[0] - tA[0] * tB[2],
                                tA[0] * tB[1] - tA[1] * tB[0]};
          const double jxw = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]) * B.qw[qa] * B.qw[qb];
          double T[3];
          for (int c = 0; c < 3; ++c) T[c] = nm.expr[c].eval(x[0], x[1], x[2], t);
          for (int ln = 0; ln < ncn; ++ln)
            for (int c = 0; c < 3; ++c) f[3 * (size_t)nodes[ln] + c] += Nv[ln] * T[c] * jxw;
        }
    }
  }
}

// constrained values of the load step (applied as the step increment at the
// first Newton iteration, mf_elasticity.h:2963 and :3211)
bool dirichlet_values(const lsmf_problem &pb, double t, std::vector<double> &g) {
  const Level &L = *pb.mesh->levels.back();
  g.assign(L.n_dofs(), 0.0);
  bool nonzero = false;
  std::vector<int> fl;
  const int ncn = L.ncn();
  for (size_t k = 0; k < L.bfaces.size(); k += 3) {
    const int cell = L.bfaces[k], face = L.bfaces[k + 1], id = L.bfaces[k + 2];
    for (const BCExpr &d : pb.prm.dirichlet) {
      if (d.id != id) continue;
      const auto mit = pb.prm.dirichlet_mask.find(id);
      const int mask = mit == pb.prm.dirichlet_mask.end() ? 7 : mit->second;
      face_local_nodes(L.p, face, fl);
      for (int ln : fl) {
        const int node = L.cell_nodes[(size_t)cell * ncn + ln];
        const double *X = &L.X[3 * (size_t)node];
        for (int c = 0; c < 3; ++c)
          if (mask & (1 << c)) {
            const double v = d.expr[c].eval(X[0], X[1], X[2], t);
            g[3 * (size_t)node + c] = v;
            if (v != 0.0) nonzero = true;
          }
      }
    }
  }
  return nonzero;
}

bool locate_point(const Level &L, const Basis &B, const double pt[3], std::vector<int> &nodes, std::vector<double> &w) {
  const int p = L.p, n1 = p + 1, ncn = L.ncn();
  std::vector<double> v[3], dv[3];
  for (int d = 0; d < 3; ++d) { v[d].resize(n1); dv[d].resize(n1); }
  for (int c = 0; c < L.n_cells; ++c) {
    const int *cn = &L.cell_nodes[(size_t)c * ncn];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int a = 0; a < ncn; ++a)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], L.X[3 * (size_t)cn[a] + d]);
        hi[d] = std::max(hi[d], L.X[3 * (size_t)cn[a] + d]);
      }
    bool in = true;
    for (int d = 0; d < 3; ++d) {
      const double h = (hi[d] - lo[d]) * 1e-9 + 1e-300;
      if (pt[d] < lo[d] - h || pt[d] > hi[d] + h) in = false;
    }
    if (!in) continue;
    double xi[3] = {0.5, 0.5, 0.5};
    for (int it = 0; it < 50; ++it) {
      for (int d = 0; d < 3; ++d) B.eval(xi[d], v[d].data(), dv[d].data());
      double x[3] = {0, 0, 0}, J[3][3] = {};
      for (int zc = 0; zc <= p; ++zc)
        for (int yb = 0; yb <= p; ++yb)
          for (int xa = 0; xa <= p; ++xa) {
            const double *X = &L.X[3 * (size_t)cn[(zc * n1 + yb) * n1 + xa]];
            const double N = v[0][xa] * v[1][yb] * v[2][zc];
            const double g[3] = {dv[0][xa] * v[1][yb] * v[2][zc], v[0][xa] * dv[1][yb] * v[2][zc],
                                 v[0][xa] * v[1][yb] * dv[2][zc]};
            for (int d = 0; d < 3; ++d) {
              x[d] += N * X[d];
              for (int e = 0; e < 3; ++e) J[d][e] += X[d] * g[e];
            }
          }
      const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                         J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                         J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
      double Ji[3][3];
      Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
      Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
      Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
      Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
      Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
      Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
      Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
      Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
      Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
      double s = 0;
      for (int d = 0; d < 3; ++d) {
        double dx = 0;
        for (int e = 0; e < 3; ++e) dx += Ji[d][e] * (pt[e] - x[e]);
        xi[d] += dx;
        s += std::fabs(dx);
      }
      if (s < 1e-14) break;
    }
    const double tol = 1e-10;
    if (xi[0] < -tol || xi[0] > 1 + tol || xi[1] < -tol || xi[1] > 1 + tol || xi[2] < -tol || xi[2] > 1 + tol)
      continue;
    for (int d = 0; d < 3; ++d) B.eval(std::min(1.0, std::max(0.0, xi[d])), v[d].data(), nullptr);
    nodes.assign(cn, cn + ncn);
    w.resize(ncn);
    for (int zc = 0; zc <= p; ++zc)
      for (int yb = 0; yb <= p; ++yb)
        for (int xa = 0; xa <= p; ++xa) w[(zc * n1 + yb) * n1 + xa] = v[0][xa] * v[1][yb] * v[2][zc];
    return true;
  }
  return false;
}

double norm_of(lsmf_problem *pb, const double *v) {
  lsmf_op *op = pb->op;
  const size_t n = (size_t)op->L().n_dofs();
  if (dot_async(v, v, false, n, op->partial.ptr, op->sc.ptr, SC_TMP, pb->stream) != LSMF_OK) return NAN;
  double r = 0;
  cudaMemcpyAsync(&r, op->sc.ptr + SC_TMP, sizeof(double), cudaMemcpyDeviceToHost, pb->stream);
  cudaStreamSynchronize(pb->stream);
  return std::sqrt(r);
}

struct Timer {
  cudaEvent_t a, b;
  cudaStream_t s;
  explicit Timer(cudaStream_t st) : s(st) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
  }
  double stop() {
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms * 1e-3;
  }
};

// R = fext - f_int(u) with the constrained entries zeroed: the right-hand
// side of assemble_system (mf_elasticity.h:2736-2921); fext is the device
// Neumann load of the step
lsmf_status residual_async(lsmf_problem *pb, const double *u, const double *fext, double *R) {
  const Level &L = *pb->mesh->levels.back();
  const size_t n = (size_t)L.n_dofs();
  cudaStream_t st = pb->stream;
  LSMF_CUDA(cudaMemcpyAsync(R, fext, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  LSMF_TRY(internal_force_async(L, pb->mesh->basis, u, pb->mu_dev.ptr, pb->prm.nu, pb->prm.formulation, R,
                                pb->op->scatter, st));
  return set_indexed_async<double>(R, L.d_constrained.ptr, (int)L.constrained.size(), 0.0, st);
}

// "gmg-gc" (global coarsening, mf_elasticity.h:1597-1632, 1892-1916) builds
// its levels by coarsening the triangulation; on the structured meshes here,
// which are refined globally and have no hanging nodes, that sequence is the
// multigrid level hierarchy itself, the two-level transfers are the nested
// Q_p interpolation with the levels' homogeneous Dirichlet constraints, and
// the preconditioner is the same as "gmg"
int precond_code(const std::string &s) { return s == "none" ? 0 : (s == "jacobi" ? 1 : 2); }

}  // namespace

// Solid::run with the device Newton loop.  Returns the status of the first
// failure (CG or Newton non-convergence, det F <= 0, CUDA errors).
lsmf_status problem_run(lsmf_problem *pb, lsmf_newton_info *info) {
  const ProblemParams &P = pb->prm;
  lsmf_op *op = pb->op;
  const Level &L = *pb->mesh->levels.back();
  const size_t n = (size_t)L.n_dofs();
  cudaStream_t st = pb->stream;
  op->stream = st;
  if (pb->gmg) lsmf_gmg_set_stream(pb->gmg, st);
  const int pc = precond_code(P.precond);
  const int nc = (int)L.constrained.size();
  const int *cidx = L.d_constrained.ptr;
  double *u_n = pb->u_n.ptr, *du = pb->du.ptr, *u_tot = pb->u_tot.ptr, *R = pb->R.ptr, *dx = pb->dx.ptr;
  LSMF_CUDA(cudaMemsetAsync(u_n, 0, n * sizeof(double), st));
  if (info) std::memset(info, 0, sizeof(*info));
  std::vector<double> fext, g;
  double time = 0.0;
  time += P.dt;  // Time::increment
  int step = 0;
  lsmf_status result = LSMF_OK;
  while (time <= P.end_time) {
    neumann_load(*pb, time, fext);
    LSMF_TRY(pb->fext.upload(fext.data(), n));
    const bool inhom = dirichlet_values(*pb, time, g);
    if (inhom) LSMF_TRY(pb->gvals.upload(g.data(), n));
    LSMF_CUDA(cudaMemsetAsync(du, 0, n * sizeof(double), st));
    double err_res = 0, err_res0 = 0, err_upd = 0, err_upd0 = 0, err_upd_norm = 0;
    int it = 0, cg_total = 0;
    bool conv = false;
    for (; it < P.max_nr; ++it) {
      // set_total_solution + assemble_system (residual part)
      Timer tr(st);
      LSMF_CUDA(cudaMemcpyAsync(u_tot, u_n, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
      LSMF_TRY(axpy_async<double>(u_tot, 1.0, du, n, st));
      LSMF_TRY(residual_async(pb, u_tot, pb->fext.ptr, R));
      bool cached = false;
      if (it == 0 && inhom) {
        // rhs -= K g over the constrained columns (the inhomogeneity that
        // AffineConstraints::distribute_local_to_global moves into the rhs)
        LSMF_TRY(lsmf_operator_cache(op, u_tot));
        cached = true;
        LSMF_TRY(launch_apply_inhomogeneous(op, pb->tmp.ptr, pb->gvals.ptr));
        LSMF_TRY(axpy_async<double>(R, -1.0, pb->tmp.ptr, n, st));
        LSMF_TRY(set_indexed_async<double>(R, cidx, nc, 0.0, st));
      }
      err_res = norm_of(pb, R);
      if (info) info->time_residual += tr.stop(); else tr.stop();
      if (it == 0) err_res0 = err_res;
      // check_convergence (mf_elasticity.h:2245-2284): at least 3 iterations
      const double rel_res = err_res0 != 0.0 ? err_res / err_res0 : err_res;
      if (it > 2) {
        if (err_res <= P.tol_f_abs || err_upd <= P.tol_u_abs) conv = true;
        if (rel_res <= P.tol_f && err_upd_norm <= P.tol_u) conv = true;
        if (conv) break;
      }
      // setup_matrix_free: fine cache, level caches, diagonals, eigenvalues
      Timer ts(st);
      if (!cached) LSMF_TRY(lsmf_operator_cache(op, u_tot));
      if (pc == 1) LSMF_TRY(lsmf_operator_compute_diagonal(op));
      if (pc == 2) LSMF_TRY(lsmf_gmg_setup(pb->gmg, u_tot));
      if (info) info->time_setup += ts.stop(); else ts.stop();
      // solve_linear_system: CG to tol_lin * ||R||
      Timer tl(st);
      LSMF_CUDA(cudaMemsetAsync(dx, 0, n * sizeof(double), st));
      lsmf_solve_info si{};
      const lsmf_status cs = lsmf_cg_solve(op, pc, P.relaxation, pb->gmg, dx, R, P.tol_lin * err_res,
                                           P.max_it_mult * (int)n, &si);
      if (info) info->time_solve += tl.stop(); else tl.stop();
      if (cs != LSMF_OK) return cs;
      cg_total += si.iterations;
      LSMF_TRY(set_indexed_async<double>(dx, cidx, nc, 0.0, st));
      err_upd = norm_of(pb, dx);
      if (it == 0 && inhom) LSMF_TRY(copy_indexed_async<double>(dx, pb->gvals.ptr, cidx, nc, st));
      if (it == 0) err_upd0 = err_upd;
      err_upd_norm = err_upd0 != 0.0 ? err_upd / err_upd0 : err_upd;
      LSMF_TRY(axpy_async<double>(du, 1.0, dx, n, st));
    }
    LSMF_TRY(axpy_async<double>(u_n, 1.0, du, n, st));
    if (info && step < 256) {
      info->newton_iterations[step] = it;
      info->cg_iterations[step] = cg_total;
      if (pb->have_point) {
        std::vector<double> vals(3 * pb->point_nodes.size());
        for (size_t a = 0; a < pb->point_nodes.size(); ++a)
          LSMF_CUDA(cudaMemcpyAsync(&vals[3 * a], u_n + 3 * (size_t)pb->point_nodes[a], 3 * sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
        LSMF_CUDA(cudaStreamSynchronize(st));
        for (int c = 0; c < 3; ++c) {
          double s = 0;
          for (size_t a = 0; a < pb->point_nodes.size(); ++a) s += pb->point_w[a] * vals[3 * a + c];
          info->point_u[step][c] = s;
        }
      }
      info->n_steps = step + 1;
    }
    ++step;
    if (!conv) {
      // the reference's AssertThrow(newton_iteration <= max) never fires;
      // this driver reports the non-converged load step instead
      set_error("No convergence in nonlinear solver!");
      result = LSMF_ERR_NEWTON_NOT_CONVERGED;
      break;
    }
    time += P.dt;
  }
  LSMF_CUDA(cudaStreamSynchronize(st));
  return result;
}

}  // namespace lsmf

using namespace lsmf;

lsmf_problem::~lsmf_problem() {
  if (gmg) lsmf_gmg_destroy(gmg);
  if (op) lsmf_operator_destroy(op);
  if (mesh) lsmf_mesh_destroy(mesh);
}

extern "C" {

// Checks of a parsed parameter set that do not need a device (the
// reference's AssertThrow / ParameterHandler pattern checks).
static lsmf_status validate_params(const ProblemParams &P, int &caching) {
  if (P.dim != 3) { set_error("only Dimension = 3 is supported"); return LSMF_ERR_UNSUPPORTED; }
  if (P.solver_type != "MF_CG") { set_error("Solver type " + P.solver_type + " is not supported (MF_CG only)"); return LSMF_ERR_UNSUPPORTED; }
  if (P.precond != "jacobi" && P.precond != "gmg" && P.precond != "gmg-gc" && P.precond != "none") {
    set_error("Preconditioner type " + P.precond + " is not supported (jacobi | gmg | gmg-gc | none)");
    return LSMF_ERR_UNSUPPORTED;
  }
  if (P.caching == "scalar") caching = LSMF_CACHE_SCALAR;
  else if (P.caching == "tensor2") caching = LSMF_CACHE_TENSOR2;
  else if (P.caching == "tensor4") caching = LSMF_CACHE_TENSOR4;
  else if (P.caching == "scalar_referential") caching = LSMF_CACHE_SCALAR_REFERENTIAL;
  else if (P.caching == "tensor4_ns") caching = LSMF_CACHE_TENSOR4_NS;
  else { set_error("Unknown caching"); return LSMF_ERR_UNKNOWN_CACHING; }
  if (P.formulation != 0 && P.formulation != 1) { set_error("Unknown material formulation"); return LSMF_ERR_PRM; }
  if (P.formulation == 0 && caching != LSMF_CACHE_SCALAR) {
    set_error("formulation 0 requires scalar caching");
    return LSMF_ERR_UNSUPPORTED;
  }
  if (P.degree < 1 || P.degree > 4 || P.quad_order != P.degree + 1) {
    set_error("supported elements: Polynomial degree 1..4 with Quadrature order = degree + 1");
    return LSMF_ERR_UNSUPPORTED;
  }
  if (P.level_precision != "float" && P.level_precision != "double") {
    set_error("MF level precision must be float or double");
    return LSMF_ERR_PRM;
  }
  if (P.scatter != "atomic" && P.scatter != "colour8" && P.scatter != "nodesum") {
    set_error("MF scatter must be atomic, colour8 or nodesum");
    return LSMF_ERR_PRM;
  }
  if (P.type != "Cook" && P.type != "Box") {
    set_error("Geometry Type " + P.type + " is not supported (Cook | Box)");
    return LSMF_ERR_UNSUPPORTED;
  }
  if (!(P.nu > -1.0 && P.nu < 0.5) || !(P.mu > 0.0)) { set_error("bad material parameters"); return LSMF_ERR_PRM; }
  if (!(P.dt > 0.0)) { set_error("Time step size must be positive"); return LSMF_ERR_PRM; }
  for (const BCExpr &d : P.dirichlet)
    if (!P.dirichlet_mask.count(d.id)) {
      set_error("Could not find component mask for ID " + std::to_string(d.id));
      return LSMF_ERR_PRM;
    }
  return LSMF_OK;
}

lsmf_status lsmf_prm_validate(const char *text) {
  if (!text) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  ProblemParams P;
  LSMF_TRY(parse_prm(text, P));
  int caching = 0;
  return validate_params(P, caching);
}

lsmf_status lsmf_problem_create(const char *text, lsmf_problem **out) {
  if (!text || !out) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  *out = nullptr;
  ProblemParams P;
  LSMF_TRY(parse_prm(text, P));
  int caching = 0;
  LSMF_TRY(validate_params(P, caching));
  lsmf_mesh_desc md{};
  md.degree = P.degree;
  md.n_q_points_1d = P.quad_order;
  md.n_refinements = P.n_refinements;
  std::vector<uint8_t> act;
  if (P.type == "Cook") {
    md.geometry = LSMF_GEOM_COOK;
    md.coarse[0] = md.coarse[1] = P.elements_per_edge;
    md.coarse[2] = 1;
    md.lo[0] = 0; md.lo[1] = 0; md.lo[2] = -0.5 * P.cook_thickness;
    md.hi[0] = 48; md.hi[1] = 44; md.hi[2] = 0.5 * P.cook_thickness;
    md.scale = P.scale;
  } else if (P.type == "Box") {
    md.geometry = LSMF_GEOM_BOX;
    for (int k = 0; k < 3; ++k) { md.coarse[k] = P.box_cells[k]; md.lo[k] = P.box_lo[k]; md.hi[k] = P.box_hi[k]; }
    md.scale = 1.0;
    if (P.void_count > 0) {
      act = void_mask(P);
      md.coarse_active = act.data();
    }
  }
  lsmf_problem *pb = new (std::nothrow) lsmf_problem();
  if (!pb) return LSMF_ERR_ALLOC;
  pb->prm = P;
  lsmf_status s = lsmf_mesh_create(&md, &pb->mesh);
  if (s != LSMF_OK) { delete pb; return s; }
  std::vector<int> ids, masks;
  for (const BCExpr &d : P.dirichlet) { ids.push_back(d.id); masks.push_back(P.dirichlet_mask[d.id]); }
  if ((s = lsmf_mesh_set_dirichlet(pb->mesh, (int)ids.size(), ids.data(), masks.data())) != LSMF_OK ||
      (s = lsmf_operator_create(pb->mesh, -1, (lsmf_caching)caching, P.formulation, LSMF_FP64, &pb->op)) != LSMF_OK) {
    delete pb;
    return s;
  }
  // the Newton driver's operator in one launch: with its cell loop chunked
  // the Newton step of the voids benchmark (60^3 Q2, FP32 and FP64 levels)
  // measured 3.5-4.5 % slower, although the chunked operator alone and in a
  // Jacobi-CG measured faster
  pb->op->chunks = 1;
  if (precond_code(P.precond) == 2) {
    lsmf_gmg_desc gd{};
    gd.caching = caching;
    gd.formulation = P.formulation;
    gd.precision = P.level_precision == "float" ? LSMF_FP32 : LSMF_FP64;
    gd.smoother_degree = P.cheb_degree;
    gd.smoothing_range = P.smoothing_range;
    gd.eig_cg_iterations = P.cheb_eig_its;
    gd.coarse_chebyshev = P.coarse_chebyshev;
    gd.coarse_accurate_eig = P.coarse_accurate_eig;
    if ((s = lsmf_gmg_create(pb->mesh, &gd, &pb->gmg)) != LSMF_OK) { delete pb; return s; }
  }
  if (P.scatter != "atomic") {
    const int mode = P.scatter == "colour8" ? LSMF_SCATTER_COLOUR8 : LSMF_SCATTER_NODESUM;
    if ((s = set_scatter_mode(pb->op, mode)) != LSMF_OK ||
        (pb->gmg && (s = lsmf_gmg_set_option(pb->gmg, LSMF_GMG_OPT_SCATTER, mode)) != LSMF_OK)) {
      delete pb;
      return s;
    }
  }
  const Level &L = *pb->mesh->levels.back();
  const size_t n = (size_t)L.n_dofs();
  for (auto *b : {&pb->u_n, &pb->du, &pb->u_tot, &pb->R, &pb->dx, &pb->fext, &pb->gvals, &pb->tmp, &pb->lam})
    if ((s = b->alloc(n)) != LSMF_OK) { delete pb; return s; }
  if ((s = pb->op->sc.alloc(SC_N)) != LSMF_OK || (s = pb->op->partial.alloc(reduce_blocks())) != LSMF_OK) {
    delete pb;
    return s;
  }
  if (!P.output_points.empty()) {
    double pt[3] = {P.output_points[0][0], P.output_points[0][1], P.output_points[0][2]};
    pb->have_point = locate_point(L, pb->mesh->basis, pt, pb->point_nodes, pb->point_w);
    if (!pb->have_point) { set_error("Found no cell with point inside!"); delete pb; return LSMF_ERR_PRM; }
  }
  std::vector<double> mu(L.n_cells, P.mu);
  if ((s = lsmf_problem_set_mu(pb, mu.data())) != LSMF_OK) { delete pb; return s; }
  *out = pb;
  return LSMF_OK;
}

void lsmf_problem_destroy(lsmf_problem *p) { delete p; }

lsmf_status lsmf_problem_set_mu(lsmf_problem *pb, const double *mu) {
  if (!pb || !mu) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  const int nc = pb->mesh->levels.back()->n_cells;
  pb->mu_fine.assign(mu, mu + nc);
  LSMF_TRY(lsmf_operator_set_material(pb->op, mu, pb->prm.nu));
  LSMF_TRY(pb->mu_dev.upload(mu, nc));
  if (pb->gmg) LSMF_TRY(lsmf_gmg_set_material(pb->gmg, mu, pb->prm.nu));
  pb->forward_done = false;
  return LSMF_OK;
}

lsmf_status lsmf_problem_info(const lsmf_problem *pb, int *n_cells, int *n_dofs, double *volume) {
  if (!pb) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  const Level &L = *pb->mesh->levels.back();
  if (n_cells) *n_cells = L.n_cells;
  if (n_dofs) *n_dofs = L.n_dofs();
  if (volume) {
    // sum of det J_ref w over the quadrature points (GridTools::volume)
    const Basis &B = pb->mesh->basis;
    const int p = L.p, q = L.q, n1 = p + 1, ncn = L.ncn();
    double vol = 0;
    for (int c = 0; c < L.n_cells; ++c) {
      const int *cn = &L.cell_nodes[(size_t)c * ncn];
      for (int qz = 0; qz < q; ++qz)
        for (int qy = 0; qy < q; ++qy)
          for (int qx = 0; qx < q; ++qx) {
            double J[3][3] = {};
            for (int zc = 0; zc <= p; ++zc)
              for (int yb = 0; yb <= p; ++yb)
                for (int xa = 0; xa <= p; ++xa) {
                  const double *X = &L.X[3 * (size_t)cn[(zc * n1 + yb) * n1 + xa]];
                  const double g[3] = {B.D[qx * n1 + xa] * B.N[qy * n1 + yb] * B.N[qz * n1 + zc],
                                       B.N[qx * n1 + xa] * B.D[qy * n1 + yb] * B.N[qz * n1 + zc],
                                       B.N[qx * n1 + xa] * B.N[qy * n1 + yb] * B.D[qz * n1 + zc]};
                  for (int d = 0; d < 3; ++d)
                    for (int e = 0; e < 3; ++e) J[d][e] += X[d] * g[e];
                }
            const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                               J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                               J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
            vol += det * B.qw[qx] * B.qw[qy] * B.qw[qz];
          }
    }
    *volume = vol;
  }
  return LSMF_OK;
}

lsmf_status lsmf_problem_set_stream(lsmf_problem *pb, void *stream) {
  if (!pb) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  pb->stream = (cudaStream_t)stream;
  return LSMF_OK;
}

lsmf_status lsmf_problem_run(lsmf_problem *pb, lsmf_newton_info *info) {
  if (!pb) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  return problem_run(pb, info);
}

lsmf_status lsmf_residual(lsmf_problem *pb, const double *d_u, double t, double *d_R, double *norm) {
  if (!pb || !d_u || !d_R) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  const size_t n = (size_t)pb->mesh->levels.back()->n_dofs();
  std::vector<double> fext;
  neumann_load(*pb, t, fext);
  LSMF_TRY(pb->fext.upload(fext.data(), n));
  LSMF_TRY(residual_async(pb, d_u, pb->fext.ptr, d_R));
  const double r = norm_of(pb, d_R);
  if (!(r == r)) { set_error("residual norm is not a number"); return LSMF_ERR_CUDA; }
  if (norm) *norm = r;
  return LSMF_OK;
}

lsmf_status lsmf_problem_get_solution(const lsmf_problem *pb, double *host_u) {
  if (!pb || !host_u) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  const size_t n = (size_t)pb->mesh->levels.back()->n_dofs();
  LSMF_CUDA(cudaStreamSynchronize(pb->stream));
  LSMF_CUDA(cudaMemcpy(host_u, pb->u_n.ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
  return LSMF_OK;
}

// J = 1/2 sum over the dofs of the nodes on boundary `obj_id` of (u - u_target)^2
lsmf_status lsmf_adjoint_forward(lsmf_problem *pb, const double *log_mu, const double *u_target, int obj_id,
                                 double *J) {
  if (!pb || !log_mu || !u_target || !J) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  const Level &L = *pb->mesh->levels.back();
  std::vector<double> mu(L.n_cells);
  for (int c = 0; c < L.n_cells; ++c) mu[c] = std::exp(log_mu[c]);
  LSMF_TRY(lsmf_problem_set_mu(pb, mu.data()));
  lsmf_newton_info info;
  LSMF_TRY(problem_run(pb, &info));
  const size_t n = (size_t)L.n_dofs();
  pb->obj_mask_dofs.assign(n, 0);
  std::vector<int> fl;
  for (size_t k = 0; k < L.bfaces.size(); k += 3)
    if (L.bfaces[k + 2] == obj_id) {
      face_local_nodes(L.p, L.bfaces[k + 1], fl);
      for (int ln : fl) {
        const int node = L.cell_nodes[(size_t)L.bfaces[k] * L.ncn() + ln];
        for (int c = 0; c < 3; ++c) pb->obj_mask_dofs[3 * (size_t)node + c] = 1;
      }
    }
  std::vector<double> u(n);
  LSMF_TRY(lsmf_problem_get_solution(pb, u.data()));
  double j = 0;
  for (size_t i = 0; i < n; ++i)
    if (pb->obj_mask_dofs[i]) j += 0.5 * (u[i] - u_target[i]) * (u[i] - u_target[i]);
  LSMF_TRY(pb->target.upload(u_target, n));
  *J = j;
  pb->adjoint_obj_id = obj_id;
  pb->forward_done = true;
  return LSMF_OK;
}

// K(u) lambda = dJ/du with the same GMG-CG (homogeneous Dirichlet rows), then
// dJ/dlog_mu_c = lambda . dR/dlog_mu_c = -lambda . f_int of cell c (the
// internal force is linear in the cell's mu for both formulations).
lsmf_status lsmf_adjoint_backward(lsmf_problem *pb, double *grad) {
  if (!pb || !grad) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (!pb->forward_done) { set_error("lsmf_adjoint_forward has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  const ProblemParams &P = pb->prm;
  const Level &L = *pb->mesh->levels.back();
  const size_t n = (size_t)L.n_dofs();
  cudaStream_t st = pb->stream;
  std::vector<double> u(n), rhs(n, 0.0), tgt(n);
  LSMF_TRY(lsmf_problem_get_solution(pb, u.data()));
  LSMF_CUDA(cudaMemcpy(tgt.data(), pb->target.ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
  for (size_t i = 0; i < n; ++i)
    if (pb->obj_mask_dofs[i] && !L.cmask[i]) rhs[i] = u[i] - tgt[i];
  LSMF_TRY(pb->R.upload(rhs.data(), n));
  LSMF_TRY(lsmf_operator_cache(pb->op, pb->u_n.ptr));
  const int pc = precond_code(P.precond);
  if (pc == 1) LSMF_TRY(lsmf_operator_compute_diagonal(pb->op));
  if (pc == 2) LSMF_TRY(lsmf_gmg_setup(pb->gmg, pb->u_n.ptr));
  LSMF_CUDA(cudaMemsetAsync(pb->lam.ptr, 0, n * sizeof(double), st));
  double nr = 0;
  for (double v : rhs) nr += v * v;
  nr = std::sqrt(nr);
  lsmf_solve_info si{};
  if (nr > 0) LSMF_TRY(lsmf_cg_solve(pb->op, pc, P.relaxation, pb->gmg, pb->lam.ptr, pb->R.ptr, 1e-13 * nr,
                                     std::max(1000, P.max_it_mult * (int)n), &si));
  LSMF_TRY(pb->grad.alloc(L.n_cells));
  LSMF_TRY(adjoint_cell_grad_async(L, pb->mesh->basis, pb->u_n.ptr, pb->mu_dev.ptr, P.nu, P.formulation,
                                   pb->lam.ptr, pb->grad.ptr, st));
  LSMF_CUDA(cudaStreamSynchronize(st));
  LSMF_CUDA(cudaMemcpy(grad, pb->grad.ptr, L.n_cells * sizeof(double), cudaMemcpyDeviceToHost));
  return LSMF_OK;
}

}  // extern "C"
