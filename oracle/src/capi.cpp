// CPU oracle (test infrastructure only): flat C interface for ctypes.
#include <cstring>
#include <exception>
#include <string>

#include "oracle.h"
#include "solver.h"

using namespace orc;

namespace {
struct MeshH { Mesh m; Basis1D b; MeshDesc d; };
struct OpH {
  MeshH *mh; bool fp32;
  Operator<double> od; Operator<float> of;
};
thread_local std::string g_err;
}  // namespace

extern "C" {

const char *orc_last_error() { return g_err.c_str(); }

void *orc_mesh_new(int geom, const int *coarse, int level, const double *lo, const double *hi,
                   double scale, int p, int q, const unsigned char *coarse_active) {
  try {
    auto *h = new MeshH();
    h->d.geometry = geom;
    for (int k = 0; k < 3; ++k) { h->d.coarse[k] = coarse[k]; h->d.lo[k] = lo[k]; h->d.hi[k] = hi[k]; }
    h->d.n_refinements = level; h->d.scale = scale; h->d.p = p; h->d.q = q;
    if (coarse_active) h->d.coarse_active.assign(coarse_active, coarse_active + coarse[0] * coarse[1] * coarse[2]);
    build_mesh(h->d, level, h->m);
    h->b.init(p, q);
    return h;
  } catch (std::exception &e) { g_err = e.what(); return nullptr; }
}
void orc_mesh_free(void *h) { delete (MeshH *)h; }
void orc_mesh_sizes(void *hh, int *out) {
  auto *h = (MeshH *)hh;
  out[0] = h->m.n_cells; out[1] = h->m.n_nodes;
  for (int k = 0; k < 3; ++k) { out[2 + k] = h->m.nc[k]; out[5 + k] = h->m.nn[k]; }
  out[8] = (int)h->m.bfaces.size() / 3;
}
void orc_mesh_arrays(void *hh, double *X, int *cell_nodes, int *cell_ijk, int *bfaces) {
  auto *h = (MeshH *)hh;
  if (X) std::memcpy(X, h->m.X.data(), sizeof(double) * h->m.X.size());
  if (cell_nodes) std::memcpy(cell_nodes, h->m.cell_nodes.data(), sizeof(int) * h->m.cell_nodes.size());
  if (cell_ijk) std::memcpy(cell_ijk, h->m.cell_ijk.data(), sizeof(int) * h->m.cell_ijk.size());
  if (bfaces) std::memcpy(bfaces, h->m.bfaces.data(), sizeof(int) * h->m.bfaces.size());
}
double orc_mesh_volume(void *hh) { auto *h = (MeshH *)hh; return mesh_volume(h->m, h->b); }
void orc_mesh_constraints(void *hh, int n, const int *ids, const int *masks, unsigned char *out) {
  auto *h = (MeshH *)hh;
  std::vector<DirichletSpec> bc;
  for (int i = 0; i < n; ++i) bc.push_back({ids[i], masks[i]});
  std::vector<uint8_t> m;
  constrained_dofs(h->m, bc, m);
  std::memcpy(out, m.data(), m.size());
}
void orc_basis(int p, int q, double *nodes, double *qpts, double *qw, double *N, double *D) {
  Basis1D b; b.init(p, q);
  std::memcpy(nodes, b.nodes.data(), sizeof(double) * (p + 1));
  std::memcpy(qpts, b.qpts.data(), sizeof(double) * q);
  std::memcpy(qw, b.qw.data(), sizeof(double) * q);
  std::memcpy(N, b.N.data(), sizeof(double) * q * (p + 1));
  std::memcpy(D, b.D.data(), sizeof(double) * q * (p + 1));
}

void *orc_op_new(void *mh, int caching, int formulation, int fp32) {
  try {
    auto *h = new OpH();
    h->mh = (MeshH *)mh; h->fp32 = fp32 != 0;
    if (h->fp32) h->of.initialize(&h->mh->m, &h->mh->b, caching, formulation);
    else h->od.initialize(&h->mh->m, &h->mh->b, caching, formulation);
    return h;
  } catch (std::exception &e) { g_err = e.what(); return nullptr; }
}
void orc_op_free(void *h) { delete (OpH *)h; }
void orc_op_set_material(void *hh, const double *mu, double nu) {
  auto *h = (OpH *)hh;
  std::vector<double> m(mu, mu + h->mh->m.n_cells);
  if (h->fp32) h->of.set_material(m, nu); else h->od.set_material(m, nu);
}
void orc_op_set_constraints(void *hh, const unsigned char *mask) {
  auto *h = (OpH *)hh;
  std::vector<uint8_t> m(mask, mask + h->mh->m.n_dofs());
  if (h->fp32) h->of.set_constraints(m); else h->od.set_constraints(m);
}
int orc_op_cache(void *hh, const void *u) {
  auto *h = (OpH *)hh;
  return h->fp32 ? h->of.cache((const float *)u) : h->od.cache((const double *)u);
}
void orc_op_vmult(void *hh, void *dst, const void *src) {
  auto *h = (OpH *)hh;
  if (h->fp32) h->of.vmult((float *)dst, (const float *)src);
  else h->od.vmult((double *)dst, (const double *)src);
}
void orc_op_apply_inhom(void *hh, void *dst, const void *g) {
  auto *h = (OpH *)hh;
  if (h->fp32) h->of.apply_inhomogeneous((float *)dst, (const float *)g);
  else h->od.apply_inhomogeneous((double *)dst, (const double *)g);
}
void orc_op_diagonal(void *hh, void *diag, void *inv) {
  auto *h = (OpH *)hh;
  const size_t n = h->mh->m.n_dofs();
  if (h->fp32) {
    h->of.compute_diagonal();
    if (diag) std::memcpy(diag, h->of.diag.data(), 4 * n);
    if (inv) std::memcpy(inv, h->of.inv_diag.data(), 4 * n);
  } else {
    h->od.compute_diagonal();
    if (diag) std::memcpy(diag, h->od.diag.data(), 8 * n);
    if (inv) std::memcpy(inv, h->od.inv_diag.data(), 8 * n);
  }
}
void orc_op_cell_apply(void *hh, int cell, const void *in, void *out) {
  auto *h = (OpH *)hh;
  if (h->fp32) h->of.cell_apply(cell, (const float *)in, (float *)out);
  else h->od.cell_apply(cell, (const double *)in, (double *)out);
}
// which: 0 scalar, 1 second scalar, 2 tensor2 (6/qp), 3 tensor4 (36/qp),
// 4 inverse Jacobian (9/qp), 5 JxW (both in the frame the variant integrates
// in), 6 scalar_referential displacement values (3/qp), 7 tensor4_ns (81/qp);
// returns the element count
long orc_op_get_table(void *hh, int which, void *out) {
  auto *h = (OpH *)hh;
  auto get = [&](auto &op) -> long {
    const bool ref = op.referential();
    const auto *v = which == 0 ? &op.c_scalar : (which == 1 || which == 6) ? &op.c_second : which == 2 ? &op.c_t2
                  : which == 3 ? &op.c_t4 : which == 7 ? &op.c_t4ns
                  : which == 4 ? (ref ? &op.jinv_ref : &op.jinv_cur) : (ref ? &op.jxw_ref : &op.jxw_cur);
    if (out) std::memcpy(out, v->data(), v->size() * sizeof((*v)[0]));
    return (long)v->size();
  };
  return h->fp32 ? get(h->of) : get(h->od);
}

double orc_residual(void *mh, const double *mu, double nu, int formulation, const double *u,
                    int n_neu, const int *neu_ids, const double *neu_ab, double time,
                    const unsigned char *cmask, double *R) {
  auto *h = (MeshH *)mh;
  std::vector<double> m(mu, mu + h->m.n_cells);
  std::vector<Neumann> neu;
  for (int i = 0; i < n_neu; ++i) {
    Neumann nm; nm.id = neu_ids[i];
    for (int c = 0; c < 3; ++c) { nm.a[c] = neu_ab[6 * i + c]; nm.b[c] = neu_ab[6 * i + 3 + c]; }
    neu.push_back(nm);
  }
  std::vector<uint8_t> cm(cmask, cmask + h->m.n_dofs());
  return residual(h->m, h->b, m, nu, formulation, u, neu, time, cm, R);
}

void orc_element_matrix(void *mh, int cell, double mu, double nu, int formulation, const double *u, double *K) {
  auto *h = (MeshH *)mh;
  Material mat(mu, nu, formulation);
  std::vector<double> k;
  element_matrix(h->m, h->b, cell, mat, u, k);
  std::memcpy(K, k.data(), sizeof(double) * k.size());
}

// Matrix-based tangent of the whole mesh (assemble_system's tangent part,
// mf_elasticity.h:2760-2843, through the FEValues-style element matrices)
// as COO triplets: slot range [cell * ND^2, (cell + 1) * ND^2) holds cell's
// entries, with row = -1 where a constrained row or column is dropped; then
// one unit diagonal entry per constrained dof (AffineConstraints keep the
// constrained rows and columns of the system matrix as an identity block,
// which is what the matrix-free operator applies).  Returns the slot count;
// with rows == nullptr only the count.
long orc_assemble_coo(void *mh, const double *mu_cell, double nu, int formulation, const double *u,
                      const unsigned char *cmask, int *rows, int *cols, double *vals) {
  auto *h = (MeshH *)mh;
  const Mesh &m = h->m;
  const int NN = m.ncn(), ND = 3 * NN;
  long n_con = 0;
  for (int i = 0; i < m.n_dofs(); ++i) n_con += cmask[i] ? 1 : 0;
  const long total = (long)m.n_cells * ND * ND + n_con;
  if (!rows) return total;
#pragma omp parallel for schedule(dynamic, 4)
  for (int cell = 0; cell < m.n_cells; ++cell) {
    std::vector<double> K;
    element_matrix(m, h->b, cell, Material(mu_cell[cell], nu, formulation), u, K);
    const int *nodes = &m.cell_nodes[(size_t)cell * NN];
    const long base = (long)cell * ND * ND;
    for (int i = 0; i < ND; ++i) {
      const int gi = 3 * nodes[i % NN] + i / NN;
      for (int j = 0; j < ND; ++j) {
        const int gj = 3 * nodes[j % NN] + j / NN;
        const long s = base + (long)i * ND + j;
        const bool keep = !cmask[gi] && !cmask[gj];
        rows[s] = keep ? gi : -1;
        cols[s] = gj;
        vals[s] = K[(size_t)i * ND + j];
      }
    }
  }
  long s = (long)m.n_cells * ND * ND;
  for (int i = 0; i < m.n_dofs(); ++i)
    if (cmask[i]) { rows[s] = i; cols[s] = i; vals[s] = 1.0; ++s; }
  return total;
}

// ------------------------------------------------------------ transfer
struct TrH { Transfer t; MeshH *c, *f; };
void *orc_transfer_new(void *coarse, void *fine) {
  auto *h = new TrH(); h->c = (MeshH *)coarse; h->f = (MeshH *)fine;
  h->t.build(h->c->m, h->f->m, h->c->b);
  return h;
}
void orc_transfer_free(void *h) { delete (TrH *)h; }
void orc_transfer_prolongate(void *hh, const unsigned char *ccmask, const double *src, double *dst) {
  auto *h = (TrH *)hh;
  std::vector<uint8_t> cm(ccmask, ccmask + h->c->m.n_dofs());
  std::memset(dst, 0, sizeof(double) * h->f->m.n_dofs());
  h->t.prolongate_add(h->c->m, cm, src, dst);
}
void orc_transfer_restrict(void *hh, const unsigned char *ccmask, const double *src, double *dst) {
  auto *h = (TrH *)hh;
  std::vector<uint8_t> cm(ccmask, ccmask + h->c->m.n_dofs());
  std::memset(dst, 0, sizeof(double) * h->c->m.n_dofs());
  h->t.restrict_add(h->c->m, cm, src, dst);
}
void orc_transfer_interpolate(void *hh, const double *fine_u, double *coarse_u) {
  auto *h = (TrH *)hh;
  h->t.interpolate(h->c->m, h->f->m, fine_u, coarse_u);
}

// ---------------------------------------------------------------- GMG
struct GmgH {
  NewtonParams prm;
  Basis1D bas;
  std::vector<Mesh> meshes;
  std::vector<std::vector<uint8_t>> lmask;
  std::vector<std::vector<double>> lmu;
  GMG<float> gf;
  GMG<double> gd;
  bool fp32;
};
// mesh description as for orc_mesh_new (levels 0..n_refinements), Dirichlet
// specs, fine per-cell mu, fine displacement u; Chebyshev parameters
void *orc_gmg_new(int geom, const int *coarse, int nref, const double *lo, const double *hi, double scale, int p,
                  int q, int caching, int formulation, int fp32, const double *mu_fine, double nu, int n_dir,
                  const int *dir_ids, const int *dir_masks, const double *u, int degree, double range, int eig_its,
                  int coarse_cheb, int coarse_accurate, const uint8_t *coarse_active) {
  try {
    auto *h = new GmgH();
    NewtonParams &P = h->prm;
    P.mesh.geometry = geom; P.mesh.n_refinements = nref; P.mesh.scale = scale; P.mesh.p = p; P.mesh.q = q;
    for (int k = 0; k < 3; ++k) { P.mesh.coarse[k] = coarse[k]; P.mesh.lo[k] = lo[k]; P.mesh.hi[k] = hi[k]; }
    if (coarse_active)
      P.mesh.coarse_active.assign(coarse_active, coarse_active + (size_t)coarse[0] * coarse[1] * coarse[2]);
    P.caching = caching; P.formulation = formulation; P.nu = nu;
    P.cheb_degree = degree; P.smoothing_range = range; P.cheb_eig_its = eig_its;
    P.coarse_chebyshev = coarse_cheb; P.coarse_accurate_eig = coarse_accurate;
    for (int i = 0; i < n_dir; ++i) P.dirichlet.push_back({dir_ids[i], dir_masks[i]});
    h->bas.init(p, q);
    const int nl = nref + 1;
    h->meshes.resize(nl);
    for (int l = 0; l < nl; ++l) build_mesh(P.mesh, l, h->meshes[l]);
    h->lmask.resize(nl);
    for (int l = 0; l < nl; ++l) constrained_dofs(h->meshes[l], P.dirichlet, h->lmask[l]);
    std::vector<double> muf(mu_fine, mu_fine + h->meshes.back().n_cells);
    h->lmu.resize(nl);
    for (int l = 0; l < nl; ++l) h->lmu[l] = coarsen_cell_field(h->meshes, l, muf);
    std::vector<double> uf(u, u + h->meshes.back().n_dofs());
    h->fp32 = fp32 != 0;
    if (h->fp32) setup_gmg<float>(P, h->meshes, h->bas, h->lmask, h->lmu, uf, h->gf, true);
    else setup_gmg<double>(P, h->meshes, h->bas, h->lmask, h->lmu, uf, h->gd, true);
    return h;
  } catch (std::exception &e) { g_err = e.what(); return nullptr; }
}
void orc_gmg_free(void *h) { delete (GmgH *)h; }
void orc_gmg_vmult(void *hh, double *dst, const double *src) {
  auto *h = (GmgH *)hh;
  const size_t n = h->meshes.back().n_dofs();
  std::vector<double> s(src, src + n), d(n);
  if (h->fp32) h->gf.vmult(d, s); else h->gd.vmult(d, s);
  std::memcpy(dst, d.data(), n * sizeof(double));
}
void orc_gmg_level_info(void *hh, int l, double *out6) {
  auto *h = (GmgH *)hh;
  auto get = [&](auto &g) {
    const auto &c = g.levels[l].cheb;
    out6[0] = c.eig_min; out6[1] = c.eig_max; out6[2] = c.degree; out6[3] = c.theta; out6[4] = c.delta; out6[5] = 0;
  };
  if (h->fp32) get(h->gf); else get(h->gd);
}

// ------------------------------------------------------------- Newton
// Flat parameter block (doubles then ints) so that ctypes can fill it.
struct orc_newton_params {
  double lo[3], hi[3], scale, mu, nu, end_time, dt, tol_f, tol_u, tol_f_abs, tol_u_abs, tol_lin,
      relaxation, smoothing_range, output_point[3];
  int geometry, coarse[3], n_refinements, p, q, caching, formulation, max_nr, max_it_mult, precond,
      cheb_degree, cheb_eig_its, coarse_chebyshev, coarse_accurate_eig, level_fp32, has_output_point,
      n_dirichlet, n_neumann;
  int dir_ids[8], dir_masks[8];
  double dir_values[24];
  int neu_ids[8];
  double neu_ab[48];
};

static NewtonParams to_params(const orc_newton_params *P, const uint8_t *coarse_active) {
  NewtonParams prm;
  prm.mesh.geometry = P->geometry;
  if (coarse_active)
    prm.mesh.coarse_active.assign(coarse_active, coarse_active + (size_t)P->coarse[0] * P->coarse[1] * P->coarse[2]);
  for (int k = 0; k < 3; ++k) { prm.mesh.coarse[k] = P->coarse[k]; prm.mesh.lo[k] = P->lo[k]; prm.mesh.hi[k] = P->hi[k]; }
  prm.mesh.n_refinements = P->n_refinements; prm.mesh.scale = P->scale;
  prm.mesh.p = P->p; prm.mesh.q = P->q;
  prm.caching = P->caching; prm.formulation = P->formulation;
  prm.mu = P->mu; prm.nu = P->nu;
  prm.end_time = P->end_time; prm.dt = P->dt; prm.max_nr = P->max_nr;
  prm.tol_f = P->tol_f; prm.tol_u = P->tol_u; prm.tol_f_abs = P->tol_f_abs; prm.tol_u_abs = P->tol_u_abs;
  prm.tol_lin = P->tol_lin; prm.max_it_mult = P->max_it_mult; prm.precond = P->precond;
  prm.relaxation = P->relaxation; prm.cheb_degree = P->cheb_degree; prm.cheb_eig_its = P->cheb_eig_its;
  prm.smoothing_range = P->smoothing_range;
  prm.coarse_chebyshev = P->coarse_chebyshev; prm.coarse_accurate_eig = P->coarse_accurate_eig;
  prm.level_fp32 = P->level_fp32; prm.has_output_point = P->has_output_point;
  for (int k = 0; k < 3; ++k) prm.output_point[k] = P->output_point[k];
  for (int i = 0; i < P->n_dirichlet; ++i) {
    prm.dirichlet.push_back({P->dir_ids[i], P->dir_masks[i]});
    prm.dirichlet_value.push_back({P->dir_values[3 * i], P->dir_values[3 * i + 1], P->dir_values[3 * i + 2]});
  }
  for (int i = 0; i < P->n_neumann; ++i) {
    Neumann nm; nm.id = P->neu_ids[i];
    for (int c = 0; c < 3; ++c) { nm.a[c] = P->neu_ab[6 * i + c]; nm.b[c] = P->neu_ab[6 * i + 3 + c]; }
    prm.neumann.push_back(nm);
  }
  return prm;
}

// out_steps: per step [time, newton_its, converged, u0, u1, u2, total_cg_its]
// coarse_active (optional, coarse[0]*coarse[1]*coarse[2] bytes, x fastest):
// coarse cells removed from the mesh (the voids geometry)
int orc_newton(const orc_newton_params *P, const double *mu_fine, int *n_cells, int *n_dofs,
               double *volume, int max_steps, double *out_steps, int *n_steps, double *u_out,
               int *cg_its_out, int max_cg_entries, const uint8_t *coarse_active, double *hist_out,
               int max_hist_entries) {
  try {
    NewtonParams prm = to_params(P, coarse_active);
    NewtonResult res;
    if (mu_fine) {
      Mesh tmp; build_mesh(prm.mesh, prm.mesh.n_refinements, tmp);
      prm.mu_fine.assign(mu_fine, mu_fine + tmp.n_cells);
    }
    int rc = newton_run(prm, res);
    *n_cells = res.n_cells; *n_dofs = res.n_dofs; *volume = res.volume;
    *n_steps = (int)res.steps.size();
    int cgk = 0, hk = 0;
    for (int s = 0; s < (int)res.steps.size() && s < max_steps; ++s) {
      const auto &st = res.steps[s];
      double *o = out_steps + 7 * s;
      o[0] = st.time; o[1] = st.newton_iterations; o[2] = st.converged;
      o[3] = st.point_u[0]; o[4] = st.point_u[1]; o[5] = st.point_u[2];
      int tot = 0;
      for (int c : st.cg_iterations) { tot += c; if (cg_its_out && cgk < max_cg_entries) cg_its_out[cgk++] = c; }
      // hist_out: per load step and Newton iteration (step, rel_res, rel_upd)
      for (size_t k = 0; k < st.rel_res.size(); ++k)
        if (hist_out && hk < max_hist_entries) {
          hist_out[3 * hk] = s; hist_out[3 * hk + 1] = st.rel_res[k]; hist_out[3 * hk + 2] = st.rel_upd[k];
          ++hk;
        }
      o[6] = tot;
    }
    if (u_out && !res.u.empty()) std::memcpy(u_out, res.u.data(), sizeof(double) * res.u.size());
    return rc;
  } catch (std::exception &e) { g_err = e.what(); return -1; }
}

// Adjoint gradient (see adjoint_run): log_mu per fine cell, u_target per dof;
// outputs J, grad (per fine cell) and the converged displacement.
int orc_adjoint(const orc_newton_params *P, const uint8_t *coarse_active, const double *log_mu, const double *u_target,
                int obj_id, double *J, double *grad, double *u_out) {
  try {
    NewtonParams prm = to_params(P, coarse_active);
    Mesh m; build_mesh(prm.mesh, prm.mesh.n_refinements, m);
    std::vector<double> lm(log_mu, log_mu + m.n_cells), tg(u_target, u_target + m.n_dofs()), g, u;
    const int rc = adjoint_run(prm, lm, tg, obj_id, *J, g, u);
    if (rc) return rc;
    std::memcpy(grad, g.data(), sizeof(double) * g.size());
    if (u_out) std::memcpy(u_out, u.data(), sizeof(double) * u.size());
    return 0;
  } catch (std::exception &e) { g_err = e.what(); return -1; }
}

}  // extern "C"
