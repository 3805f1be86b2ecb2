// CPU oracle (test infrastructure only): NeoHookOperator restatement.
// Sum factorisation on each cell (deal.II FEEvaluation evaluate/integrate),
// quadrature-point physics of mf_nh_operator.h:922-1499, and the cache of
// mf_nh_operator.h:447-592.  OpenMP over cells with an 8-colour partition of
// the structured mesh, so that scatter-adds never race.
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "oracle.h"
#include "oracle_cell.h"

namespace orc {

template <typename Number>
void Operator<Number>::initialize(const Mesh *m, const Basis1D *b, int caching_,
                                  int formulation_) {
  // mf_nh_operator.h:394-443: choose the caching variant, size the tables.
  mesh = m; basis = b; caching = caching_; formulation = formulation_;
  if (caching < 0 || caching > CACHE_TENSOR4_NS)
    throw std::runtime_error("Unknown caching");  // :441
  if (formulation == 0 && caching != CACHE_SCALAR)
    throw std::runtime_error("formulation 0 needs scalar caching");
  const size_t nqt = (size_t)m->n_cells * nq();
  c_scalar.clear(); c_second.clear(); c_t2.clear(); c_t4.clear(); c_t4ns.clear();
  if (caching == CACHE_SCALAR) c_scalar.resize(nqt);
  // scalar_referential: c and the displacement at the points (:512-534)
  if (caching == CACHE_SCALAR_REFERENTIAL) { c_scalar.resize(nqt); c_second.resize(3 * nqt); }
  // tensor4_ns: dP/dF (81 per point, :563-582)
  if (caching == CACHE_TENSOR4_NS) c_t4ns.resize(81 * nqt);
  if (caching == CACHE_TENSOR2) { c_scalar.resize(nqt); c_second.resize(nqt); c_t2.resize(6 * nqt); }
  if (caching == CACHE_TENSOR4) { c_t2.resize(6 * nqt); c_t4.resize(36 * nqt); }
  jinv_cur.resize(9 * nqt); jxw_cur.resize(nqt);
  jinv_ref.resize(9 * nqt); jxw_ref.resize(nqt);
  mu_cell.assign(m->n_cells, 1.0);
  cmask.assign(m->n_dofs(), 0);
  constrained.clear();
}

template <typename Number>
void Operator<Number>::set_material(const std::vector<double> &mu, double nu_) {
  mu_cell = mu; nu = nu_;
}

template <typename Number>
void Operator<Number>::set_constraints(const std::vector<uint8_t> &mask) {
  cmask = mask;
  constrained.clear();
  for (size_t i = 0; i < mask.size(); ++i)
    if (mask[i]) constrained.push_back((int)i);
}

template <typename Number>
int Operator<Number>::cache(const Number *disp) {
  u.assign(disp, disp + mesh->n_dofs());
  int bad = 0;
  DISPATCH_PQ(mesh->p, basis->q, {
    bad = CellOps<P_, Q_, Number>::cache_all(*this);
  });
  return bad;
}

template <typename Number>
void Operator<Number>::vmult(Number *dst, const Number *src) const {
  // vmult = zero dst, then vmult_add (mf_nh_operator.h:612-622, :649-706)
  std::memset(dst, 0, sizeof(Number) * mesh->n_dofs());
  DISPATCH_PQ(mesh->p, basis->q, {
    CellOps<P_, Q_, Number>::apply_all(*this, dst, src);
  });
  // constrained dofs: dst += src (:702-705)
  for (int dof : constrained) dst[dof] += src[dof];
}

template <typename Number>
void Operator<Number>::apply_inhomogeneous(Number *dst, const Number *g) const {
  std::memset(dst, 0, sizeof(Number) * mesh->n_dofs());
  DISPATCH_PQ(mesh->p, basis->q, {
    CellOps<P_, Q_, Number>::apply_all(*this, dst, g, false);
  });
}

template <typename Number>
void Operator<Number>::cell_apply(int cell, const Number *in, Number *out) const {
  DISPATCH_PQ(mesh->p, basis->q, {
    CellOps<P_, Q_, Number>::cell_apply(*this, cell, in, out);
  });
}

template <typename Number>
void Operator<Number>::compute_diagonal() {
  // mf_nh_operator.h:789-918 (unit-vector trick per cell, constrained
  // entries skipped by distribute_local_to_global), :1503-1557 (constrained
  // entries set to one, then inverted).
  const int n = mesh->n_dofs();
  diag.assign(n, Number(0));
  DISPATCH_PQ(mesh->p, basis->q, {
    CellOps<P_, Q_, Number>::diagonal_all(*this, diag.data());
  });
  for (int dof : constrained) diag[dof] = Number(1);
  inv_diag.resize(n);
  for (int i = 0; i < n; ++i) inv_diag[i] = Number(1) / diag[i];
}

template struct Operator<double>;
template struct Operator<float>;

}  // namespace orc
