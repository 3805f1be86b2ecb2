// Host side of the mesh hierarchy: 1D basis, structured hexahedral levels,
// boundary ids, Dirichlet masks, inter-level transfer maps, device upload.
//
// Replaces, for the structured meshes of this path, deal.II's Triangulation /
// DoFHandler / MGConstrainedDoFs set-up done by Solid::make_grid and
// Solid::system_setup (mf_elasticity.h:1339-1708, 2932-3007).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "lsmf_internal.h"

namespace lsmf {

static void legendre(int n, double x, double &P, double &dP) {
  double p0 = 1.0, p1 = x;
  if (n == 0) { P = 1.0; dP = 0.0; return; }
  for (int k = 2; k <= n; ++k) {
    const double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1; p1 = pk;
  }
  P = p1;
  dP = n * (x * p1 - p0) / (x * x - 1.0);
}

void Basis::eval(double x, double *val, double *der) const {
  const int n = p + 1;
  for (int i = 0; i < n; ++i) {
    double v = 1.0, d = 0.0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const double inv = 1.0 / (nodes[i] - nodes[j]);
      d = d * (x - nodes[j]) * inv + v * inv;
      v *= (x - nodes[j]) * inv;
    }
    if (val) val[i] = v;
    if (der) der[i] = d;
  }
}

// QGauss (Gauss-Legendre) points/weights and FE_Q Gauss-Lobatto nodes on [0,1]
void Basis::init(int p_, int q_) {
  p = p_; q = q_;
  qpts.assign(q, 0.0); qw.assign(q, 0.0);
  for (int i = 0; i < q; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (q + 0.5));
    for (int it = 0; it < 100; ++it) {
      double P, dP; legendre(q, z, P, dP);
      const double dz = P / dP; z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double P, dP; legendre(q, z, P, dP);
    qpts[q - 1 - i] = 0.5 * (1.0 + z);
    qw[q - 1 - i] = 1.0 / ((1.0 - z * z) * dP * dP);
  }
  nodes.assign(p + 1, 0.0);
  nodes[p] = 1.0;
  for (int i = 1; i < p; ++i) {
    double z = -std::cos(M_PI * i / p);
    for (int it = 0; it < 100; ++it) {
      double P, dP; legendre(p, z, P, dP);
      const double d2P = (2.0 * z * dP - p * (p + 1.0) * P) / (1.0 - z * z);
      const double dz = dP / d2P; z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    nodes[i] = 0.5 * (1.0 + z);
  }
  if (p % 2 == 0 && p > 0) nodes[p / 2] = 0.5;
  N.assign(q * (p + 1), 0.0); D.assign(q * (p + 1), 0.0);
  for (int k = 0; k < q; ++k) eval(qpts[k], &N[k * (p + 1)], &D[k * (p + 1)]);
  // collocation derivative: Dc[k][m] = l_m'(x_k) for the Lagrange basis l_m on
  // the quadrature points (l_m'(x_m) = sum_{j != m} 1 / (x_m - x_j))
  Dc.assign(q * q, 0.0);
  for (int k = 0; k < q; ++k)
    for (int m = 0; m < q; ++m) {
      if (k == m) {
        double s = 0.0;
        for (int j = 0; j < q; ++j)
          if (j != m) s += 1.0 / (qpts[m] - qpts[j]);
        Dc[k * q + m] = s;
      } else {
        double num = 1.0, den = 1.0;
        for (int j = 0; j < q; ++j) {
          if (j != m) den *= qpts[m] - qpts[j];
          if (j != m && j != k) num *= qpts[k] - qpts[j];
        }
        Dc[k * q + m] = num / den;
      }
    }
}

namespace {

// grid_y_transform of mf_elasticity.h:1251-1270
void cook_transform(double &x, double &y) {
  const double y_upper = 44.0 + (16.0 / 48.0) * x;
  const double y_lower = (44.0 / 48.0) * x;
  const double theta = y / 44.0;
  y = (1 - theta) * y_lower + theta * y_upper;
}

void build_level(const lsmf_mesh &M, int level, Level &L) {
  const lsmf_mesh_desc &d = M.desc;
  const int p = d.degree;
  L.p = p; L.q = d.n_q_points_1d;
  // axis-aligned box cells have a constant reference Jacobian; the Cook
  // transformation bends them
  L.affine = d.geometry == LSMF_GEOM_BOX;
  for (int k = 0; k < 3; ++k) { L.nc[k] = d.coarse[k] << level; L.nn[k] = p * L.nc[k] + 1; }
  const int ncx = L.nc[0], ncy = L.nc[1], ncz = L.nc[2];
  // active: a cell of the whole mesh; member: a cell of this mesh (of its
  // z-slab when the mesh is one part of a partition).  Faces between two
  // active cells are interior, also across a partition interface.
  auto active = [&](int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= ncx || j >= ncy || k >= ncz) return false;
    if (M.coarse_active.empty()) return true;
    const int ci = i >> level, cj = j >> level, ck = k >> level;
    return M.coarse_active[(size_t)(ck * d.coarse[1] + cj) * d.coarse[0] + ci] != 0;
  };
  auto member = [&](int i, int j, int k) {
    if (!active(i, j, k)) return false;
    if (M.layout.n_parts <= 1) return true;
    const int ck = k >> level;
    return ck >= M.layout.k0 && ck < M.layout.k1;
  };
  const size_t nlat = (size_t)L.nn[0] * L.nn[1] * L.nn[2];
  L.lattice_to_node.assign(nlat, -1);
  L.cell_of_lattice.assign((size_t)ncx * ncy * ncz, -1);
  for (int k = 0; k < ncz; ++k)
    for (int j = 0; j < ncy; ++j)
      for (int i = 0; i < ncx; ++i) {
        if (!member(i, j, k)) continue;
        L.cell_of_lattice[((size_t)k * ncy + j) * ncx + i] = L.n_cells++;
        L.cell_ijk.insert(L.cell_ijk.end(), {i, j, k});
        for (int c = 0; c <= p; ++c)
          for (int b = 0; b <= p; ++b)
            for (int a = 0; a <= p; ++a)
              L.lattice_to_node[((size_t)(k * p + c) * L.nn[1] + (j * p + b)) * L.nn[0] + (i * p + a)] = 0;
      }
  for (size_t l = 0; l < nlat; ++l)
    if (L.lattice_to_node[l] == 0) {
      L.lattice_to_node[l] = L.n_nodes++;
      L.node_lattice.push_back((int)l);
    }
  L.X.resize(3 * (size_t)L.n_nodes);
  for (int n = 0; n < L.n_nodes; ++n) {
    const size_t l = L.node_lattice[n];
    const int lat[3] = {(int)(l % L.nn[0]), (int)((l / L.nn[0]) % L.nn[1]), (int)(l / ((size_t)L.nn[0] * L.nn[1]))};
    double x[3];
    for (int dd = 0; dd < 3; ++dd) {
      int cell; double xi;
      if (lat[dd] == L.nn[dd] - 1) { cell = L.nc[dd] - 1; xi = 1.0; }
      else { cell = lat[dd] / p; xi = M.basis.nodes[lat[dd] % p]; }
      x[dd] = d.lo[dd] + (d.hi[dd] - d.lo[dd]) * ((cell + xi) / L.nc[dd]);
    }
    if (d.geometry == LSMF_GEOM_COOK) cook_transform(x[0], x[1]);
    for (int dd = 0; dd < 3; ++dd) L.X[3 * (size_t)n + dd] = x[dd] * d.scale;
  }
  const int ncn = L.ncn();
  L.cell_nodes.resize((size_t)L.n_cells * ncn);
  for (int cell = 0; cell < L.n_cells; ++cell) {
    const int i = L.cell_ijk[3 * cell], j = L.cell_ijk[3 * cell + 1], k = L.cell_ijk[3 * cell + 2];
    int idx = 0;
    for (int c = 0; c <= p; ++c)
      for (int b = 0; b <= p; ++b)
        for (int a = 0; a <= p; ++a)
          L.cell_nodes[(size_t)cell * ncn + idx++] =
              L.lattice_to_node[((size_t)(k * p + c) * L.nn[1] + (j * p + b)) * L.nn[0] + (i * p + a)];
  }
  static const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
  for (int cell = 0; cell < L.n_cells; ++cell) {
    const int i = L.cell_ijk[3 * cell], j = L.cell_ijk[3 * cell + 1], k = L.cell_ijk[3 * cell + 2];
    for (int f = 0; f < 6; ++f) {
      const int ni = i + off[f][0], nj = j + off[f][1], nk = k + off[f][2];
      if (active(ni, nj, nk)) continue;
      const bool outer = ni < 0 || nj < 0 || nk < 0 || ni >= ncx || nj >= ncy || nk >= ncz;
      int id;
      if (d.geometry == LSMF_GEOM_COOK) id = outer ? (f == 0 ? 1 : (f == 1 ? 11 : 0)) : 6;
      else id = outer ? f : 6;
      L.bfaces.insert(L.bfaces.end(), {cell, f, id});
    }
  }
}

void face_nodes(int p, int f, std::vector<int> &out) {
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

}  // namespace

lsmf_status level_constraints(const lsmf_mesh &M, Level &L) {
  L.cmask.assign((size_t)L.n_dofs(), 0);
  std::vector<int> fl;
  const int ncn = L.ncn();
  for (size_t t = 0; t < L.bfaces.size(); t += 3) {
    const int cell = L.bfaces[t], f = L.bfaces[t + 1], id = L.bfaces[t + 2];
    for (size_t s = 0; s < M.dir_ids.size(); ++s) {
      if (M.dir_ids[s] != id) continue;
      face_nodes(L.p, f, fl);
      for (int ln : fl) {
        const int node = L.cell_nodes[(size_t)cell * ncn + ln];
        for (int c = 0; c < 3; ++c)
          if (M.dir_masks[s] & (1 << c)) L.cmask[3 * (size_t)node + c] = 1;
      }
    }
  }
  L.constrained.clear();
  for (size_t i = 0; i < L.cmask.size(); ++i)
    if (L.cmask[i]) L.constrained.push_back((int)i);
  std::vector<int> packed(L.cell_nodes.size());
  for (size_t i = 0; i < packed.size(); ++i) {
    const int node = L.cell_nodes[i];
    const int cm = L.cmask[3 * (size_t)node] | (L.cmask[3 * (size_t)node + 1] << 1) | (L.cmask[3 * (size_t)node + 2] << 2);
    packed[i] = node | (cm << NODE_BITS);
  }
  LSMF_TRY(L.d_cell_nodes.upload(packed.data(), packed.size()));
  LSMF_TRY(L.d_constrained.upload(L.constrained.data(), L.constrained.size()));
  LSMF_TRY(L.d_cmask.upload(L.cmask.data(), L.cmask.size()));
  return LSMF_OK;
}

// Transfer maps between level l-1 and l (MGTransferMatrixFree semantics:
// cell-wise embedding, multiplicity weights, coarse Dirichlet zeroed).
static lsmf_status build_transfer(const lsmf_mesh &M, const Level &C, const Level &F, TransferMap &T) {
  const int p = C.p, n1 = p + 1, nf1 = 2 * p + 1, nfb = nf1 * nf1 * nf1;
  T.P1.assign((size_t)nf1 * n1, 0.0);
  for (int f = 0; f < nf1; ++f) {
    int child = f / p, loc = f - child * p;
    if (child > 1) { child = 1; loc = p; }
    const double xi = 0.5 * (child + (loc == p ? 1.0 : M.basis.nodes[loc]));
    M.basis.eval(xi, &T.P1[f * n1], nullptr);
  }
  T.fine_nodes.resize((size_t)C.n_cells * nfb);
  std::vector<int> mult(F.n_nodes, 0);
  for (int c = 0; c < C.n_cells; ++c) {
    const int i = C.cell_ijk[3 * c], j = C.cell_ijk[3 * c + 1], k = C.cell_ijk[3 * c + 2];
    int idx = 0;
    for (int fz = 0; fz < nf1; ++fz)
      for (int fy = 0; fy < nf1; ++fy)
        for (int fx = 0; fx < nf1; ++fx) {
          const int node = F.lattice_to_node[((size_t)(2 * k * p + fz) * F.nn[1] + (2 * j * p + fy)) * F.nn[0] +
                                             (2 * i * p + fx)];
          T.fine_nodes[(size_t)c * nfb + idx++] = node;
          mult[node]++;
        }
  }
  T.weight.resize(F.n_nodes);
  for (int n = 0; n < F.n_nodes; ++n) T.weight[n] = mult[n] ? 1.0 / mult[n] : 0.0;
  LSMF_TRY(T.d_fine_nodes.upload(T.fine_nodes.data(), T.fine_nodes.size()));
  LSMF_TRY(T.d_weight.upload(T.weight.data(), T.weight.size()));
  // interpolation of the fine displacement at the coarse nodes: each coarse
  // node is evaluated in one fine cell containing it (interpolate_to_mg)
  std::vector<int> icell(C.n_nodes, -1);
  std::vector<double> iw((size_t)C.n_nodes * C.ncn(), 0.0);
  const int ncn = C.ncn();
  std::vector<double> vx(n1), vy(n1), vz(n1);
  for (int c = 0; c < C.n_cells; ++c) {
    const int ci[3] = {C.cell_ijk[3 * c], C.cell_ijk[3 * c + 1], C.cell_ijk[3 * c + 2]};
    for (int lz = 0; lz < n1; ++lz)
      for (int ly = 0; ly < n1; ++ly)
        for (int lx = 0; lx < n1; ++lx) {
          const int cnode = C.cell_nodes[(size_t)c * ncn + (lz * n1 + ly) * n1 + lx];
          if (icell[cnode] >= 0) continue;
          const int li[3] = {lx, ly, lz};
          int child[3]; double xf[3];
          for (int dd = 0; dd < 3; ++dd) {
            const double s = 2.0 * M.basis.nodes[li[dd]];
            child[dd] = std::min(1, (int)std::floor(s));
            xf[dd] = s - child[dd];
          }
          const int fi = 2 * ci[0] + child[0], fj = 2 * ci[1] + child[1], fk = 2 * ci[2] + child[2];
          icell[cnode] = F.cell_of_lattice[((size_t)fk * F.nc[1] + fj) * F.nc[0] + fi];
          M.basis.eval(xf[0], vx.data(), nullptr);
          M.basis.eval(xf[1], vy.data(), nullptr);
          M.basis.eval(xf[2], vz.data(), nullptr);
          for (int z = 0; z < n1; ++z)
            for (int y = 0; y < n1; ++y)
              for (int x = 0; x < n1; ++x) iw[(size_t)cnode * ncn + (z * n1 + y) * n1 + x] = vx[x] * vy[y] * vz[z];
        }
  }
  T.interp_fine_cell = icell;
  LSMF_TRY(T.d_interp_cell.upload(icell.data(), icell.size()));
  LSMF_TRY(T.d_interp_w.upload(iw.data(), iw.size()));
  return LSMF_OK;
}

// Global node numbers and interface lists of a z-slab part on the finest
// level L (see PartLayout).  A lattice point is a node of the whole mesh when
// an active cell touches it; the whole mesh numbers its nodes in lattice
// order, so a prefix count over the lattice gives the global numbers.
static void build_layout(lsmf_mesh &M, const Level &L, int level) {
  PartLayout &P = M.layout;
  const lsmf_mesh_desc &d = M.desc;
  const int p = L.p, ncx = L.nc[0], ncy = L.nc[1], ncz = L.nc[2];
  auto active = [&](int i, int j, int k) {
    if (i < 0 || j < 0 || k < 0 || i >= ncx || j >= ncy || k >= ncz) return false;
    if (M.coarse_active.empty()) return true;
    return M.coarse_active[(size_t)((k >> level) * d.coarse[1] + (j >> level)) * d.coarse[0] + (i >> level)] != 0;
  };
  // cells of layer k touching lattice point (a, b) of a z-plane
  auto touches_layer = [&](int a, int b, int k) {
    const int ia[2] = {a % p == 0 ? a / p - 1 : a / p, a / p};
    const int jb[2] = {b % p == 0 ? b / p - 1 : b / p, b / p};
    for (int s = 0; s < 2; ++s)
      for (int t = 0; t < 2; ++t)
        if (active(ia[s], jb[t], k)) return true;
    return false;
  };
  const size_t nlat = (size_t)L.nn[0] * L.nn[1] * L.nn[2];
  std::vector<int> gnum(nlat, -1);
  int g = 0;
  const size_t plane = (size_t)L.nn[0] * L.nn[1];
  for (size_t l = 0; l < nlat; ++l) {
    const int a = (int)(l % L.nn[0]), b = (int)((l / L.nn[0]) % L.nn[1]), c = (int)(l / plane);
    const int ks[2] = {c % p == 0 ? c / p - 1 : c / p, c / p};
    if (touches_layer(a, b, ks[0]) || (ks[1] != ks[0] && touches_layer(a, b, ks[1]))) gnum[l] = g++;
  }
  P.n_global_nodes = g;
  P.global_node.resize(L.n_nodes);
  P.lower_shared.clear();
  P.upper_shared.clear();
  const int zlo = P.k0 * (1 << level) * p, zhi = P.k1 * (1 << level) * p;
  for (int n = 0; n < L.n_nodes; ++n) {
    const size_t l = L.node_lattice[n];
    P.global_node[n] = gnum[l];
    const int a = (int)(l % L.nn[0]), b = (int)((l / L.nn[0]) % L.nn[1]), c = (int)(l / plane);
    if (P.part > 0 && c == zlo && touches_layer(a, b, zlo / p - 1)) P.lower_shared.push_back(n);
    if (P.part < P.n_parts - 1 && c == zhi && touches_layer(a, b, zhi / p)) P.upper_shared.push_back(n);
  }
}

lsmf_status build_mesh(lsmf_mesh &M) {
  const lsmf_mesh_desc &d = M.desc;
  if (d.degree < 1 || d.degree > 4 || d.n_q_points_1d != d.degree + 1) {
    set_error("supported elements: degree 1..4 with n_q_points_1d = degree + 1");
    return LSMF_ERR_UNSUPPORTED;
  }
  for (int k = 0; k < 3; ++k)
    if (d.coarse[k] < 1 || d.hi[k] <= d.lo[k]) { set_error("bad mesh extents"); return LSMF_ERR_INVALID_ARG; }
  if (d.n_refinements < 0 || d.n_refinements > 12) { set_error("bad n_refinements"); return LSMF_ERR_INVALID_ARG; }
  M.basis.init(d.degree, d.n_q_points_1d);
  const int nl = d.n_refinements + 1;
  for (int l = 0; l < nl; ++l) {
    Level *L = new Level();
    M.levels.push_back(L);
    build_level(M, l, *L);
    if ((long long)L->n_nodes >= (1LL << NODE_BITS)) { set_error("too many nodes"); return LSMF_ERR_UNSUPPORTED; }
    if (M.host_only) continue;
    LSMF_TRY(L->d_X.upload(L->X.data(), L->X.size()));
    LSMF_TRY(level_constraints(M, *L));
    // cells by lattice colour: two cells of one colour are two or more
    // lattice steps apart in some direction, so they share no node
    L->colour_cells.clear();
    for (int c = 0; c < 8; ++c) {
      L->colour_off[c] = (int)L->colour_cells.size();
      for (int e = 0; e < L->n_cells; ++e) {
        const int *ijk = &L->cell_ijk[3 * (size_t)e];
        if ((ijk[0] & 1) + 2 * (ijk[1] & 1) + 4 * (ijk[2] & 1) == c) L->colour_cells.push_back(e);
      }
    }
    L->colour_off[8] = (int)L->colour_cells.size();
    LSMF_TRY(L->d_colour_cells.upload(L->colour_cells.data(), L->colour_cells.size()));
  }
  M.transfer.assign(nl, nullptr);
  for (int l = 1; l < nl && !M.host_only; ++l) {
    M.transfer[l] = new TransferMap();
    LSMF_TRY(build_transfer(M, *M.levels[l - 1], *M.levels[l], *M.transfer[l]));
  }
  if (M.layout.n_parts > 1) build_layout(M, *M.levels[nl - 1], nl - 1);
  return LSMF_OK;
}

}  // namespace lsmf

lsmf_mesh::~lsmf_mesh() {
  for (auto *L : levels) delete L;
  for (auto *T : transfer) delete T;
}
