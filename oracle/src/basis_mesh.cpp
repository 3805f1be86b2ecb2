// CPU oracle (test infrastructure only): 1D basis, structured hex meshes,
// boundary ids and Dirichlet masks.  See oracle.h for the scope statement.
#include <cmath>
#include <stdexcept>

#include "oracle.h"

namespace orc {

// Legendre polynomial P_n and derivative at x in [-1,1].
static void legendre(int n, double x, double &P, double &dP) {
  double p0 = 1.0, p1 = x;
  if (n == 0) { P = 1.0; dP = 0.0; return; }
  for (int k = 2; k <= n; ++k) {
    double pk = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
    p0 = p1; p1 = pk;
  }
  P = p1;
  dP = n * (x * p1 - p0) / (x * x - 1.0);
}

// QGauss<1>(n) mapped to [0,1] (deal.II QGauss: Gauss-Legendre points).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
  x.assign(n, 0.0); w.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double P, dP; legendre(n, z, P, dP);
      double dz = P / dP; z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double P, dP; legendre(n, z, P, dP);
    double wi = 2.0 / ((1.0 - z * z) * dP * dP);
    // ascending order on [0,1]
    x[n - 1 - i] = 0.5 * (1.0 + z);
    w[n - 1 - i] = 0.5 * wi;
  }
}

// Gauss-Lobatto nodes (FE_Q support points): endpoints + roots of P'_{n-1}.
void gauss_lobatto(int n, std::vector<double> &x) {
  x.assign(n, 0.0);
  x[0] = 0.0; x[n - 1] = 1.0;
  const int m = n - 1;
  for (int i = 1; i < m; ++i) {
    double z = -std::cos(M_PI * i / m);
    for (int it = 0; it < 100; ++it) {
      // roots of (1-z^2) P'_m(z): Newton on P'_m using the Legendre ODE
      double P, dP; legendre(m, z, P, dP);
      double d2P = (2.0 * z * dP - m * (m + 1.0) * P) / (1.0 - z * z);
      double dz = dP / d2P; z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = 0.5 * (1.0 + z);
  }
  if (n % 2 == 1) x[n / 2] = 0.5;  // exact midpoint for odd counts
}

void Basis1D::eval(double xx, double *val, double *der) const {
  const int n = p + 1;
  for (int i = 0; i < n; ++i) {
    double v = 1.0, d = 0.0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      double f = (xx - nodes[j]) / (nodes[i] - nodes[j]);
      double df = 1.0 / (nodes[i] - nodes[j]);
      d = d * f + v * df;
      v *= f;
    }
    if (val) val[i] = v;
    if (der) der[i] = d;
  }
}

void Basis1D::init(int p_, int q_) {
  p = p_; q = q_;
  gauss_lobatto(p + 1, nodes);
  gauss_legendre(q, qpts, qw);
  N.assign(q * (p + 1), 0.0); D.assign(q * (p + 1), 0.0);
  for (int k = 0; k < q; ++k) eval(qpts[k], &N[k * (p + 1)], &D[k * (p + 1)]);
}

// ---------------------------------------------------------------- geometry
// grid_y_transform (mf_elasticity.h:1251-1270): bilinear map of the
// 48 x 44 rectangle onto the tapered Cook membrane.
static void cook_transform(double &x, double &y) {
  const double y_upper = 44.0 + (16.0 / 48.0) * x;
  const double y_lower = 0.0 + (44.0 / 48.0) * x;
  const double theta = y / 44.0;
  y = (1 - theta) * y_lower + theta * y_upper;
}

static void lattice_coord(int I, int nc, int p, const std::vector<double> &gl,
                          int &cell, double &xi) {
  const int nn = p * nc + 1;
  if (I == nn - 1) { cell = nc - 1; xi = 1.0; return; }
  cell = I / p; xi = gl[I % p];
}

void build_mesh(const MeshDesc &d, int level, Mesh &m) {
  m = Mesh();
  m.p = d.p; m.q = d.q; m.geometry = d.geometry;
  Basis1D b; b.init(d.p, d.q);
  const int p = d.p;
  for (int k = 0; k < 3; ++k) {
    m.nc[k] = d.coarse[k] << level;
    m.nn[k] = p * m.nc[k] + 1;
  }
  const int ncx = m.nc[0], ncy = m.nc[1], ncz = m.nc[2];
  auto cell_active = [&](int i, int j, int k) -> bool {
    if (i < 0 || j < 0 || k < 0 || i >= ncx || j >= ncy || k >= ncz) return false;
    if (d.coarse_active.empty()) return true;
    int ci = i >> level, cj = j >> level, ck = k >> level;
    return d.coarse_active[(size_t)(ck * d.coarse[1] + cj) * d.coarse[0] + ci] != 0;
  };
  const size_t nlat = (size_t)m.nn[0] * m.nn[1] * m.nn[2];
  m.lattice_to_node.assign(nlat, -1);
  // cells in lexicographic order
  m.cell_of_lattice.assign((size_t)ncx * ncy * ncz, -1);
  for (int k = 0; k < ncz; ++k)
    for (int j = 0; j < ncy; ++j)
      for (int i = 0; i < ncx; ++i)
        if (cell_active(i, j, k)) {
          m.cell_of_lattice[((size_t)k * ncy + j) * ncx + i] = m.n_cells++;
          m.cell_ijk.push_back(i); m.cell_ijk.push_back(j); m.cell_ijk.push_back(k);
          for (int c = 0; c <= p; ++c)
            for (int bb = 0; bb <= p; ++bb)
              for (int a = 0; a <= p; ++a) {
                size_t L = ((size_t)(k * p + c) * m.nn[1] + (j * p + bb)) * m.nn[0] + (i * p + a);
                m.lattice_to_node[L] = 0;  // mark active
              }
        }
  // compact node numbering, lexicographic over the lattice (x fastest)
  for (size_t L = 0; L < nlat; ++L)
    if (m.lattice_to_node[L] == 0) {
      m.lattice_to_node[L] = m.n_nodes++;
      m.node_lattice.push_back((int)L);
    }
  m.X.resize(3 * (size_t)m.n_nodes);
  for (int n = 0; n < m.n_nodes; ++n) {
    size_t L = m.node_lattice[n];
    int I = L % m.nn[0], J = (L / m.nn[0]) % m.nn[1], K = L / ((size_t)m.nn[0] * m.nn[1]);
    int lat[3] = {I, J, K};
    double x[3];
    for (int dd = 0; dd < 3; ++dd) {
      int c; double xi;
      lattice_coord(lat[dd], m.nc[dd], p, b.nodes, c, xi);
      x[dd] = d.lo[dd] + (d.hi[dd] - d.lo[dd]) * ((c + xi) / m.nc[dd]);
    }
    if (d.geometry == GEOM_COOK) cook_transform(x[0], x[1]);
    for (int dd = 0; dd < 3; ++dd) m.X[3 * (size_t)n + dd] = x[dd] * d.scale;
  }
  const int ncn = m.ncn();
  m.cell_nodes.resize((size_t)m.n_cells * ncn);
  for (int cell = 0; cell < m.n_cells; ++cell) {
    int i = m.cell_ijk[3 * cell], j = m.cell_ijk[3 * cell + 1], k = m.cell_ijk[3 * cell + 2];
    int idx = 0;
    for (int c = 0; c <= p; ++c)
      for (int bb = 0; bb <= p; ++bb)
        for (int a = 0; a <= p; ++a) {
          size_t L = ((size_t)(k * p + c) * m.nn[1] + (j * p + bb)) * m.nn[0] + (i * p + a);
          m.cell_nodes[(size_t)cell * ncn + idx++] = m.lattice_to_node[L];
        }
  }
  // boundary faces and ids
  const int off[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
  for (int cell = 0; cell < m.n_cells; ++cell) {
    int i = m.cell_ijk[3 * cell], j = m.cell_ijk[3 * cell + 1], k = m.cell_ijk[3 * cell + 2];
    for (int f = 0; f < 6; ++f) {
      int ni = i + off[f][0], nj = j + off[f][1], nk = k + off[f][2];
      if (cell_active(ni, nj, nk)) continue;
      bool outer = (ni < 0 || nj < 0 || nk < 0 || ni >= ncx || nj >= ncy || nk >= ncz);
      int id;
      if (d.geometry == GEOM_COOK) {
        // mf_elasticity.h:1369-1390: x=0 -> 1, x=48 -> 11; the +/-Z test
        // compares center[0] with 0.5 and never fires.
        id = (f == 0) ? 1 : (f == 1 ? 11 : 0);
        if (!outer) id = 6;
      } else {
        id = outer ? f : 6;
      }
      m.bfaces.push_back(cell); m.bfaces.push_back(f); m.bfaces.push_back(id);
    }
  }
}

double mesh_volume(const Mesh &m, const Basis1D &b) {
  const int p = m.p, q = b.q, n1 = p + 1, ncn = m.ncn();
  double vol = 0.0;
  for (int cell = 0; cell < m.n_cells; ++cell) {
    const int *nodes = &m.cell_nodes[(size_t)cell * ncn];
    for (int qz = 0; qz < q; ++qz)
      for (int qy = 0; qy < q; ++qy)
        for (int qx = 0; qx < q; ++qx) {
          double J[3][3] = {};
          for (int c = 0; c <= p; ++c)
            for (int bb = 0; bb <= p; ++bb)
              for (int a = 0; a <= p; ++a) {
                const double *X = &m.X[3 * (size_t)nodes[(c * n1 + bb) * n1 + a]];
                double g[3] = {b.D[qx * n1 + a] * b.N[qy * n1 + bb] * b.N[qz * n1 + c],
                               b.N[qx * n1 + a] * b.D[qy * n1 + bb] * b.N[qz * n1 + c],
                               b.N[qx * n1 + a] * b.N[qy * n1 + bb] * b.D[qz * n1 + c]};
                for (int dd = 0; dd < 3; ++dd)
                  for (int e = 0; e < 3; ++e) J[dd][e] += X[dd] * g[e];
              }
          double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                       J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                       J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
          vol += det * b.qw[qx] * b.qw[qy] * b.qw[qz];
        }
  }
  return vol;
}

// Nodes of face f of a cell in lexicographic cell numbering.
static void face_local_nodes(int p, int f, std::vector<int> &out) {
  out.clear();
  const int n1 = p + 1;
  for (int c = 0; c <= p; ++c)
    for (int bb = 0; bb <= p; ++bb)
      for (int a = 0; a <= p; ++a) {
        bool on = (f == 0 && a == 0) || (f == 1 && a == p) || (f == 2 && bb == 0) ||
                  (f == 3 && bb == p) || (f == 4 && c == 0) || (f == 5 && c == p);
        if (on) out.push_back((c * n1 + bb) * n1 + a);
      }
}

void constrained_dofs(const Mesh &m, const std::vector<DirichletSpec> &bc,
                      std::vector<uint8_t> &mask) {
  mask.assign((size_t)m.n_dofs(), 0);
  std::vector<int> fl;
  const int ncn = m.ncn();
  for (size_t t = 0; t < m.bfaces.size(); t += 3) {
    int cell = m.bfaces[t], f = m.bfaces[t + 1], id = m.bfaces[t + 2];
    for (const auto &s : bc) {
      if (s.id != id) continue;
      face_local_nodes(m.p, f, fl);
      for (int ln : fl) {
        int node = m.cell_nodes[(size_t)cell * ncn + ln];
        for (int c = 0; c < 3; ++c)
          if (s.comp_mask & (1 << c)) mask[3 * (size_t)node + c] = 1;
      }
    }
  }
}

}  // namespace orc
