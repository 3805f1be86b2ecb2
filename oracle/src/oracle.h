// CPU oracle for the matrix-free Neo-Hookean tangent operator and its
// GMG-preconditioned CG / Newton driver.
//
// TEST INFRASTRUCTURE ONLY. This library is the checker: the pytest suite,
// the smoke() entry point and the CPU baseline leg of bench.py load it to
// compare against / time beside the CUDA path. Nothing in the product links it.
//
// It restates, in plain C++ (double and float, OpenMP over cells), the algorithm
// of davydden/large-strain-matrix-free:
//   include/material.h             Material_Compressible_Neo_Hook_One_Field
//   include/mf_nh_operator.h       NeoHookOperator (initialize/cache/vmult/diagonal)
//   include/mf_elasticity.h        residual assembly, constraints, CG, GMG, Newton
// plus the deal.II semantics those files rely on (FE_Q on Gauss-Lobatto nodes,
// QGauss, FEEvaluation sum factorisation, MappingQEulerian, MGTransferMatrixFree,
// PreconditionChebyshev, SolverCG) restated from their published definitions.
// Each function cites the reference file:line it follows.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace orc {

// ---------------------------------------------------------------- 1D basis
// FE_Q(p) Lagrange basis on Gauss-Lobatto nodes, evaluated at QGauss(q) points
// on [0,1] (mf_elasticity.h:1028 fe(FE_Q<dim>(degree), dim); :1070 QGauss).
struct Basis1D {
  int p = 0, q = 0;
  std::vector<double> nodes;   // p+1 GL nodes on [0,1]
  std::vector<double> qpts;    // q Gauss points on [0,1]
  std::vector<double> qw;      // q Gauss weights (sum 1)
  std::vector<double> N;       // [q][p+1] shape values
  std::vector<double> D;       // [q][p+1] shape derivatives
  void init(int p, int q);
  void eval(double x, double *val, double *der) const;  // at arbitrary x
};
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w);
void gauss_lobatto(int n, std::vector<double> &x);

// ------------------------------------------------------------------- mesh
// Logically structured hexahedral mesh: a box of nc[0]*nc[1]*nc[2] cells with
// an optional active-cell mask, a geometry map applied to the lattice, Q_p
// node lattice, boundary ids per face.  Geometries:
//   GEOM_BOX  : axis aligned box [lo,hi], deal.II colorize ids
//               (-x:0,+x:1,-y:2,+y:3,-z:4,+z:5), faces next to masked
//               cells get id 6.
//   GEOM_COOK : the Cook membrane of mf_elasticity.h:1339-1398 (ids 1 / 11,
//               plane-strain id 2 never set, :1387-1389), grid_y_transform
//               (:1251-1270), extruded over [lo[2],hi[2]] and scaled.
enum { GEOM_BOX = 0, GEOM_COOK = 1 };

struct MeshDesc {
  int geometry = GEOM_BOX;
  int coarse[3] = {1, 1, 1};
  int n_refinements = 0;
  double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  double scale = 1.0;
  int p = 2, q = 3;
  std::vector<uint8_t> coarse_active;  // empty = all active
};

struct Mesh {
  int p = 2, q = 3, geometry = GEOM_BOX;
  int nc[3] = {0, 0, 0};        // cells per direction
  int nn[3] = {0, 0, 0};        // node lattice per direction (p*nc+1)
  int n_cells = 0, n_nodes = 0;
  std::vector<int> lattice_to_node;  // -1 for inactive lattice nodes
  std::vector<int> node_lattice;     // compact node -> lattice index
  std::vector<double> X;             // 3*n_nodes reference coordinates
  std::vector<int> cell_nodes;       // n_cells*(p+1)^3, x fastest
  std::vector<int> cell_ijk;         // 3*n_cells
  std::vector<int> cell_of_lattice;  // lattice cell -> cell or -1
  // boundary faces: (cell, face 0..5 = -x,+x,-y,+y,-z,+z, boundary id)
  std::vector<int> bfaces;
  int ncn() const { return (p + 1) * (p + 1) * (p + 1); }
  int n_dofs() const { return 3 * n_nodes; }
};
void build_mesh(const MeshDesc &d, int level, Mesh &m);
double mesh_volume(const Mesh &m, const Basis1D &b);

// Per-dof constraint mask from Dirichlet boundary ids + component masks
// (mf_elasticity.h:2932-3007; DoFTools/interpolate_boundary_values on faces).
struct DirichletSpec {
  int id;
  int comp_mask;   // bit c set = component c constrained
};
void constrained_dofs(const Mesh &m, const std::vector<DirichletSpec> &bc,
                      std::vector<uint8_t> &mask);

// --------------------------------------------------------------- material
// material.h:78-94: kappa, c_1, mu, lambda from (mu, nu)
struct Material {
  double mu, nu, lambda, kappa, c1;
  int formulation;
  Material(double mu_ = 1, double nu_ = 0.3, int f = 1) { set(mu_, nu_, f); }
  void set(double mu_, double nu_, int f) {
    mu = mu_; nu = nu_; formulation = f;
    kappa = (2.0 * mu * (1.0 + nu)) / (3.0 * (1.0 - 2.0 * nu));
    c1 = mu / 2.0;
    lambda = (2.0 * mu * nu) / (1.0 - 2.0 * nu);
  }
};

enum Caching { CACHE_SCALAR = 0, CACHE_TENSOR2 = 1, CACHE_TENSOR4 = 2,
               CACHE_SCALAR_REFERENTIAL = 3, CACHE_TENSOR4_NS = 4 };

// ---------------------------------------------------------------- operator
// NeoHookOperator<3, p, q, Number> (mf_nh_operator.h:147-296).
template <typename Number>
struct Operator {
  const Mesh *mesh = nullptr;
  const Basis1D *basis = nullptr;
  int caching = CACHE_TENSOR4;
  int formulation = 1;
  std::vector<double> mu_cell;   // per cell shear modulus (material id -> mu)
  double nu = 0.3;
  std::vector<uint8_t> cmask;    // per dof constrained flag
  std::vector<int> constrained;  // list of constrained dofs
  // displacement around which we linearise (borrowed, like :261)
  std::vector<Number> u;
  // metric of the current (Eulerian) configuration: 9 inverse Jacobian + JxW
  std::vector<Number> jinv_cur, jxw_cur;
  // metric of the reference configuration (scalar caching needs both)
  std::vector<Number> jinv_ref, jxw_ref;
  // cache tables, [cell][qp][comp] (mf_nh_operator.h:263-267)
  std::vector<Number> c_scalar, c_second, c_t2, c_t4, c_t4ns;
  // scalar_referential and tensor4_ns work in the reference configuration
  bool referential() const { return caching == CACHE_SCALAR_REFERENTIAL || caching == CACHE_TENSOR4_NS; }
  std::vector<Number> diag, inv_diag;
  int nq() const { return basis->q * basis->q * basis->q; }
  void initialize(const Mesh *m, const Basis1D *b, int caching, int formulation);
  void set_material(const std::vector<double> &mu, double nu);
  void set_constraints(const std::vector<uint8_t> &mask);
  // interpolate metric + cache (mf_nh_operator.h:447-592, mf_elasticity.h:1949-1982)
  int cache(const Number *disp);   // returns 0, or 1 if det F <= 0 somewhere
  void vmult(Number *dst, const Number *src) const;       // :612-706
  // K g over constrained columns: gather without zeroing constrained
  // entries, scatter skipping constrained rows (the inhomogeneity term that
  // AffineConstraints::distribute_local_to_global moves into the rhs).
  void apply_inhomogeneous(Number *dst, const Number *g) const;
  void compute_diagonal();                                 // :1503-1557
  // apply on one cell to a local vector (component-blocked), used by tests
  void cell_apply(int cell, const Number *in, Number *out) const;
};

// ------------------------------------------------------- residual (FP64)
// assemble_system rhs part (mf_elasticity.h:2736-2921):
// R = -int tau : grad^s N dV + int T . N dA, constrained entries zeroed.
struct Neumann {
  int id;
  // traction components = a[c] + b[c]*t (linear in load time), evaluated
  // at the reference face point.  Expressions of x,y,z are handled by the
  // product's .prm reader; the oracle needs only load-linear tractions.
  double a[3], b[3];
};
double residual(const Mesh &m, const Basis1D &b, const std::vector<double> &mu,
                double nu, int formulation, const double *u,
                const std::vector<Neumann> &neu, double time,
                const std::vector<uint8_t> &cmask, double *R);

// Adjoint building block: g[c] = lambda . dR/dlog mu_c for every cell, with
// R the internal-force part of the residual (mf_elasticity.h:2736-2804) and
// tau differentiated in mu (lambda(mu), kappa(mu) of material.h:82-94).
void dresidual_dlogmu_dot(const Mesh &m, const Basis1D &b, const std::vector<double> &mu, double nu,
                          int formulation, const double *u, const double *lam, double *g);

// ------------------------------------------------ single-cell element matrix
// Independent FEValues-style assembly in the reference configuration
// (tests/mf_neo_hook_operator.cc:300-470 and mf_elasticity.h:2760-2843):
// K_ij = int grad^s N_i : Jc(grad^s N_j) + grad N_i : (grad N_j tau) dV.
void element_matrix(const Mesh &m, const Basis1D &b, int cell, const Material &mat,
                    const double *u, std::vector<double> &K);

}  // namespace orc
