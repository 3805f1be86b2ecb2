// CPU oracle (test infrastructure only): solver-level structures.
#pragma once
#include <limits>
#include <vector>

#include "oracle.h"

namespace orc {

// Cell-wise nested-Lagrange transfer between level l-1 (coarse) and l (fine)
// (deal.II MGTransferMatrixFree as built in mf_elasticity.h:1919-1922).
struct Transfer {
  std::vector<double> P1;       // (2p+1) x (p+1) 1D interpolation matrix
  std::vector<int> fine_nodes;  // per coarse cell (2p+1)^3 fine node ids
  std::vector<double> weight;   // 1 / multiplicity per fine node
  int n_coarse_cells = 0, nfb = 0;
  void build(const Mesh &coarse, const Mesh &fine, const Basis1D &b);
  template <typename T>
  void prolongate_add(const Mesh &coarse, const std::vector<uint8_t> &ccmask, const T *src, T *dst) const;
  template <typename T>
  void restrict_add(const Mesh &coarse, const std::vector<uint8_t> &ccmask, const T *src, T *dst) const;
  template <typename T>
  void interpolate(const Mesh &coarse, const Mesh &fine, const T *fine_u, T *coarse_u) const;
};

template <typename T>
struct Chebyshev {
  const Operator<T> *op = nullptr;
  std::vector<T> inv_diag;
  int degree = 5;
  double theta = 1, delta = 0, eig_min = 1, eig_max = 1;
  // degree <= 0 selects the "solver" mode with range = target reduction
  void setup(const Operator<T> &A, const std::vector<T> &inv_diag, int degree, double range, int eig_its);
  void run(std::vector<T> &x, const std::vector<T> &b, bool zero_start) const;
};

template <typename T>
struct GMG {
  struct Level {
    Mesh mesh;
    std::vector<uint8_t> cmask;
    Operator<T> op;
    Chebyshev<T> cheb;
    Transfer transfer;  // from level-1 to this level (unused on level 0)
  };
  std::vector<Level> levels;
  // coarse solve: Chebyshev "solver" mode, or (coarse_cg) CG preconditioned
  // by the level-0 Chebyshev smoother to a 1e-3 reduction
  // (MGCoarseGridIterativeSolver, mf_elasticity.h:2116-2127)
  bool coarse_cg = false;
  void vcycle(int l, std::vector<T> &x, const std::vector<T> &b) const;
  void vmult(std::vector<double> &dst, const std::vector<double> &src) const;
};

struct NewtonParams {
  MeshDesc mesh;
  int caching = CACHE_TENSOR4, formulation = 1;
  double mu = 1.0, nu = 0.3;
  std::vector<double> mu_fine;      // optional per fine cell (lexicographic cell order)
  std::vector<DirichletSpec> dirichlet;
  std::vector<std::vector<double>> dirichlet_value;  // per spec, 3 values (step increment)
  std::vector<Neumann> neumann;
  double end_time = 1.0, dt = 0.1;
  int max_nr = 10;
  double tol_f = 1e-9, tol_u = 1e-6, tol_f_abs = 0.0, tol_u_abs = 0.0;
  double tol_lin = 1e-6;
  int max_it_mult = 1;
  int precond = 2;  // 0 none, 1 jacobi, 2 gmg
  double relaxation = 0.65;
  int cheb_degree = 5, cheb_eig_its = 30;
  double smoothing_range = 20.0;
  int coarse_chebyshev = 1, coarse_accurate_eig = 1;
  int level_fp32 = 1;
  int has_output_point = 0;
  double output_point[3] = {0, 0, 0};
};

struct StepResult {
  double time = 0;
  int newton_iterations = 0;
  bool converged = false;
  std::vector<int> cg_iterations;
  // per Newton iteration: relative residual and relative update norm seen
  // by the convergence check
  std::vector<double> rel_res, rel_upd;
  double point_u[3] = {0, 0, 0};
};

struct NewtonResult {
  int n_cells = 0, n_dofs = 0;
  double volume = 0;
  std::vector<StepResult> steps;
  std::vector<double> u;
};

bool point_value(const Mesh &m, const Basis1D &b, const double *u, const double pt[3], double out[3]);
std::vector<double> coarsen_cell_field(const std::vector<Mesh> &meshes, int l, const std::vector<double> &fine);
template <typename LT>
void setup_gmg(const NewtonParams &prm, const std::vector<Mesh> &meshes, const Basis1D &bas,
               const std::vector<std::vector<uint8_t>> &lmask, const std::vector<std::vector<double>> &lmu,
               const std::vector<double> &u_fine, GMG<LT> &gmg, bool first);
int newton_run(const NewtonParams &prm, NewtonResult &res);
// adjoint gradient of a boundary misfit with respect to the per-cell log
// shear modulus (returns 0, or the newton_run / CG failure code)
int adjoint_run(const NewtonParams &prm, const std::vector<double> &log_mu, const std::vector<double> &target,
                int obj_id, double &J, std::vector<double> &grad, std::vector<double> &u);

}  // namespace orc
