// Problem layer: parameters of a reference-format .prm file, boundary
// expressions, and the state of the device Newton driver.
#pragma once
#include <array>
#include <map>
#include <string>
#include <vector>

#include "solver_internal.h"

namespace lsmf {

// A parsed function of (x, y, z, t) (the FunctionParser expressions of the
// "Boundary conditions" subsection, mf_elasticity.h:215-248).
struct Expr {
  struct Ins {
    int op;
    double v;
    int f;
  };
  std::vector<Ins> prog;
  std::string text;
  bool parse(const std::string &src, std::string &err);
  double eval(double x, double y, double z, double t) const;
};

struct BCExpr {
  int id = 0;
  Expr expr[3];
};

// Keys of mf_elasticity.h:156-607 (defaults as declared there) plus the
// additive keys without a reference counterpart: Geometry / Type = Box, Box
// cells, Box lower / upper corner, Void spheres, Cook thickness; Linear
// solver / MF level precision, MF Chebyshev degree, MF Chebyshev smoothing
// range, MF scatter.
struct ProblemParams {
  // Finite element system
  int degree = 2, quad_order = 3;
  // Geometry
  int elements_per_edge = 32, n_refinements = 0, extrusion_slices = 5, dim = 2;
  double scale = 1e-3, extrusion_height = 1;
  std::string type = "Cook";
  int box_cells[3] = {1, 1, 1};
  double box_lo[3] = {0, 0, 0}, box_hi[3] = {1, 1, 1};
  double cook_thickness = 1.0;
  int void_count = 0, void_seed = 0;
  double void_radius = 0;
  // Material properties
  double nu = 0.3, mu = 0.4225e6;
  int formulation = 0;
  // Linear solver
  std::string solver_type = "CG", precond = "jacobi", caching = "scalar", level_precision = "float";
  std::string scatter = "atomic";  // atomic | colour8 (bit-reproducible cell loops)
  double tol_lin = 1e-6, relaxation = 0.65, amg_threshold = 1e-4, smoothing_range = 20.0;
  int max_it_mult = 1, cond_cg_its = 20, cheb_eig_its = 30, cheb_degree = 5;
  bool coarse_chebyshev = true, coarse_accurate_eig = true;
  // Nonlinear solver
  int max_nr = 10;
  double tol_f = 1e-9, tol_f_abs = 0.0, tol_u = 1e-6, tol_u_abs = 0.0;
  // Time
  double end_time = 1.0, dt = 0.1;
  // Misc
  std::string output_folder;
  bool output_solution = true, always_assemble = true, output_abs_norms = false;
  std::vector<std::array<double, 3>> output_points;
  // Boundary conditions
  std::vector<BCExpr> dirichlet, neumann;
  std::map<int, int> dirichlet_mask;
};

lsmf_status parse_prm(const std::string &text, ProblemParams &P);

}  // namespace lsmf

struct lsmf_problem {
  lsmf::ProblemParams prm;
  lsmf_mesh *mesh = nullptr;
  lsmf_op *op = nullptr;       // FP64 fine operator
  lsmf_gmg *gmg = nullptr;     // level hierarchy (gmg preconditioner)
  std::vector<double> mu_fine;
  lsmf::DevBuf<double> u_n, du, u_tot, R, dx, fext, gvals, tmp, lam, grad, target, mu_dev;
  std::vector<uint8_t> obj_mask_dofs;
  bool inhom = false;
  // output point: fine cell node ids + shape weights
  bool have_point = false;
  std::vector<int> point_nodes;
  std::vector<double> point_w;
  int adjoint_obj_id = -1;
  bool forward_done = false;
  cudaStream_t stream = 0;
  ~lsmf_problem();
};
