/*
 * lsmf.h — C ABI of the B200-native matrix-free Neo-Hookean tangent operator
 * and its GMG-preconditioned CG / Newton driver.
 *
 * Drop-in boundary for the hot path of davydden/large-strain-matrix-free:
 * each entry point names the reference interface it replaces (file:line,
 * paths inside that project).  All device buffers are caller-owned raw CUDA
 * device pointers; vectors are FP64 ("double") or FP32 ("float") arrays of
 * n_dofs = 3 * n_nodes entries, node-major (dof = 3 * node + component).
 * Every call is asynchronous on the handle's CUDA stream unless it returns a
 * host value.  Handles are not thread-safe.  No function throws; failures
 * are reported as lsmf_status codes (lsmf_status_string gives the text and
 * lsmf_last_error the detail of the most recent failure on this thread).
 */
#ifndef LSMF_H
#define LSMF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LSMF_OK = 0,
  LSMF_ERR_INVALID_ARG = 1,
  LSMF_ERR_UNKNOWN_CACHING = 2,      /* mf_nh_operator.h:439-442 AssertThrow */
  LSMF_ERR_DETF_NONPOSITIVE = 3,     /* mf_nh_operator.h:477-483 det_F > 0   */
  LSMF_ERR_NOT_INITIALIZED = 4,
  LSMF_ERR_CG_NOT_CONVERGED = 5,     /* SolverControl::NoConvergence         */
  LSMF_ERR_NEWTON_NOT_CONVERGED = 6, /* mf_elasticity.h:2557-2558            */
  LSMF_ERR_CUDA = 7,
  LSMF_ERR_TIMEOUT = 8,
  LSMF_ERR_PRM = 9,                  /* ParameterHandler::parse_input        */
  LSMF_ERR_UNSUPPORTED = 10,
  LSMF_ERR_ALLOC = 11
} lsmf_status;

/* MF caching variants: "MF caching" (mf_elasticity.h:445-450) */
typedef enum {
  LSMF_CACHE_SCALAR = 0,
  LSMF_CACHE_TENSOR2 = 1,
  LSMF_CACHE_TENSOR4 = 2,
  LSMF_CACHE_SCALAR_REFERENTIAL = 3, /* reference frame, mf_nh_operator.h:1255-1400 (formulation 1) */
  LSMF_CACHE_TENSOR4_NS = 4          /* dP/dF, reference frame, mf_nh_operator.h:563-582 (formulation 1) */
} lsmf_caching;

typedef enum { LSMF_FP64 = 0, LSMF_FP32 = 1 } lsmf_precision;

/* MFMask stage bits (mf_nh_operator.h:74-85) for vmult breakdowns */
enum {
  LSMF_MASK_ZERO = 1, LSMF_MASK_MPI = 2, LSMF_MASK_RW = 4, LSMF_MASK_SF = 8, LSMF_MASK_QD = 16,
  LSMF_MASK_DEFAULT = 31
};

typedef enum { LSMF_GEOM_BOX = 0, LSMF_GEOM_COOK = 1 } lsmf_geometry;

/* Structured hexahedral mesh description.  coarse[] cells are refined
 * n_refinements times (levels 0 .. n_refinements).  BOX: [lo,hi] with
 * boundary ids -x:0 +x:1 -y:2 +y:3 -z:4 +z:5 and 6 on faces next to masked
 * (void) cells.  COOK: the Cook membrane of mf_elasticity.h:1339-1398
 * (x in [0,48], y in [0,44] mapped by grid_y_transform, z in [lo[2],hi[2]],
 * times scale), ids 1 (x=0) and 11 (x=48).  coarse_active (optional,
 * coarse[0]*coarse[1]*coarse[2] bytes, x fastest) removes coarse cells. */
typedef struct {
  int geometry;
  int coarse[3];
  int n_refinements;
  double lo[3], hi[3];
  double scale;
  int degree;        /* "Polynomial degree" */
  int n_q_points_1d; /* "Quadrature order"  */
  const uint8_t *coarse_active;
} lsmf_mesh_desc;

typedef struct lsmf_mesh lsmf_mesh;
typedef struct lsmf_op lsmf_op;
typedef struct lsmf_gmg lsmf_gmg;
typedef struct lsmf_problem lsmf_problem;

const char *lsmf_status_string(lsmf_status s);
const char *lsmf_last_error(void);
const char *lsmf_version(void);

/* ---- mesh: replaces make_grid + system_setup (mf_elasticity.h:1339-1708)
 * for the structured meshes of this path; builds every multigrid level. */
lsmf_status lsmf_mesh_create(const lsmf_mesh_desc *desc, lsmf_mesh **out);
void lsmf_mesh_destroy(lsmf_mesh *m);
/* sizes of a level (level = -1: finest) */
lsmf_status lsmf_mesh_info(const lsmf_mesh *m, int level, int *n_cells, int *n_nodes, int *n_dofs);
int lsmf_mesh_n_levels(const lsmf_mesh *m);
/* host copies: X[3*n_nodes], cell_nodes[n_cells*(p+1)^3], cell_ijk[3*n_cells] */
lsmf_status lsmf_mesh_arrays(const lsmf_mesh *m, int level, double *X, int *cell_nodes, int *cell_ijk);
/* Dirichlet constraints, the "Dirichlet IDs and component mask" of
 * mf_elasticity.h:215-248 / make_constraints :2932-3007: n pairs of
 * (boundary id, component bits).  Applied on every level. */
lsmf_status lsmf_mesh_set_dirichlet(lsmf_mesh *m, int n, const int *ids, const int *comp_masks);
/* host copy of the per-dof constrained flags of a level */
lsmf_status lsmf_mesh_constraint_mask(const lsmf_mesh *m, int level, uint8_t *mask);

/* ---- operator: NeoHookOperator<dim,p,q,number> (mf_nh_operator.h:147-296) */
/* initialize(): mf_nh_operator.h:394-443 (caching selection, tables sized) */
lsmf_status lsmf_operator_create(lsmf_mesh *m, int level, lsmf_caching caching, int formulation,
                                 lsmf_precision precision, lsmf_op **out);
void lsmf_operator_destroy(lsmf_op *op);
/* set_material(): mf_nh_operator.h:594-608, generalised to a per-cell shear
 * modulus (host array, n_cells of the operator's level) and one Poisson
 * ratio (material.h:82-94 gives kappa, c_1, lambda). */
lsmf_status lsmf_operator_set_material(lsmf_op *op, const double *mu_per_cell, double nu);
/* cache(): mf_nh_operator.h:447-592 plus the Eulerian MatrixFree metric of
 * mf_elasticity.h:1949-1982.  d_displacement: device vector of the
 * operator's precision, borrowed (must outlive the operator, like :261).
 * Returns LSMF_ERR_DETF_NONPOSITIVE if det F <= 0 at any quadrature point. */
lsmf_status lsmf_operator_cache(lsmf_op *op, const void *d_displacement);
/* vmult<mask>(): mf_nh_operator.h:612-706 (dst = A src; constrained rows
 * are identity, :702-705).  Tvmult is the same operator (:626-645). */
lsmf_status lsmf_operator_vmult(lsmf_op *op, void *d_dst, const void *d_src, unsigned mask);
/* vmult_add(): dst += A src */
lsmf_status lsmf_operator_vmult_add(lsmf_op *op, void *d_dst, const void *d_src);
/* compute_diagonal(): mf_nh_operator.h:789-918, 1503-1557 */
lsmf_status lsmf_operator_compute_diagonal(lsmf_op *op);
/* get_matrix_diagonal_inverse(): device pointer owned by the operator */
lsmf_status lsmf_operator_get_diagonal(lsmf_op *op, const void **d_diag, const void **d_inv_diag);
/* precondition_Jacobi(): dst = omega * D^-1 src (mf_nh_operator.h:348-360) */
lsmf_status lsmf_operator_precondition_jacobi(lsmf_op *op, void *d_dst, const void *d_src, double omega);
/* m(), n(), memory_consumption() (mf_nh_operator.h:300-392): rows and
 * columns (n_dofs); bytes of the cache tables plus the index map and node
 * coordinates (the MatrixFree data), diagonals excluded like the reference */
int lsmf_operator_m(const lsmf_op *op);
int lsmf_operator_n(const lsmf_op *op);
size_t lsmf_operator_memory_consumption(const lsmf_op *op);
/* el(row, col) (mf_nh_operator.h:1562-1571): the diagonal entry; needs
 * compute_diagonal(); row != col gives LSMF_ERR_UNSUPPORTED (the reference's
 * ExcNotImplemented).  Synchronous (one value copied to the host). */
lsmf_status lsmf_operator_el(lsmf_op *op, int row, int col, double *value);
/* execution options (no reference counterpart; defaults are the fast path):
 * LSMF_OPT_BULK_PIPELINE: depth 1..3 of the shared-memory ring through which
 *   each warp streams its cell records with bulk copies; 0 = plain coalesced
 *   loads; -1 (default) = measured choice: 1 for tensor4, tensor4_ns and
 *   scalar_referential of degree 1 or 2 while a cell record fits in 24 KB,
 *   else 0.  The
 *   depth is reduced when the ring would not fit in shared memory.
 * LSMF_OPT_BASIC_KERNEL: 1 = the basic vmult kernel (per-warp shared-memory
 *   sweeps, plain loads); the stage mask of vmult always uses it.
 * LSMF_OPT_MAX_WARPS: cap on warps per block of the vmult kernel (1..8;
 *   0 = default: 8 for FP64 tensor2 and scalar, 2 for FP64
 *   scalar_referential, 4 otherwise).
 * LSMF_OPT_WAIT_TRIES: bound of the pipelined kernel's wait for a cell
 *   record (mbarrier try_wait calls; -1 = default 2^22, seconds).  A wait
 *   that runs out sets the operator's device error word, lets every copy
 *   the warp still has in flight land (default bound) and ends the warp;
 *   0 makes every wait run out at once (for tests of that path).
 * LSMF_OPT_SCATTER: 0 (default) = the cell loop adds its contributions
 *   with atomics (summation order varies run to run); 1 = colour8: the
 *   cells are processed in the 8 parity colours of the structured lattice,
 *   one launch per colour, so that no two cells of a launch share a node
 *   and the sums are formed in a fixed order without atomics
 *   (bit-reproducible vmult, for parity and debugging); 2 = nodesum: one
 *   full cell loop stores every cell's results to a per-cell buffer
 *   (n_cells x 3 (p+1)^3 values, allocated when the mode is selected) and
 *   a node kernel adds each node's cell contributions in increasing cell
 *   order (bit-reproducible as well, one cell loop instead of eight; the
 *   diagonal and the other cell loops of a nodesum operator use the
 *   colours).
 * LSMF_OPT_RECORD_PREFETCH: with plain record loads, 1 issues an L1
 *   prefetch of the cell's record before its sum-factorisation sweeps, 2 of
 *   the next cell's record, 0 none; -1 (default): 1, except 0 for the FP64
 *   scalar variant (measured).
 * LSMF_OPT_CELL_PAIRS: FP32 operators only: 1 = the vmult cell loop takes
 *   two cells per warp and runs their sum factorisation and point physics
 *   as the two halves of packed FP32x2 registers (one sm_100 f32x2
 *   instruction for both cells); 0 = one cell per warp; -1 (default) =
 *   measured choice (pairs for Q1 tensor2 / scalar formulation 1, Q2
 *   tensor2 / scalar formulation 1 / scalar_referential, Q4
 *   scalar_referential).  Ignored for FP64 operators.
 * LSMF_OPT_CHUNKS: the atomic-scatter vmult cell loop split into 2..8
 *   contiguous cell chunks on streams of the operator's own, forked from
 *   and joined back into its stream: each chunk zeroes its range of dst and
 *   applies the identity rows there, then runs its cells once the next
 *   chunk has zeroed its range, so the zeroing, the identity rows and the
 *   ends of the chunks' launches overlap other chunks' cell loops (levels
 *   with fewer than 1024 cells per chunk run in one piece); 1 = one launch;
 *   -1 (default) = measured choice: from 131,072 cells 8 for
 *   scalar_referential and tensor4_ns, 2 for tensor2, 4 otherwise; from
 *   32,768 cells 2; below that 1.  The operators a GMG object or a problem
 *   creates start at 1 (measured faster inside the Newton solve).  The
 *   chunks' streams and events are created by lsmf_operator_cache (and by
 *   this option on a cached operator), not by the vmult.
 * A bounded device wait that runs out in the pipelined kernel is reported
 * as LSMF_ERR_TIMEOUT by lsmf_operator_sync, lsmf_cg_solve and the GMG
 * set-up (the next synchronising call on the operator). */
enum { LSMF_OPT_BULK_PIPELINE = 1, LSMF_OPT_BASIC_KERNEL = 2, LSMF_OPT_MAX_WARPS = 3, LSMF_OPT_WAIT_TRIES = 4,
       LSMF_OPT_SCATTER = 5, LSMF_OPT_RECORD_PREFETCH = 6, LSMF_OPT_CELL_PAIRS = 7, LSMF_OPT_CHUNKS = 8 };
enum { LSMF_SCATTER_ATOMIC = 0, LSMF_SCATTER_COLOUR8 = 1, LSMF_SCATTER_NODESUM = 2 };
lsmf_status lsmf_operator_set_option(lsmf_op *op, int option, int value);
/* The value of an option as set (-1 / 0 for the automatic choices), except
 * LSMF_OPT_CHUNKS, which reports the chunk count the next full vmult cell
 * loop runs in (the automatic choice resolved; 1 = one launch).  No
 * reference counterpart. */
lsmf_status lsmf_operator_get_option(lsmf_op *op, int option, int *value);
/* Wait for the operator's stream and report a device error its kernels
 * recorded since the last report (LSMF_ERR_TIMEOUT for a bounded wait that
 * ran out; the word is cleared once reported).  No reference counterpart:
 * deal.II's vmult is synchronous and has no device waits. */
lsmf_status lsmf_operator_sync(lsmf_op *op);
/* the CUDA stream every operator call is ordered on (cudaStream_t) */
lsmf_status lsmf_operator_set_stream(lsmf_op *op, void *stream);
/* copy a cache table to the host for checking: which = 0 scalar / c1,
 * 1 second scalar, 2 tau/J (6 per qp), 3 tensor4 (36 per qp), 4 inverse
 * Jacobian (9 per qp; Eulerian, or referential for scalar_referential and
 * tensor4_ns), 5 JxW (same frame), 6 scalar_referential displacement values
 * (3 per qp), 7 tensor4_ns dP/dF (81 per qp, index ((i*3+j)*3+k)*3+l);
 * layout [cell][qp][comp] converted to double.  tensor4, tensor2 and
 * tensor4_ns cache their coefficients multiplied by JxW (the point result
 * is linear in them): tables 0-3 and 7 of those hold the coefficient times
 * JxW, and table 5 is LSMF_ERR_INVALID_ARG.  Returns the number of doubles
 * in *count. */
lsmf_status lsmf_operator_get_table(lsmf_op *op, int which, double *host, size_t *count);

/* ---- geometric multigrid preconditioner (mf_elasticity.h:1712-2241) ---- */
typedef struct {
  int caching;              /* level operators' caching */
  int formulation;
  lsmf_precision precision; /* LevelNumberType (float in the reference) */
  int smoother_degree;      /* Chebyshev degree (5 in mf_elasticity.h:2104) */
  double smoothing_range;   /* 20 */
  int eig_cg_iterations;    /* "MF Chebyshev number CG iterations" (30) */
  int coarse_chebyshev;     /* "MF Chebyshev coarse" (true) */
  int coarse_accurate_eig;  /* "MF Chebyshev coarse accurate eigenvalues" */
} lsmf_gmg_desc;

lsmf_status lsmf_gmg_create(lsmf_mesh *m, const lsmf_gmg_desc *desc, lsmf_gmg **out);
void lsmf_gmg_destroy(lsmf_gmg *g);
lsmf_status lsmf_gmg_set_material(lsmf_gmg *g, const double *mu_per_fine_cell, double nu);
/* interpolate_to_mg + level cache + diagonal + Chebyshev eigenvalue
 * estimates (mf_elasticity.h:1929-2113); d_u_fine: FP64 device vector */
lsmf_status lsmf_gmg_setup(lsmf_gmg *g, const double *d_u_fine);
/* PreconditionMG::vmult: one V-cycle, dst = M^-1 src (FP64 device vectors) */
lsmf_status lsmf_gmg_vmult(lsmf_gmg *g, double *d_dst, const double *d_src);
/* Chebyshev data of a level: out6 = {eig_min, eig_max (Lanczos estimates),
 * degree, theta, delta, eigenvalue-CG iterations} */
lsmf_status lsmf_gmg_level_info(const lsmf_gmg *g, int level, double *out6);
/* CUDA stream of every level operation (cudaStream_t) */
lsmf_status lsmf_gmg_set_stream(lsmf_gmg *g, void *stream);
/* the level operator of a level (the reference's mg_matrices[level],
 * mf_elasticity.h:2046-2077), owned by the GMG object: for its options
 * (lsmf_operator_set_option) and for inspection; a changed option takes
 * effect from the next set-up */
lsmf_status lsmf_gmg_level_operator(lsmf_gmg *g, int level, lsmf_op **op);
/* options: LSMF_GMG_OPT_GRAPH = 1 (default) replays the V-cycle as one CUDA
 * graph (for a given pair of vmult buffers); the first vmult after a set-up
 * captures the new launch sequence and updates the executable graph in
 * place, or instantiates it again when the sequence changed (another coarse
 * Chebyshev degree).  0 launches the kernels one by one.
 * LSMF_GMG_OPT_SCATTER: LSMF_SCATTER_ATOMIC (default), LSMF_SCATTER_COLOUR8
 * or LSMF_SCATTER_NODESUM for every level operator; diagonal, restriction
 * and prolongation use the colours for either deterministic mode (a
 * bit-reproducible V-cycle). */
enum { LSMF_GMG_OPT_GRAPH = 1, LSMF_GMG_OPT_SCATTER = 2 };
lsmf_status lsmf_gmg_set_option(lsmf_gmg *g, int option, int value);

/* ---- CG (SolverCG as driven by solve_linear_system, mf_elasticity.h:3012-3214) */
typedef struct {
  int iterations;
  double residual;
  int converged;
} lsmf_solve_info;
/* Solve A x = b to ||b - A x|| <= tol_abs (x is the initial guess).  precond:
 * 0 none, 1 Jacobi (omega * D^-1), 2 the given GMG. */
lsmf_status lsmf_cg_solve(lsmf_op *fine, int precond, double omega, lsmf_gmg *gmg, double *d_x,
                          const double *d_b, double tol_abs, int max_it, lsmf_solve_info *info);


/* ---- full problem: .prm driven load stepping (Solid::run) ---- */
/* Parse a reference-format .prm text (ParameterHandler syntax, keys of
 * mf_elasticity.h:156-607) plus the additive keys (Geometry: Type = Box,
 * Box cells, Box lower corner, Box upper corner, Void spheres, Cook
 * thickness; Linear solver: MF level precision, MF Chebyshev degree, MF
 * Chebyshev smoothing range), build mesh, operators, GMG and loads. */
lsmf_status lsmf_problem_create(const char *prm_text, lsmf_problem **out);
/* Parse and check a .prm text without touching the device (undeclared keys,
 * bad values and unsupported options give LSMF_ERR_PRM / _UNSUPPORTED). */
lsmf_status lsmf_prm_validate(const char *prm_text);
void lsmf_problem_destroy(lsmf_problem *p);
/* per fine cell shear modulus override (host array) */
lsmf_status lsmf_problem_set_mu(lsmf_problem *p, const double *mu_per_cell);
lsmf_status lsmf_problem_info(const lsmf_problem *p, int *n_cells, int *n_dofs, double *volume);
/* CUDA stream of the Newton driver and its operators (cudaStream_t) */
lsmf_status lsmf_problem_set_stream(lsmf_problem *p, void *stream);
/* Run all load steps (Solid::run, mf_elasticity.h:1187-1235). */
typedef struct {
  int n_steps;
  int newton_iterations[256];   /* per load step */
  int cg_iterations[256];       /* sum over the Newton steps of a load step */
  double point_u[256][3];       /* displacement at the first output point */
  double time_residual, time_setup, time_solve; /* seconds, device-timed */
} lsmf_newton_info;
lsmf_status lsmf_problem_run(lsmf_problem *p, lsmf_newton_info *info);
/* final displacement (host, n_dofs doubles) */
lsmf_status lsmf_problem_get_solution(const lsmf_problem *p, double *host_u);

/* ---- residual: the right-hand side part of assemble_system
 * (mf_elasticity.h:2708-2922) for the problem's mesh, per-cell shear
 * modulus, Poisson ratio and formulation:
 *   R = -int tau(u) : grad N dV  (:2736-2804, FP64)
 *       + int T(x, t) . N dA      (Neumann faces of the .prm, :2859-2892)
 * with the entries of Dirichlet-constrained dofs set to zero (:2917-2921),
 * and *norm = ||R||_2 over the dofs (the reference's error_residual).
 * d_u, d_R: FP64 device vectors of n_dofs; t: load time of the traction
 * expressions.  Waits for the problem's stream (norm is a host value). */
lsmf_status lsmf_residual(lsmf_problem *p, const double *d_u, double t, double *d_R, double *norm);

/* ---- z-slab partitions and the distributed operator ----
 * The reference distributes its mesh over MPI ranks and exchanges the
 * interface values around every cell loop (src.update_ghost_values(), cell
 * loop, dst.compress(add): mf_nh_operator.h:680-700) and all-reduces the CG
 * scalars (SolverCG, mf_elasticity.h:3175-3180).  Here part r of n_parts
 * owns the coarse cell layers k in [floor(r nz / n), floor((r+1) nz / n)) of
 * the structured mesh (with all refinements); the nodes of an interface
 * plane are owned by the upper part.  Local vectors of a part hold its owned
 * nodes and its ghost nodes (the upper interface), node-major. */
lsmf_status lsmf_mesh_create_part(const lsmf_mesh_desc *desc, int n_parts, int part, lsmf_mesh **out);
/* Host-only layout of a part (no device needed): its node count, the node
 * count of the whole mesh, the whole-mesh node number of each local node,
 * and the local nodes shared with part - 1 (owned here) and with part + 1
 * (ghosts here), both in whole-mesh node order.  Output arrays may be NULL
 * (sizes only). */
lsmf_status lsmf_partition_layout(const lsmf_mesh_desc *desc, int n_parts, int part, int *n_nodes, int *n_global_nodes,
                                  int *global_node, int *n_lower, int *lower, int *n_upper, int *upper);
typedef struct lsmf_dist lsmf_dist;
/* All parts in this process: ops[r] is the FP64 finest-level operator of
 * part r (on any GPU; create it after its mesh's Dirichlet set); each part's
 * work is ordered on its operator's stream.  The interface exchange is
 * fused into the cell loops where every part can reach its upper
 * neighbour's memory (same GPU, or peer access, which this call enables):
 * the cells next to an interface read the owners' src values and add their
 * contributions to the owners' dst directly (P2P loads and atomics), with
 * events ordering the neighbours' streams.  Otherwise the packed exchange
 * (cudaMemcpyAsync between the parts' streams) is used. */
lsmf_status lsmf_dist_create_group(int n_parts, lsmf_op *const *ops, lsmf_dist **out);
/* Interface exchange of the distributed vmult: PACKED (pack, copy / NCCL,
 * unpack around the cell loops, as update_ghost_values and compress(add))
 * or FUSED (group objects only, the default where it applies; operators
 * with the basic kernel or a deterministic scatter use PACKED).  Setting
 * FUSED where it cannot apply is LSMF_ERR_UNSUPPORTED.  get reports the
 * form the next vmult uses.  No reference counterpart (deal.II always
 * exchanges through MPI buffers). */
enum { LSMF_DIST_EXCHANGE_PACKED = 0, LSMF_DIST_EXCHANGE_FUSED = 1 };
lsmf_status lsmf_dist_set_exchange(lsmf_dist *d, int mode);
lsmf_status lsmf_dist_get_exchange(const lsmf_dist *d, int *mode);
/* One part per process over NCCL (libnccl.so.2 loaded at run time): every
 * process passes the same 128-byte id, made by one of them with
 * lsmf_dist_nccl_unique_id and shared by the host framework. */
lsmf_status lsmf_dist_nccl_unique_id(unsigned char *id128);
lsmf_status lsmf_dist_create_nccl(lsmf_op *op, const unsigned char *id128, lsmf_dist **out);
void lsmf_dist_destroy(lsmf_dist *d);
/* dst = A src over all parts (arrays of this object's local vectors, one
 * per part it holds): the owners' values of the ghost entries of src are
 * used by the cell loops, the ghosts' partial sums are added on the owners
 * and the ghost entries of dst are zero.  dst is valid on the owned
 * entries.  The packed exchange also sets the ghost entries of src from
 * their owners; the fused one leaves them as they are. */
lsmf_status lsmf_dist_vmult(lsmf_dist *d, double *const *dst, double *const *src);
/* sum over the owned entries of a . b, over all parts (host value) */
lsmf_status lsmf_dist_dot(lsmf_dist *d, const double *const *a, const double *const *b, double *out);
/* SolverCG over the parts, precond 0 (none) or 1 (Jacobi with the
 * diagonal summed across the interfaces).  b: right-hand side on the owned
 * entries (its ghost entries are ignored).  x: initial guess, solution on
 * return (ghost entries set from their owners). */
lsmf_status lsmf_dist_cg_solve(lsmf_dist *d, int precond, double omega, double *const *x, const double *const *b,
                               double tol_abs, int max_it, lsmf_solve_info *info);

/* ---- allocation-free residual norm (no counterpart in the reference) ----
 * *d_norm = ||d_b - A d_x||_2 for a cached FP64 operator, computed without
 * calling cudaMalloc: for callers that cannot allocate device memory while
 * they run (their device memory is owned by another framework's caching
 * allocator, or a no-allocation-after-start-up rule applies).  The scratch
 * (A x and the reduction partials) is a static device array of
 * LSMF_NOALLOC_MAX_DOFS + 1024 doubles (16 MiB), kept by every GPU that has
 * loaded it until exit; operators with more dofs are rejected with
 * LSMF_ERR_INVALID_ARG.  Under CUDA's lazy module loading (the default) the
 * array is placed in device memory when a device first uses it, that is at
 * the first call on that device: make one call at start-up, before another
 * framework's allocator reserves the pool, or set
 * CUDA_MODULE_LOADING=EAGER.  That first call on a device should also come
 * before any stream capture.  Every call looks up the array's device address
 * (cudaGetSymbolAddress) for the operator's device, which must be current
 * (else LSMF_ERR_INVALID_ARG).  All calls share the array, so calls that
 * overlap on the GPU (different streams, no ordering between them) race.
 * Asynchronous on the operator's stream; d_norm is a device pointer to one
 * double. */
#define LSMF_NOALLOC_MAX_DOFS 2097152
lsmf_status lsmf_residual_norm_noalloc(lsmf_op *op, const double *d_x, const double *d_b, double *d_norm);

/* ---- adjoint gradient (new, no reference counterpart) ----
 * forward: solve with mu = exp(log_mu) per fine cell; J = 1/2 sum over the
 * dofs of boundary id `obj_id` of (u - u_target)^2.
 * backward: K(u)^T lambda = dJ/du with the same GMG-CG, then
 * dJ/dlog_mu_c = -lambda^T dR_int/dlog_mu_c evaluated cell by cell. */
lsmf_status lsmf_adjoint_forward(lsmf_problem *p, const double *log_mu_cell, const double *u_target,
                                 int obj_id, double *J);
lsmf_status lsmf_adjoint_backward(lsmf_problem *p, double *dJ_dlogmu);

#ifdef __cplusplus
}
#endif
#endif /* LSMF_H */
