"""GPU problem layer: .prm-driven load-stepping Newton on the device.

1. The reference's own 3D Cook goldens (tests/cook_3d_quad_mf, cook_3d_lin_mf:
   formulation 0, scalar caching, Jacobi-CG) through lsmf_problem: mesh size,
   volume, Newton iterations and the printed displacement to 6 digits.
2. GMG-CG Newton (FP32 and FP64 levels) against the CPU oracle's Newton,
   both solved tightly (CG 1e-10, Newton force 1e-11 / displacement 1e-10
   relative; the relative residual levels off near 4e-13 while the update
   keeps falling, so each convergence decision has a wide margin):
   identical Newton iteration counts, displacement within 1e-10 relative.
3. Inhomogeneous Dirichlet data (a displaced face) against the oracle, same
   tolerances.
4. Adjoint gradient of a top-face misfit w.r.t. the per-cell log shear
   modulus against central finite differences (20 seeded directions, step
   1e-6) within 1e-6, and entrywise against the oracle's FP64 reference
   gradient (its own adjoint solve with tau differentiated in mu) within
   1e-8, formulations 0 and 1; the same FD check on the benchmark's voids
   mesh (8^3 coarse cells minus 16 spheres, refined twice: 808,587 DoFs).
"""
import json
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
import oracle as O  # noqa: E402
from prm_util import prm_text  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("case", ["cook_3d_quad_mf", "cook_3d_lin_mf"])
def test_cook_3d_golden_on_gpu(case):
    with open(os.path.join(HERE, "golden", "cook_3d_goldens.json")) as f:
        g = json.load(f)[case]
    pb = lsmf.Problem(prm_text(g["prm"]))
    out = g["output"]
    assert pb.n_cells == out["n_cells"] and pb.n_dofs == out["n_dofs"]
    assert float("%g" % pb.volume) == out["volume"]
    res = pb.run()
    assert len(res["steps"]) == len(out["steps"])
    for s, gs in zip(res["steps"], out["steps"]):
        assert s["newton_iterations"] == gs["newton_iterations"]
        for c in range(3):
            assert float("%g" % s["point_u"][c]) == gs["displacement"][c], (case, s, gs)


# CG 1e-10 relative to the current residual: the last Newton iteration
# starts from a residual near its rounding floor, and a CG asked to reduce
# that by 1e-12 or more can stall when the V-cycle varies by rounding from
# one application to the next (atomic scatter); the convergence decisions
# are made by the update norm with wide margins either way
TIGHT = {"Residual": 1e-10, "Tolerance force": 1e-11, "Tolerance displacement": 1e-10,
         "Max iterations Newton-Raphson": 25}
TIGHT_ORACLE = dict(tol_lin=1e-10, tol_f=1e-11, tol_u=1e-10, max_nr=25)
U_TOL = 1e-10


def _cook_prm(precision, precond="gmg", caching="tensor4", end=0.4, dt=0.2):
    return prm_text(dict({
        "Polynomial degree": 2, "Quadrature order": 3, "Dimension": 3, "Type": "Cook", "Elements per edge": 2,
        "Global refinement": 1, "Grid scale": 1, "Cook thickness": 10, "Poisson's ratio": 0.3,
        "Shear modulus": 80.194, "Formulation": 1, "Solver type": "MF_CG", "Residual": 1e-8,
        "Preconditioner type": precond, "MF caching": caching, "MF level precision": precision,
        "Dirichlet IDs and expressions": "1:0,0,0", "Dirichlet IDs and component mask": "1:true,true,true",
        "Neumann IDs and expressions": "11:0,6.25*t,0", "End time": end, "Time step size": dt,
        "Output points": "48, 60, 5"}, **TIGHT))


@pytest.mark.parametrize("precision", ["float", "double"])
def test_newton_gmg_matches_oracle(precision, parity):
    pb = lsmf.Problem(_cook_prm(precision))
    res = pb.run()
    ref = O.newton(geometry=O.GEOM_COOK, coarse=(2, 2, 1), n_refinements=1, lo=(0, 0, -5), hi=(48, 44, 5),
                   scale=1.0, p=2, q=3, caching="tensor4", formulation=1, mu=80.194, nu=0.3,
                   dirichlet=[(1, 7, (0, 0, 0))], neumann=[(11, (0, 0, 0), (0, 6.25, 0))], end_time=0.4, dt=0.2,
                   precond="gmg", level_fp32=(precision == "float"), output_point=(48, 60, 5),
                   return_u=True, **TIGHT_ORACLE)
    assert ref["rc"] == 0
    assert [s["newton_iterations"] for s in res["steps"]] == [s["newton_iterations"] for s in ref["steps"]]
    for a, b in zip(res["steps"], ref["steps"]):
        assert abs(a["cg_iterations"] - b["cg_iterations"]) <= 2 * a["newton_iterations"]
    u = pb.solution()
    parity("Cook 2x2x1 GMG Newton (%s levels): displacement" % precision,
           np.max(np.abs(u - ref["u"])) / np.max(np.abs(ref["u"])), U_TOL)
    assert np.max(np.abs(u - ref["u"])) <= U_TOL * np.max(np.abs(ref["u"]))


@pytest.mark.parametrize("precision", ["float", "double"])
def test_newton_gmg_q4_matches_oracle(precision, parity):
    # Q4 elements (5^3 Gauss points) with Q4 multigrid levels
    prm = prm_text(dict({
        "Polynomial degree": 4, "Quadrature order": 5, "Dimension": 3, "Type": "Box", "Box cells": "1, 1, 1",
        "Global refinement": 2, "Poisson's ratio": 0.3, "Shear modulus": 1.0, "Formulation": 1,
        "Solver type": "MF_CG", "Preconditioner type": "gmg", "MF caching": "tensor4",
        "MF level precision": precision, "Dirichlet IDs and expressions": "4:0,0,0",
        "Dirichlet IDs and component mask": "4:true,true,true",
        "Neumann IDs and expressions": "5:0.02*t,0,-0.05*t", "End time": 1, "Time step size": 0.5}, **TIGHT))
    pb = lsmf.Problem(prm)
    res = pb.run()
    ref = O.newton(geometry=O.GEOM_BOX, coarse=(1, 1, 1), n_refinements=2, p=4, q=5, caching="tensor4",
                   formulation=1, mu=1.0, nu=0.3, dirichlet=[(4, 7, (0, 0, 0))],
                   neumann=[(5, (0, 0, 0), (0.02, 0, -0.05))], end_time=1.0, dt=0.5, precond="gmg",
                   level_fp32=(precision == "float"), return_u=True, **TIGHT_ORACLE)
    assert ref["rc"] == 0
    assert [s["newton_iterations"] for s in res["steps"]] == [s["newton_iterations"] for s in ref["steps"]]
    u = pb.solution()
    parity("Q4 box GMG Newton (%s levels): displacement" % precision,
           np.max(np.abs(u - ref["u"])) / np.max(np.abs(ref["u"])), U_TOL)
    assert np.max(np.abs(u - ref["u"])) <= U_TOL * np.max(np.abs(ref["u"]))


def test_newton_gmg_gc_equals_gmg():
    # global coarsening on a globally refined mesh builds the same levels and
    # transfers, so the solve is the same
    pb = lsmf.Problem(_cook_prm("float", precond="gmg-gc", end=0.2, dt=0.2))
    res = pb.run()
    pb2 = lsmf.Problem(_cook_prm("float", precond="gmg", end=0.2, dt=0.2))
    res2 = pb2.run()
    assert [s["newton_iterations"] for s in res["steps"]] == [s["newton_iterations"] for s in res2["steps"]]
    assert np.max(np.abs(pb.solution() - pb2.solution())) <= U_TOL * np.max(np.abs(pb2.solution()))


@pytest.mark.parametrize("caching", ["tensor2", "scalar", "scalar_referential", "tensor4_ns"])
def test_newton_other_cachings(caching):
    pb = lsmf.Problem(_cook_prm("float", caching=caching, end=0.2, dt=0.2))
    res = pb.run()
    pb4 = lsmf.Problem(_cook_prm("float", caching="tensor4", end=0.2, dt=0.2))
    res4 = pb4.run()
    assert [s["newton_iterations"] for s in res["steps"]] == [s["newton_iterations"] for s in res4["steps"]]
    assert np.max(np.abs(pb.solution() - pb4.solution())) <= U_TOL * np.max(np.abs(pb4.solution()))


def test_inhomogeneous_dirichlet_matches_oracle(parity):
    prm = prm_text(dict({
        "Polynomial degree": 2, "Quadrature order": 3, "Dimension": 3, "Type": "Box", "Box cells": "2, 2, 2",
        "Global refinement": 1, "Poisson's ratio": 0.3, "Shear modulus": 1.0, "Formulation": 1,
        "Solver type": "MF_CG", "Residual": 1e-8, "Preconditioner type": "gmg", "MF caching": "tensor4",
        "Dirichlet IDs and expressions": "4:0,0,0;5:0,0,-0.01",
        "Dirichlet IDs and component mask": "4:true,true,true;5:false,false,true",
        "End time": 0.2, "Time step size": 0.1, "Output points": "0.5, 0.5, 1"}, **TIGHT))
    pb = lsmf.Problem(prm)
    res = pb.run()
    ref = O.newton(geometry=O.GEOM_BOX, coarse=(2, 2, 2), n_refinements=1, caching="tensor4", formulation=1,
                   mu=1.0, nu=0.3, dirichlet=[(4, 7, (0, 0, 0)), (5, 4, (0, 0, -0.01))], end_time=0.2, dt=0.1,
                   precond="gmg", output_point=(0.5, 0.5, 1.0), return_u=True, **TIGHT_ORACLE)
    assert ref["rc"] == 0
    assert [s["newton_iterations"] for s in res["steps"]] == [s["newton_iterations"] for s in ref["steps"]]
    u = pb.solution()
    parity("displaced face Newton: displacement", np.max(np.abs(u - ref["u"])) / np.max(np.abs(ref["u"])), U_TOL)
    assert np.max(np.abs(u - ref["u"])) <= U_TOL * np.max(np.abs(ref["u"]))
    # the top face moved by the two imposed increments
    assert abs(res["steps"][-1]["point_u"][2] + 0.02) < 1e-12


def _adjoint_prm(formulation=1):
    # the tight tolerances of the Newton parity tests: converged through the
    # update norm well before the relative residual reaches its rounding
    # floor (a CG asked to reduce a floor-level residual by 1e-13 can stall)
    return prm_text(dict({
        "Polynomial degree": 2, "Quadrature order": 3, "Dimension": 3, "Type": "Box", "Box cells": "2, 2, 2",
        "Global refinement": 1, "Poisson's ratio": 0.3, "Shear modulus": 1.0, "Formulation": formulation,
        "Solver type": "MF_CG", "Preconditioner type": "gmg",
        "MF caching": "tensor4" if formulation == 1 else "scalar", "MF level precision": "double",
        "Dirichlet IDs and expressions": "4:0,0,0", "Dirichlet IDs and component mask": "4:true,true,true",
        "Neumann IDs and expressions": "5:0.02*t,0,-0.05*t", "End time": 1, "Time step size": 1}, **TIGHT))


def test_adjoint_gradient_matches_finite_differences(parity):
    pb = lsmf.Problem(_adjoint_prm())
    rng = np.random.default_rng(11)
    theta = rng.normal(0.0, 0.3, pb.n_cells)
    target = rng.uniform(-1e-3, 1e-3, pb.n_dofs)
    J0 = pb.adjoint_forward(theta, target, 5)
    grad = pb.adjoint_backward()
    assert np.all(np.isfinite(grad)) and np.max(np.abs(grad)) > 0
    h = 1e-6
    fd, ad = [], []
    for k in range(20):
        v = rng.normal(size=pb.n_cells)
        v /= np.linalg.norm(v)
        jp = pb.adjoint_forward(theta + h * v, target, 5)
        jm = pb.adjoint_forward(theta - h * v, target, 5)
        fd.append((jp - jm) / (2 * h))
        ad.append(grad @ v)
    fd, ad = np.array(fd), np.array(ad)
    parity("adjoint vs central FD, 4^3 Q2, 20 unit directions", np.max(np.abs(fd - ad)) / np.max(np.abs(fd)), 1e-6)
    assert np.max(np.abs(fd - ad)) <= 1e-6 * np.max(np.abs(fd)), (fd, ad)
    # FP64 reference objective from the oracle's Newton solve
    ref = O.newton(geometry=O.GEOM_BOX, coarse=(2, 2, 2), n_refinements=1, caching="tensor4", formulation=1,
                   mu=1.0, mu_fine=np.exp(theta), nu=0.3, dirichlet=[(4, 7, (0, 0, 0))],
                   neumann=[(5, (0, 0, 0), (0.02, 0, -0.05))], end_time=1.0, dt=1.0, precond="gmg",
                   level_fp32=False, return_u=True, **TIGHT_ORACLE)
    gm = lsmf.Mesh("box", (2, 2, 2), 1, degree=2)
    X, _, _ = gm.arrays()
    top = np.repeat(np.isclose(X[:, 2], 1.0), 3)
    Jref = 0.5 * np.sum((ref["u"][top] - target[top]) ** 2)
    assert abs(J0 - Jref) <= 1e-9 * abs(Jref)


@pytest.mark.parametrize("formulation", [0, 1])
def test_adjoint_gradient_matches_oracle_gradient(formulation, parity):
    """Per-cell gradient against the oracle's FP64 reference gradient."""
    pb = lsmf.Problem(_adjoint_prm(formulation))
    rng = np.random.default_rng(23)
    theta = rng.normal(0.0, 0.3, pb.n_cells)
    target = rng.uniform(-1e-3, 1e-3, pb.n_dofs)
    J = pb.adjoint_forward(theta, target, 5)
    grad = pb.adjoint_backward()
    Jref, gref, uref = O.adjoint(theta, target, 5, geometry=O.GEOM_BOX, coarse=(2, 2, 2), n_refinements=1,
                                 caching="tensor4" if formulation == 1 else "scalar", formulation=formulation,
                                 mu=1.0, nu=0.3, dirichlet=[(4, 7, (0, 0, 0))],
                                 neumann=[(5, (0, 0, 0), (0.02, 0, -0.05))], end_time=1.0, dt=1.0,
                                 tol_lin=1e-10, tol_f=1e-11, tol_u=1e-10, max_nr=25, precond="gmg",
                                 level_fp32=False)
    assert abs(J - Jref) <= 1e-10 * Jref
    assert np.max(np.abs(pb.solution() - uref)) <= 1e-10 * np.max(np.abs(uref))
    parity("adjoint gradient vs oracle FP64 gradient, formulation %d" % formulation,
           np.max(np.abs(grad - gref)) / np.max(np.abs(gref)), 1e-8)
    assert np.max(np.abs(grad - gref)) <= 1e-8 * np.max(np.abs(gref)), np.max(np.abs(grad - gref))


def test_adjoint_config_size_finite_differences(parity):
    """The adjoint benchmark workload (the voids mesh reduced to ~1 M DoFs:
    8^3 coarse cells minus the 16 seeded spheres, refined twice, 808,587
    DoFs; log mu ~ N(0, 0.3^2), top-face misfit): 20 seeded +-1 directions
    (each cell's log mu moves by the step 1e-6), max |fd - g.v| <= 1e-6
    max |fd|."""
    import bench
    pb = lsmf.Problem(bench.adjoint_prm())
    om = O.Mesh(O.GEOM_BOX, (8, 8, 8), 2, (0, 0, 0), (1, 1, 1), 1.0, 2, 3,
                coarse_active=O.void_mask((8, 8, 8), 16, 0.08, 2024))
    assert (pb.n_cells, pb.n_dofs) == (om.n_cells, om.n_dofs) == (31872, 808587)
    rng = np.random.default_rng(4321)
    theta = rng.normal(0.0, 0.3, pb.n_cells)
    target = rng.uniform(-1e-3, 1e-3, pb.n_dofs)
    pb.adjoint_forward(theta, target, 5)
    grad = pb.adjoint_backward()
    fd, ad = bench.fd_check(pb, theta, target, grad, rng, 20, 1e-6)
    parity("adjoint vs central FD, voids 32^3 Q2 (808,587 DoFs), 20 directions, h = 1e-6",
           np.max(np.abs(fd - ad)) / np.max(np.abs(fd)), 1e-6)
    assert np.max(np.abs(fd - ad)) <= 1e-6 * np.max(np.abs(fd)), (fd, ad)
