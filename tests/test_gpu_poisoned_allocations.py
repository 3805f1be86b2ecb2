"""The solve paths with every new device buffer poisoned.

With LSMF_POISON_ALLOC set, liblsmf fills each new floating-point device
buffer (vectors, records, diagonals, level vectors) with 0xFF bytes, a NaN in
FP32 and FP64.  A value read before it is written then turns the result into
NaN, where a freshly mapped (zeroed) or finite stale buffer would hide it.
The first CG direction used to read its own buffer this way (d = 0 * d - h):
harmless on finite stale bytes, a NaN residual whenever a freed buffer that
held a NaN or an infinity was handed back.

Covered: CG with no, Jacobi and GMG preconditioning; a Newton solve and the
adjoint gradient of both formulations against the oracle; the partitioned
(two-part) Jacobi CG against the whole-mesh CG; the node-sum vmult (its
per-cell buffer) against the atomic one.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
import oracle as O  # noqa: E402
from prm_util import prm_text  # noqa: E402


@pytest.fixture(autouse=True)
def poisoned(monkeypatch):
    # read by the library at every allocation
    monkeypatch.setenv("LSMF_POISON_ALLOC", "1")


@pytest.mark.parametrize("precond", ["none", "jacobi", "gmg"])
def test_cg_with_poisoned_buffers(precond):
    gm = lsmf.Mesh("box", (1, 1, 1), 2, degree=2)
    gm.set_dirichlet([(4, 7)])
    nc, nn, nd = gm.info()
    X, _, _ = gm.arrays()
    rng = np.random.default_rng(3)
    mu = rng.choice([1.0, 10.0], size=nc)
    u = (0.02 * np.sin(np.pi * X[:, [1, 2, 0]])).reshape(-1)
    du = torch.tensor(u, device="cuda")
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    op.set_material(mu, 0.3)
    op.cache(du)
    g = None
    if precond == "gmg":
        g = lsmf.GMG(gm, "tensor4", 1, "fp32")
        g.set_material(mu, 0.3)
        g.setup(du)
    if precond == "jacobi":
        op.compute_diagonal()
    b = rng.uniform(-1, 1, nd)
    b[gm.constraint_mask() == 1] = 0
    db = torch.tensor(b, device="cuda")
    x = torch.zeros_like(db)
    tol = 1e-10 * np.linalg.norm(b)
    info = lsmf.cg_solve(op, x, db, tol, 10 * nd, precond, g, 0.65)
    assert info["converged"], info
    r = torch.empty_like(x)
    op.vmult(r, x)
    assert torch.linalg.norm(r - db).item() <= 1.01 * tol


def _adjoint_prm(formulation):
    return prm_text({
        "Polynomial degree": 2, "Quadrature order": 3, "Dimension": 3, "Type": "Box", "Box cells": "2, 2, 2",
        "Global refinement": 1, "Poisson's ratio": 0.3, "Shear modulus": 1.0, "Formulation": formulation,
        "Solver type": "MF_CG", "Preconditioner type": "gmg",
        "MF caching": "tensor4" if formulation == 1 else "scalar", "MF level precision": "double",
        "Dirichlet IDs and expressions": "4:0,0,0", "Dirichlet IDs and component mask": "4:true,true,true",
        "Neumann IDs and expressions": "5:0.02*t,0,-0.05*t", "End time": 1, "Time step size": 1,
        "Residual": 1e-10, "Tolerance force": 1e-11, "Tolerance displacement": 1e-10,
        "Max iterations Newton-Raphson": 25})


@pytest.mark.parametrize("formulation", [0, 1])
def test_newton_and_adjoint_with_poisoned_buffers(formulation):
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
    assert np.max(np.abs(grad - gref)) <= 1e-8 * np.max(np.abs(gref))


def test_partitioned_cg_with_poisoned_buffers():
    from test_gpu_dist import _problem
    gm, gop, gu, parts, rng = _problem(2, False)
    nd = gm.info()[2]
    D = lsmf.Dist.group([p["op"] for p in parts])
    b = np.where(gm.constraint_mask() == 1, 0.0, rng.uniform(-1, 1, nd))
    tol = 1e-10 * np.linalg.norm(b)
    gop.compute_diagonal()
    xg = torch.zeros(nd, dtype=torch.float64, device="cuda")
    ig = lsmf.cg_solve(gop, xg, torch.tensor(b, device="cuda"), tol, 5000, "jacobi", omega=1.0)
    assert ig["converged"]
    bs = [torch.tensor(b[p["gd"]], device="cuda") for p in parts]
    xl = [torch.zeros_like(t) for t in bs]
    info = D.cg_solve(xl, bs, tol, 5000, "jacobi", omega=1.0)
    assert info["converged"] and info["residual"] <= tol
    xg = xg.cpu().numpy()
    for p, x in zip(parts, xl):
        assert np.max(np.abs(x.cpu().numpy() - xg[p["gd"]])) <= 1e-9 * np.max(np.abs(xg))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("caching", ["tensor4", "tensor2"])
def test_nodesum_vmult_with_poisoned_buffers(precision, caching):
    # the per-cell buffer of the node-sum scatter is new device memory: every
    # slot must be written by the cell loop before the node sums read it
    gm = lsmf.Mesh("box", (3, 2, 3), 1, degree=2)
    gm.set_dirichlet([(4, 7)])
    nc, nn, nd = gm.info()
    X, _, _ = gm.arrays()
    rng = np.random.default_rng(9)
    mu = rng.choice([1.0, 10.0], size=nc)
    dt = torch.float64 if precision == "fp64" else torch.float32
    u = torch.tensor((0.02 * np.sin(np.pi * X[:, [1, 2, 0]])).reshape(-1), device="cuda", dtype=dt)
    src = torch.tensor(rng.uniform(-1, 1, nd), device="cuda", dtype=dt)
    op = lsmf.NeoHookOperator(gm, caching, 1, precision)
    op.set_material(mu, 0.3)
    op.cache(u)
    a = torch.empty_like(src)
    op.vmult(a, src)
    op.set_scatter("nodesum")
    b = torch.empty_like(src)
    op.vmult(b, src)
    assert torch.all(torch.isfinite(b))
    assert (torch.max(torch.abs(a - b)) / torch.max(torch.abs(a))).item() < (1e-13 if precision == "fp64" else 2e-6)
