"""GPU parity of the multigrid preconditioner and the CG solver against the
CPU oracle (same meshes, materials, displacement, right-hand sides).

Tolerances: FP64 level operators within 1e-10 relative of the oracle's FP64
V-cycle; FP32 level operators within 1e-4 of the oracle's FP32 V-cycle.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
import oracle as O  # noqa: E402


def _problem(caching="tensor4", formulation=1, p=2, coarse=(1, 1, 1), nref=2, seed=5, geometry="box"):
    rng = np.random.default_rng(seed)
    if geometry == "box":
        lo, hi, dirichlet = (0, 0, 0), (1, 1, 1), [(4, 7)]
    else:
        lo, hi, dirichlet = (0, 0, -5), (48, 44, 5), [(1, 7)]
    gm = lsmf.Mesh(geometry, coarse, nref, lo=lo, hi=hi, degree=p)
    gm.set_dirichlet(dirichlet)
    nc, nn, nd = gm.info()
    X, _, _ = gm.arrays()
    mu = rng.choice([1.0, 10.0], size=nc)
    amp = 0.02 * (hi[0] - lo[0])
    u = (amp * np.sin(np.pi * X[:, [1, 2, 0]] / np.array(hi)[None, [1, 2, 0]].clip(1))).reshape(-1)
    return gm, mu, u, dirichlet, (lo, hi), rng


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("caching,formulation", [("tensor4", 1), ("tensor2", 1), ("scalar", 1), ("scalar", 0),
                                                 ("scalar_referential", 1), ("tensor4_ns", 1)])
def test_vcycle_matches_oracle(precision, caching, formulation):
    gm, mu, u, dirichlet, (lo, hi), rng = _problem(caching, formulation)
    og = O.GMG(O.GEOM_BOX, (1, 1, 1), 2, lo, hi, 1.0, 2, 3, caching, formulation, precision == "fp32", mu, 0.3,
               dirichlet, u)
    g = lsmf.GMG(gm, caching, formulation, precision)
    g.set_material(mu, 0.3)
    du = torch.tensor(u, device="cuda")
    g.setup(du)
    for l in range(gm.n_levels):
        a, b = g.level_info(l), og.level_info(l)
        assert a[2] == b[2], (l, a, b)   # Chebyshev degree
        tol = 1e-9 if precision == "fp64" else 2e-3
        assert abs(a[0] - b[0]) <= tol * abs(b[1]) and abs(a[1] - b[1]) <= tol * abs(b[1]), (l, a, b)
    src = rng.uniform(-1, 1, u.size)
    src[gm.constraint_mask() == 1] = 0
    dsrc = torch.tensor(src, device="cuda")
    ddst = torch.empty_like(dsrc)
    g.vmult(ddst, dsrc)
    got, want = ddst.cpu().numpy(), og.vmult(src)
    tol = 1e-10 if precision == "fp64" else 1e-4
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want))
    # the V-cycle replayed as a CUDA graph equals the kernel-by-kernel launch
    # (up to the order of the floating-point atomics)
    g.set_graph(False)
    d2 = torch.empty_like(dsrc)
    g.vmult(d2, dsrc)
    assert torch.max(torch.abs(d2 - ddst)).item() <= (1e-12 if precision == "fp64" else 1e-5) * np.max(np.abs(got))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("coarse_chebyshev", [True, False])
def test_vcycle_large_coarse_level(precision, coarse_chebyshev):
    # a 6^3-cell coarse level: a high-degree coarse Chebyshev (or the coarse
    # CG with its Chebyshev preconditioner) over many blocks
    gm, mu, u, dirichlet, (lo, hi), rng = _problem("tensor4", 1, coarse=(6, 6, 6), nref=1)
    og = O.GMG(O.GEOM_BOX, (6, 6, 6), 1, lo, hi, 1.0, 2, 3, "tensor4", 1, precision == "fp32", mu, 0.3,
               dirichlet, u, coarse_chebyshev=coarse_chebyshev)
    g = lsmf.GMG(gm, "tensor4", 1, precision, coarse_chebyshev=coarse_chebyshev)
    g.set_material(mu, 0.3)
    du = torch.tensor(u, device="cuda")
    g.setup(du)
    a, b = g.level_info(0), og.level_info(0)
    assert a[2] == b[2] and (a[2] > 20 or not coarse_chebyshev), (a, b)
    src = rng.uniform(-1, 1, u.size)
    src[gm.constraint_mask() == 1] = 0
    dsrc = torch.tensor(src, device="cuda")
    ddst = torch.empty_like(dsrc)
    g.vmult(ddst, dsrc)
    got, want = ddst.cpu().numpy(), og.vmult(src)
    tol = 1e-10 if precision == "fp64" else 1e-4
    assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vcycle_graph_follows_each_setup(precision):
    # the executable V-cycle graph outlives a set-up and is updated in place
    # from the next capture (or instantiated again when the coarse degree
    # changes): after every set-up the replayed V-cycle is the new one
    gm, mu, u, dirichlet, (lo, hi), rng = _problem("tensor4", 1, coarse=(6, 6, 6), nref=1)
    g = lsmf.GMG(gm, "tensor4", 1, precision)
    g.set_material(mu, 0.3)
    src = rng.uniform(-1, 1, u.size)
    src[gm.constraint_mask() == 1] = 0
    dsrc = torch.tensor(src, device="cuda")
    tol = 1e-10 if precision == "fp64" else 1e-4
    for scale in (1.0, 1.0, 2.5, 0.5):
        us = scale * u
        g.setup(torch.tensor(us, device="cuda"))
        ddst = torch.empty_like(dsrc)
        g.vmult(ddst, dsrc)
        og = O.GMG(O.GEOM_BOX, (6, 6, 6), 1, lo, hi, 1.0, 2, 3, "tensor4", 1, precision == "fp32", mu, 0.3,
                   dirichlet, us)
        assert g.level_info(0)[2] == og.level_info(0)[2]
        want = og.vmult(src)
        assert np.max(np.abs(ddst.cpu().numpy() - want)) <= tol * np.max(np.abs(want)), scale


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [1, 3, 4])
@pytest.mark.parametrize("caching", ["tensor4", "tensor2", "scalar_referential"])
def test_vcycle_other_degrees_match_oracle(precision, p, caching):
    # h-multigrid with Q_p on every level (the transfer maps of degree p, the
    # level operators' sweeps of degree p; FP32 tensor2 at Q1 and
    # scalar_referential at Q4 run the cell-pair kernel by default)
    coarse, nref = ((2, 2, 2), 2) if p == 1 else ((1, 1, 1), 2)
    gm, mu, u, dirichlet, (lo, hi), rng = _problem(caching, 1, p=p, coarse=coarse, nref=nref)
    og = O.GMG(O.GEOM_BOX, coarse, nref, lo, hi, 1.0, p, p + 1, caching, 1, precision == "fp32", mu, 0.3,
               dirichlet, u)
    g = lsmf.GMG(gm, caching, 1, precision)
    g.set_material(mu, 0.3)
    g.setup(torch.tensor(u, device="cuda"))
    tol = 1e-9 if precision == "fp64" else 2e-3
    for l in range(gm.n_levels):
        a, b = g.level_info(l), og.level_info(l)
        assert a[2] == b[2], (l, a, b)
        assert abs(a[0] - b[0]) <= tol * abs(b[1]) and abs(a[1] - b[1]) <= tol * abs(b[1]), (l, a, b)
    src = rng.uniform(-1, 1, u.size)
    src[gm.constraint_mask() == 1] = 0
    dsrc = torch.tensor(src, device="cuda")
    ddst = torch.empty_like(dsrc)
    g.vmult(ddst, dsrc)
    want = og.vmult(src)
    vtol = 1e-10 if precision == "fp64" else 1e-4
    assert np.max(np.abs(ddst.cpu().numpy() - want)) <= vtol * np.max(np.abs(want))


def test_vcycle_cook_geometry():
    gm, mu, u, dirichlet, (lo, hi), rng = _problem("tensor4", 1, coarse=(2, 2, 1), nref=1, geometry="cook")
    og = O.GMG(O.GEOM_COOK, (2, 2, 1), 1, lo, hi, 1.0, 2, 3, "tensor4", 1, False, mu, 0.3, dirichlet, u)
    g = lsmf.GMG(gm, "tensor4", 1, "fp64")
    g.set_material(mu, 0.3)
    g.setup(torch.tensor(u, device="cuda"))
    src = rng.uniform(-1, 1, u.size)
    dsrc = torch.tensor(src, device="cuda")
    ddst = torch.empty_like(dsrc)
    g.vmult(ddst, dsrc)
    want = og.vmult(src)
    assert np.max(np.abs(ddst.cpu().numpy() - want)) <= 1e-10 * np.max(np.abs(want))


@pytest.mark.parametrize("precond", ["gmg", "jacobi", "none"])
def test_cg_solves_to_tolerance(precond):
    gm, mu, u, dirichlet, _, rng = _problem("tensor4", 1)
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    op.set_material(mu, 0.3)
    du = torch.tensor(u, device="cuda")
    op.cache(du)
    g = None
    if precond == "gmg":
        g = lsmf.GMG(gm, "tensor4", 1, "fp32")
        g.set_material(mu, 0.3)
        g.setup(du)
    if precond == "jacobi":
        op.compute_diagonal()
    b = rng.uniform(-1, 1, u.size)
    b[gm.constraint_mask() == 1] = 0
    db = torch.tensor(b, device="cuda")
    x = torch.zeros_like(db)
    tol = 1e-10 * np.linalg.norm(b)
    info = lsmf.cg_solve(op, x, db, tol, 10 * u.size, precond, g, 0.65)
    assert info["converged"], info
    r = torch.empty_like(x)
    op.vmult(r, x)
    assert torch.linalg.norm(r - db).item() <= 1.01 * tol
    # the oracle operator agrees on the solution
    om = O.Mesh(O.GEOM_BOX, (1, 1, 1), 2, (0, 0, 0), (1, 1, 1), 1.0, 2, 3)
    ref = O.Operator(om, "tensor4", 1)
    ref.set_material(mu, 0.3)
    ref.set_constraints(gm.constraint_mask())
    ref.cache(u)
    assert np.linalg.norm(ref.vmult(x.cpu().numpy()) - b) <= 1e-8 * np.linalg.norm(b)
    if precond == "gmg":
        assert info["iterations"] < 40


def test_cg_reports_non_convergence():
    gm, mu, u, dirichlet, _, rng = _problem("tensor4", 1)
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    op.set_material(mu, 0.3)
    op.cache(torch.tensor(u, device="cuda"))
    b = torch.tensor(rng.uniform(-1, 1, u.size), device="cuda")
    x = torch.zeros_like(b)
    info = lsmf.cg_solve(op, x, b, 1e-14, 3, "none")
    assert not info["converged"] and info["status"] == 5 and info["iterations"] == 3


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vcycle_coarse_cg_matches_oracle(precision):
    """'MF Chebyshev coarse = false': CG preconditioned by the level-0 Chebyshev
    smoother to a 1e-3 reduction (MGCoarseGridIterativeSolver)."""
    gm, mu, u, dirichlet, (lo, hi), rng = _problem("tensor4", 1)
    og = O.GMG(O.GEOM_BOX, (1, 1, 1), 2, lo, hi, 1.0, 2, 3, "tensor4", 1, precision == "fp32", mu, 0.3,
               dirichlet, u, coarse_chebyshev=False)
    g = lsmf.GMG(gm, "tensor4", 1, precision, coarse_chebyshev=False)
    g.set_material(mu, 0.3)
    g.setup(torch.tensor(u, device="cuda"))
    assert g.level_info(0)[2] == og.level_info(0)[2] == 5
    src = rng.uniform(-1, 1, u.size)
    src[gm.constraint_mask() == 1] = 0
    dsrc = torch.tensor(src, device="cuda")
    ddst = torch.empty_like(dsrc)
    g.vmult(ddst, dsrc)
    want = og.vmult(src)
    tol = 1e-9 if precision == "fp64" else 1e-4
    assert np.max(np.abs(ddst.cpu().numpy() - want)) <= tol * np.max(np.abs(want))

