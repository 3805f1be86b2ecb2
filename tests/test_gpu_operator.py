"""GPU parity of the tangent operator (cache / vmult / diagonal) against the
CPU oracle on seeded inputs, through the C ABI of include/lsmf.h.

Tolerances: FP64 vmult and diagonal within 1e-10 relative (max norm) of the
FP64 oracle; FP32 within 2e-5 relative of the FP64 oracle.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
import oracle as O  # noqa: E402

FP64_TOL = 1e-10
FP32_TOL = 2e-5


def _setup(p=2, coarse=(2, 2, 2), level=1, seed=0, amp=0.01):
    rng = np.random.default_rng(seed)
    gm = lsmf.Mesh("box", coarse, level, degree=p)
    gm.set_dirichlet([(4, 7)])  # bottom face clamped
    om = O.Mesh(O.GEOM_BOX, coarse, level, (0, 0, 0), (1, 1, 1), 1.0, p, p + 1)
    X, cn, ijk = gm.arrays()
    assert np.array_equal(X, om.X) and np.array_equal(cn, om.cell_nodes) and np.array_equal(ijk, om.cell_ijk)
    cmask = gm.constraint_mask()
    assert np.array_equal(cmask, om.constraints([(4, 7)]))
    mu = rng.choice([1.0, 10.0], size=om.n_cells)
    u = rng.uniform(-amp, amp, size=om.n_dofs)
    src = rng.uniform(-1, 1, size=om.n_dofs)
    return gm, om, cmask, mu, u, src


def _oracle_op(om, cmask, mu, u, caching, formulation, fp32=False):
    op = O.Operator(om, caching, formulation, fp32=fp32)
    op.set_material(mu, 0.3)
    op.set_constraints(cmask)
    assert op.cache(u.astype(np.float32) if fp32 else u) == 0
    return op


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


VARIANTS = [("tensor4", 1), ("tensor2", 1), ("scalar", 1), ("scalar", 0), ("scalar_referential", 1),
            ("tensor4_ns", 1)]


KERNELS = ["bulk1", "bulk2", "bulk3", "plain", "basic"]
# FP32 also has the cell-pair kernel (two cells per warp, packed f32x2)
KERNELS32 = KERNELS + ["pairs"]


def _select(op, kernel):
    # the one-cell kernels are selected with pairs off (the default turns
    # them on for some FP32 variants; FP64 operators ignore the option)
    op.set_cell_pairs(1 if kernel == "pairs" else 0)
    if kernel == "basic":
        op.set_basic_kernel(True)
    elif kernel != "pairs":
        op.set_pipeline({"bulk1": 1, "bulk2": 2, "bulk3": 3, "plain": 0}[kernel])


@pytest.mark.parametrize("caching,formulation", VARIANTS)
@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("kernel", KERNELS)
def test_vmult_fp64_matches_oracle(caching, formulation, p, kernel):
    gm, om, cmask, mu, u, src = _setup(p=p, coarse=(2, 2, 2) if p < 4 else (1, 2, 1), level=1 if p < 4 else 1)
    ref = _oracle_op(om, cmask, mu, u, caching, formulation)
    op = lsmf.NeoHookOperator(gm, caching, formulation, "fp64")
    _select(op, kernel)
    op.set_material(mu, 0.3)
    du = torch.tensor(u, device="cuda")
    op.cache(du)
    dsrc = torch.tensor(src, device="cuda")
    ddst = torch.empty_like(dsrc)
    op.vmult(ddst, dsrc)
    got = ddst.cpu().numpy()
    want = ref.vmult(src)
    assert _rel(got, want) < FP64_TOL
    # constrained rows are identity (mf_nh_operator.h:702-705)
    assert np.array_equal(got[cmask == 1], src[cmask == 1])
    # vmult_add accumulates
    op.vmult_add(ddst, dsrc)
    assert _rel(ddst.cpu().numpy(), 2 * want) < FP64_TOL


@pytest.mark.parametrize("caching,formulation", VARIANTS)
@pytest.mark.parametrize("p", [1, 2, 3, 4])
@pytest.mark.parametrize("kernel", KERNELS32)
def test_vmult_fp32_matches_oracle(caching, formulation, p, kernel):
    gm, om, cmask, mu, u, src = _setup(p=p, coarse=(2, 2, 2) if p < 4 else (1, 2, 1), level=1)
    ref = _oracle_op(om, cmask, mu, u, caching, formulation)
    op = lsmf.NeoHookOperator(gm, caching, formulation, "fp32")
    _select(op, kernel)
    op.set_material(mu, 0.3)
    du = torch.tensor(u, device="cuda", dtype=torch.float32)
    op.cache(du)
    dsrc = torch.tensor(src, device="cuda", dtype=torch.float32)
    ddst = torch.empty_like(dsrc)
    op.vmult(ddst, dsrc)
    assert _rel(ddst.cpu().numpy().astype(np.float64), ref.vmult(src)) < FP32_TOL


@pytest.mark.parametrize("caching,formulation", VARIANTS)
def test_cache_tables_match_oracle(caching, formulation):
    gm, om, cmask, mu, u, src = _setup(p=2)
    ref = _oracle_op(om, cmask, mu, u, caching, formulation)
    op = lsmf.NeoHookOperator(gm, caching, formulation, "fp64")
    op.set_material(mu, 0.3)
    du = torch.tensor(u, device="cuda")
    op.cache(du)
    whichs = {"tensor4": [2, 3, 4], "tensor2": [0, 1, 2, 4], "scalar": [0, 4, 5],
              "scalar_referential": [0, 4, 5, 6], "tensor4_ns": [4, 7]}[caching]
    # tensor4 / tensor2 / tensor4_ns store their coefficients times JxW and
    # no JxW table
    folded = caching in ("tensor4", "tensor2", "tensor4_ns")
    jxw = ref.table(5)
    for w in whichs:
        want = ref.table(w)
        if folded and w != 4:
            want = (want.reshape(jxw.size, -1) * jxw[:, None]).reshape(-1)
        assert _rel(op.table(w), want) < 1e-13, w
    if folded:
        with pytest.raises(lsmf.LsmfError):
            op.table(5)


@pytest.mark.parametrize("caching,formulation", VARIANTS)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_diagonal_matches_oracle(caching, formulation, precision):
    gm, om, cmask, mu, u, src = _setup(p=2)
    ref = _oracle_op(om, cmask, mu, u, caching, formulation)
    d_ref, inv_ref = ref.diagonal()
    op = lsmf.NeoHookOperator(gm, caching, formulation, precision)
    op.set_material(mu, 0.3)
    dt = torch.float32 if precision == "fp32" else torch.float64
    du = torch.tensor(u, device="cuda", dtype=dt)
    op.cache(du)
    op.compute_diagonal()
    tol = FP64_TOL if precision == "fp64" else FP32_TOL
    assert _rel(op.get_matrix_diagonal().cpu().numpy().astype(np.float64), d_ref) < tol
    assert _rel(op.get_matrix_diagonal_inverse().cpu().numpy().astype(np.float64), inv_ref) < tol
    # Jacobi: dst = omega D^-1 src
    dsrc = torch.tensor(src, device="cuda", dtype=dt)
    ddst = torch.empty_like(dsrc)
    op.precondition_Jacobi(ddst, dsrc, 0.65)
    assert _rel(ddst.cpu().numpy().astype(np.float64), 0.65 * inv_ref * src) < tol


def test_cook_geometry_vmult():
    """Non-affine (bilinear Cook) cells exercise the per-point metric."""
    rng = np.random.default_rng(3)
    gm = lsmf.Mesh("cook", (4, 4, 1), 1, lo=(0, 0, -5), hi=(48, 44, 5), degree=2)
    gm.set_dirichlet([(1, 7)])
    om = O.Mesh(O.GEOM_COOK, (4, 4, 1), 1, (0, 0, -5), (48, 44, 5), 1.0, 2, 3)
    cmask = om.constraints([(1, 7)])
    assert np.array_equal(cmask, gm.constraint_mask())
    u = rng.uniform(-0.3, 0.3, om.n_dofs)
    src = rng.uniform(-1, 1, om.n_dofs)
    for caching, form in VARIANTS:
        ref = _oracle_op(om, cmask, 80.194, u, caching, form)
        op = lsmf.NeoHookOperator(gm, caching, form, "fp64")
        op.set_material(np.full(om.n_cells, 80.194), 0.3)
        du = torch.tensor(u, device="cuda")
        op.cache(du)
        dsrc = torch.tensor(src, device="cuda")
        ddst = torch.empty_like(dsrc)
        op.vmult(ddst, dsrc)
        assert _rel(ddst.cpu().numpy(), ref.vmult(src)) < FP64_TOL, caching


def test_stage_mask_breakdown():
    """vmult<mask> stages: RW only gives identity rows only; SF without QD gives zero."""
    gm, om, cmask, mu, u, src = _setup(p=2)
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    op.set_material(mu, 0.3)
    du = torch.tensor(u, device="cuda")
    op.cache(du)
    dsrc = torch.tensor(src, device="cuda")
    ddst = torch.full_like(dsrc, 7.0)
    op.vmult(ddst, dsrc, lsmf.MASK_ZERO | lsmf.MASK_RW | lsmf.MASK_SF)
    got = ddst.cpu().numpy()
    want = np.where(cmask == 1, src, 0.0)
    assert np.array_equal(got, want)


def test_detf_nonpositive_reported():
    """A displacement with det F < 0 returns LSMF_ERR_DETF_NONPOSITIVE (host-side check of the device flag)."""
    gm, om, cmask, mu, u, src = _setup(p=2)
    X, _, _ = gm.arrays()
    bad = torch.tensor((-2.0 * X).reshape(-1), device="cuda")  # F = -I
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    op.set_material(mu, 0.3)
    with pytest.raises(lsmf.LsmfError) as e:
        op.cache(bad)
    assert e.value.status == 3
    dsrc = torch.tensor(src, device="cuda")
    with pytest.raises(lsmf.LsmfError) as e:
        op.vmult(torch.empty_like(dsrc), dsrc)
    assert e.value.status == 4


def test_cached_volume_ratio_matches_det_f():
    """The reference's consistency check of the formulation-0 cache
    (mf_nh_operator.h:1131-1156): at every point JxW_ref / JxW_cur * det F
    = 1, with det F = c^-3 from the cached c = J^(-1/3).  On the box mesh the
    reference JxW is h^3 times the Gauss weight of the point."""
    gm, om, cmask, mu, u, src = _setup(p=2, coarse=(2, 2, 2), level=1)
    op = lsmf.NeoHookOperator(gm, "scalar", 0, "fp64")
    op.set_material(mu, 0.3)
    op.cache(torch.tensor(u, device="cuda"))
    c = op.table(0).reshape(-1, 27)
    jxw = op.table(5).reshape(-1, 27)
    g = np.array([5.0, 8.0, 5.0]) / 18.0  # 3-point Gauss weights on [0, 1]
    wq = (g[None, None, :] * g[None, :, None] * g[:, None, None]).reshape(-1)  # q = qx + 3 qy + 9 qz
    h = 0.25
    ratio = (h ** 3 * wq[None, :]) / jxw * c ** -3.0
    assert np.max(np.abs(ratio - 1.0)) < 1e-12
