"""GPU tests of the chunked vmult cell loop (LSMF_OPT_CHUNKS): the cells in
2..8 contiguous chunks on the operator's own streams, each chunk zeroing
its range of dst and applying the identity rows there before its cells run
(once the next chunk has zeroed its range).

* For every caching variant, FP64 and FP32, degrees 1 / 2 / 4 and chunk
  counts 2 / 3 / 8, the chunked vmult equals the one-launch vmult to the
  rounding of the atomic summation order (1e-13 FP64, 1e-6 FP32), keeps the
  identity rows, writes every entry of a NaN-filled dst, and vmult_add
  accumulates through it.
* On a mesh with voids (compacted node numbers) the same holds.
* Levels with fewer than 1024 cells per chunk run in one piece (same result).
* The cells-only loop of the multigrid smoothers and transfers runs chunked
  too: a V-cycle replayed from its CUDA graph equals the unchunked one.
* The option is validated.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
import oracle as O  # noqa: E402
from test_gpu_operator import VARIANTS  # noqa: E402


def _mesh(p, coarse, level, voids=False):
    act = O.void_mask(coarse, 3, 0.2, 5) if voids else None
    gm = lsmf.Mesh("box", coarse, level, degree=p, coarse_active=act)
    gm.set_dirichlet([(4, 7), (5, 4)])
    return gm


def _op(gm, caching, formulation, precision, seed=0):
    nc, nn, nd = gm.info()
    X, _, _ = gm.arrays()
    rng = np.random.default_rng(seed)
    dt = torch.float64 if precision == "fp64" else torch.float32
    op = lsmf.NeoHookOperator(gm, caching, formulation, precision)
    op.set_material(rng.choice([1.0, 10.0], nc), 0.3)
    u = torch.tensor((0.01 * np.sin(np.pi * X[:, [1, 2, 0]])).reshape(-1), device="cuda", dtype=dt)
    op.cache(u)
    src = torch.tensor(rng.uniform(-1, 1, nd), device="cuda", dtype=dt)
    return op, src


def _check(gm, op, src, precision, ks):
    tol = 1e-13 if precision == "fp64" else 1e-6
    op.set_chunks(1)
    want = torch.empty_like(src)
    op.vmult(want, src)
    cm = torch.tensor(gm.constraint_mask() == 1, device="cuda")
    for k in ks:
        op.set_chunks(k)
        got = torch.full_like(src, float("nan"))
        op.vmult(got, src)
        torch.cuda.synchronize()
        assert torch.all(torch.isfinite(got)), k
        assert (torch.max(torch.abs(got - want)) / torch.max(torch.abs(want))).item() < tol, k
        # identity rows (mf_nh_operator.h:702-705)
        assert torch.equal(got[cm], src[cm])
        op.vmult_add(got, src)
        assert (torch.max(torch.abs(got - 2 * want)) / torch.max(torch.abs(want))).item() < tol, k
    op.set_chunks(-1)


@pytest.mark.parametrize("caching,formulation", VARIANTS)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_chunks_equal_one_launch_q2(caching, formulation, precision):
    gm = _mesh(2, (3, 3, 3), 3)  # 24^3 cells: 1728 per chunk at 8 chunks
    op, src = _op(gm, caching, formulation, precision)
    _check(gm, op, src, precision, (2, 3, 8))


@pytest.mark.parametrize("p,coarse,level", [(1, (4, 4, 4), 3), (4, (2, 2, 4), 3)])
@pytest.mark.parametrize("caching,formulation", [("tensor4", 1), ("scalar", 1), ("tensor2", 1)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_chunks_other_degrees(p, coarse, level, caching, formulation, precision):
    gm = _mesh(p, coarse, level)
    op, src = _op(gm, caching, formulation, precision)
    _check(gm, op, src, precision, (2, 4))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_chunks_with_voids(precision):
    gm = _mesh(2, (4, 4, 4), 2, voids=True)
    op, src = _op(gm, "tensor4", 1, precision)
    _check(gm, op, src, precision, (2, 3, 4))


def test_small_level_runs_in_one_piece():
    gm = _mesh(2, (2, 2, 2), 2)  # 512 cells
    op, src = _op(gm, "tensor4", 1, "fp64")
    _check(gm, op, src, "fp64", (2, 8))


def test_effective_chunk_count():
    # automatic: one launch below 32,768 cells, 2 from there (tensor4); an
    # explicit count where the level has 1024 cells per chunk, else 1
    small = _mesh(2, (3, 3, 3), 3)  # 13,824 cells
    op, _ = _op(small, "tensor4", 1, "fp64")
    assert op.get_option(8) == 1
    op.set_chunks(3)
    assert op.get_option(8) == 3
    op.set_chunks(8)
    assert op.get_option(8) == 8
    op.set_scatter("colour8")  # deterministic scatters run unchunked
    assert op.get_option(8) == 1
    big = _mesh(1, (4, 4, 4), 3)  # 32,768 Q1 cells
    op2, src = _op(big, "tensor4", 1, "fp32")
    assert op2.get_option(8) == 2
    tiny = _mesh(2, (2, 2, 2), 1)
    op3, _ = _op(tiny, "tensor4", 1, "fp64")
    op3.set_chunks(8)
    assert op3.get_option(8) == 1


def test_multigrid_levels_start_unchunked():
    # the operators a GMG object creates run their cell loops in one launch
    # unless the option is set on a level
    import ctypes
    mesh = lsmf.Mesh("box", (8, 8, 8), 2, degree=2)  # fine level 32,768 cells
    mesh.set_dirichlet([(4, 7)])
    g = lsmf.GMG(mesh, "tensor4", 1, "fp32")
    h, v = lsmf.vp(), ctypes.c_int()
    assert lsmf.lib().lsmf_gmg_level_operator(g.h, 2, ctypes.byref(h)) == 0
    assert lsmf.lib().lsmf_operator_get_option(h, 8, ctypes.byref(v)) == 0
    assert v.value == 1
    g.level_option(2, 8, -1)
    assert lsmf.lib().lsmf_operator_get_option(h, 8, ctypes.byref(v)) == 0
    assert v.value == 2


def test_get_option_reports_what_was_set():
    gm = _mesh(2, (2, 2, 2), 1)
    op, src = _op(gm, "tensor4", 1, "fp32")
    for opt, val in ((1, 2), (2, 1), (3, 6), (4, 1000), (6, 0), (7, 1)):
        lsmf.lib().lsmf_operator_set_option(op.h, opt, val)
        assert op.get_option(opt) == val, opt
    op.set_scatter("nodesum")
    assert op.get_option(5) == 2
    with pytest.raises(lsmf.LsmfError):
        op.get_option(99)


def test_option_validation():
    gm = _mesh(2, (2, 2, 2), 1)
    op, src = _op(gm, "tensor4", 1, "fp64")
    for bad in (0, 9, -2):
        with pytest.raises(lsmf.LsmfError):
            op.set_chunks(bad)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_vcycle_with_chunked_fine_level(precision):
    # the smoother's cells-only loops and the residual vmult of the fine level
    # run chunked inside the captured graph
    mesh = lsmf.Mesh("box", (6, 6, 6), 2, degree=2)  # fine level 24^3 cells
    mesh.set_dirichlet([(4, 7)])
    nc, nn, nd = mesh.info()
    X, _, _ = mesh.arrays()
    u = torch.tensor((0.01 * np.sin(np.pi * X[:, [1, 2, 0]])).reshape(-1), device="cuda")
    b = torch.tensor(np.random.default_rng(1).uniform(-1, 1, nd), device="cuda")
    out = []
    for k in (1, 4):
        g = lsmf.GMG(mesh, "tensor4", 1, precision)
        g.set_material(np.ones(nc), 0.3)
        g.level_option(2, 8, k)
        g.setup(u)
        x = torch.empty_like(b)
        g.vmult(x, b)
        y = torch.empty_like(b)
        g.vmult(y, b)  # replayed graph
        torch.cuda.synchronize()
        out.append((x.cpu().numpy(), y.cpu().numpy()))
        del g
    tol = 1e-12 if precision == "fp64" else 1e-5
    ref = out[0][0]
    for x, y in out:
        assert np.max(np.abs(x - ref)) <= tol * np.max(np.abs(ref))
        assert np.max(np.abs(y - ref)) <= tol * np.max(np.abs(ref))
