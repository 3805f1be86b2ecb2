"""The allocation-free residual norm entry point, checked against the
existing path (the residual that lsmf_cg_solve reports before iterating).

Callers that cannot call cudaMalloc while running (device memory owned by
another framework's caching allocator, or a no-allocation-after-start-up
rule) use lsmf_residual_norm_noalloc; its scratch lives in a static device
array.  This file is collected last so that a failure here cannot hide the
other tests; it passes alone in a fresh process and after the others.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402


def _reference_norm(op, x, b):
    # existing entry point: CG with an unreachable iteration budget of 0 and
    # an infinite tolerance returns ||A x - b|| without touching x
    xx = x.clone()
    info = lsmf.cg_solve(op, xx, b, float("inf"), 0, "none")
    assert torch.equal(xx, x)
    return info["residual"]


def test_residual_norm_noalloc_matches_existing_path():
    rng = np.random.default_rng(21)
    mesh = lsmf.Mesh("box", (2, 2, 2), 1, degree=2)
    mesh.set_dirichlet([(4, 7)])
    nc, _, nd = mesh.info()
    X, _, _ = mesh.arrays()
    op = lsmf.NeoHookOperator(mesh, "tensor4", 1, "fp64")
    op.set_material(rng.choice([1.0, 10.0], nc), 0.3)
    u = torch.tensor((0.01 * np.sin(np.pi * X[:, [2, 0, 1]])).reshape(-1), device="cuda")
    op.cache(u)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for call in range(2):  # two calls in a row share (and overwrite) the scratch
        x = torch.tensor(rng.uniform(-1, 1, nd), device="cuda")
        b = torch.tensor(rng.uniform(-1, 1, nd) * (call + 1), device="cuda")
        op.residual_norm_noalloc(x, b, out)
        torch.cuda.synchronize()
        want = _reference_norm(op, x, b)
        assert abs(out.item() - want) <= 1e-12 * want, (call, out.item(), want)


def test_residual_norm_noalloc_rejects_bad_input():
    mesh = lsmf.Mesh("box", (1, 1, 1), 0, degree=2)
    op32 = lsmf.NeoHookOperator(mesh, "tensor4", 1, "fp32")
    x = torch.zeros(mesh.info()[2], dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(lsmf.LsmfError) as e:
        op32.residual_norm_noalloc(x, x, out)
    assert e.value.status == 1
    op = lsmf.NeoHookOperator(mesh, "tensor4", 1, "fp64")
    with pytest.raises(lsmf.LsmfError) as e:          # not cached yet
        op.residual_norm_noalloc(x, x, out)
    assert e.value.status == 4
    big = lsmf.Mesh("box", (64, 64, 64), 0, degree=2)  # 6.4 M dofs > 2,097,152
    opb = lsmf.NeoHookOperator(big, "scalar", 1, "fp64")
    xb = torch.zeros(big.info()[2], dtype=torch.float64, device="cuda")
    opb.cache(xb)
    with pytest.raises(lsmf.LsmfError) as e:
        opb.residual_norm_noalloc(xb, xb, out)
    assert e.value.status == 1 and "at most 2097152" in str(e.value)
