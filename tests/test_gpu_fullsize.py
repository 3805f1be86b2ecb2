"""Size-independent properties of the tangent operator at the benchmark size
(64^3 Q2 unit cube, 6,440,067 DoFs, tensor4 records 2.9 GB), where the CPU
oracle is too slow to compare against:

  * symmetry:   y . A x = x . A y             (1e-12 relative)
  * linearity:  A (a x + y) = a A x + A y     (1e-12 relative)
  * the production kernel equals the basic (independent) kernel   (1e-12)
  * every caching variant gives the tensor4 operator              (1e-10)
  * FP32 equals FP64                                               (2e-5)
  * the z-slab distributed operator (2 and 4 parts on this GPU, ghost
    update and compress(add)) equals the whole-mesh operator on every
    owned entry                                                     (1e-12)

Inputs as in bench.py: per-cell mu in {1, 10}, a smooth displacement bounded
by 0.01 (det F > 0.5), bottom face clamped.
"""
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402

CELLS = 64


@pytest.fixture(scope="module")
def setup():
    mesh = lsmf.Mesh("box", (CELLS,) * 3, 0, degree=2)
    mesh.set_dirichlet([(4, 7)])
    n_cells, _, n_dofs = mesh.info()
    X, _, _ = mesh.arrays()
    rng = np.random.default_rng(2024)
    mu = rng.choice([1.0, 10.0], size=n_cells)
    u = torch.tensor(bench.smooth_field(X, 7).reshape(-1), device="cuda")
    x = torch.tensor(rng.uniform(-1, 1, n_dofs), device="cuda")
    y = torch.tensor(rng.uniform(-1, 1, n_dofs), device="cuda")
    return mesh, mu, u, x, y


def _op(mesh, mu, u, caching="tensor4", precision="fp64"):
    op = lsmf.NeoHookOperator(mesh, caching, 1, precision)
    op.set_material(mu, 0.3)
    op.cache(u if precision == "fp64" else u.float())
    return op


def _apply(op, v):
    out = torch.empty_like(v)
    op.vmult(out, v)
    return out


def _rel(a, b):
    return (torch.max(torch.abs(a - b)) / torch.max(torch.abs(b))).item()


def test_symmetry_and_linearity(setup):
    mesh, mu, u, x, y = setup
    op = _op(mesh, mu, u)
    ax, ay = _apply(op, x), _apply(op, y)
    lhs, rhs = torch.dot(y, ax).item(), torch.dot(x, ay).item()
    scale = (torch.linalg.norm(y) * torch.linalg.norm(ax)).item()
    assert abs(lhs - rhs) <= 1e-12 * scale
    a = 0.37
    assert _rel(_apply(op, a * x + y), a * ax + ay) < 1e-12


def test_fast_kernel_equals_basic_kernel(setup):
    mesh, mu, u, x, y = setup
    op = _op(mesh, mu, u)
    fast = _apply(op, x)
    op.set_basic_kernel(True)
    assert _rel(_apply(op, x), fast) < 1e-12


@pytest.mark.parametrize("caching", ["tensor2", "scalar", "scalar_referential", "tensor4_ns"])
def test_every_caching_gives_the_tensor4_operator(setup, caching):
    mesh, mu, u, x, y = setup
    ref = _apply(_op(mesh, mu, u), x)
    torch.cuda.empty_cache()
    assert _rel(_apply(_op(mesh, mu, u, caching), x), ref) < 1e-10


def test_fp32_equals_fp64(setup):
    mesh, mu, u, x, y = setup
    ref = _apply(_op(mesh, mu, u), x)
    got = _apply(_op(mesh, mu, u, precision="fp32"), x.float())
    assert _rel(got.double(), ref) < 2e-5


def test_partitioned_operator_at_benchmark_size():
    out = bench.dist_vmult_times(CELLS, (2, 4), reps=2)
    assert out["n_dofs"] == 6440067
    for n in (2, 4):
        for mode in ("packed", "fused"):
            assert out["parts_%d" % n][mode]["rel_err_owned"] <= 1e-12, out
