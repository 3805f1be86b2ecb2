"""GPU tests of the FP32 cell-pair vmult kernel (LSMF_OPT_CELL_PAIRS): two
cells per warp whose sum factorisation and point physics run as the two
halves of packed f32x2 registers.

* For every variant and degree, with atomic and colour8 scatter, on cell
  counts that leave a cell without a partner and on even ones, the pair
  kernel equals the one-cell kernel to FP32 rounding (1e-6 relative; the
  two differ only in where the compiler contracts products into FMAs).
* Its output matches the oracle's FP64 vmult within the FP32 tolerance
  (2e-5) and keeps the identity rows of constrained entries.
* With colour8 it is bit-reproducible, and the automatic choice is the pair
  kernel exactly for tensor2, scalar formulation 1 and scalar_referential.
* The option is validated; FP64 operators ignore it.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
from test_gpu_operator import VARIANTS, _oracle_op, _rel, _setup  # noqa: E402

PAIRED_BY_DEFAULT = {("tensor2", 1), ("scalar", 1), ("scalar_referential", 1)}


def _op(gm, mu, u, caching, formulation, precision="fp32"):
    op = lsmf.NeoHookOperator(gm, caching, formulation, precision)
    op.set_material(mu, 0.3)
    op.cache(torch.tensor(u, device="cuda", dtype=op.dtype))
    return op


def _vmult(op, src):
    dsrc = torch.tensor(src, device="cuda", dtype=op.dtype)
    ddst = torch.empty_like(dsrc)
    op.vmult(ddst, dsrc)
    torch.cuda.synchronize()
    return ddst


@pytest.mark.parametrize("caching,formulation", VARIANTS)
@pytest.mark.parametrize("p,coarse,level", [(1, (3, 3, 3), 0), (2, (3, 3, 3), 0), (2, (2, 2, 2), 1), (3, (3, 1, 3), 0),
                                            (4, (1, 2, 1), 1)])
@pytest.mark.parametrize("scatter", ["atomic", "colour8"])
def test_pairs_equal_one_cell_kernel(caching, formulation, p, coarse, level, scatter):
    gm, om, cmask, mu, u, src = _setup(p=p, coarse=coarse, level=level)
    op = _op(gm, mu, u, caching, formulation)
    op.set_scatter(scatter)
    op.set_cell_pairs(0)
    one = _vmult(op, src).double().cpu().numpy()
    op.set_cell_pairs(1)
    pair = _vmult(op, src)
    got = pair.double().cpu().numpy()
    assert _rel(got, one) < 1e-6
    ref = _oracle_op(om, cmask, mu, u, caching, formulation)
    assert _rel(got, ref.vmult(src)) < 2e-5
    # constrained rows are identity (mf_nh_operator.h:702-705)
    assert np.array_equal(got[cmask == 1], src[cmask == 1].astype(np.float32).astype(np.float64))
    # vmult_add accumulates through the pair kernel as well
    op.vmult_add(pair, torch.tensor(src, device="cuda", dtype=torch.float32))
    assert _rel(pair.double().cpu().numpy(), 2 * got) < 1e-6
    if scatter == "colour8":
        assert torch.equal(_vmult(op, src), _vmult(op, src))


@pytest.mark.parametrize("caching,formulation", VARIANTS)
def test_default_choice_of_pairs(caching, formulation):
    # with colour8 the result identifies the kernel bit for bit
    gm, om, cmask, mu, u, src = _setup(p=2, coarse=(3, 3, 3), level=0)
    op = _op(gm, mu, u, caching, formulation)
    op.set_scatter("colour8")
    default = _vmult(op, src)
    op.set_cell_pairs(1 if (caching, formulation) in PAIRED_BY_DEFAULT else 0)
    assert torch.equal(default, _vmult(op, src))


def test_option_validation_and_fp64():
    gm, om, cmask, mu, u, src = _setup(p=2, coarse=(2, 2, 2), level=0)
    op = _op(gm, mu, u, "tensor2", 1, "fp64")
    for bad in (2, -2):
        with pytest.raises(lsmf.LsmfError):
            op.set_cell_pairs(bad)
    op.set_scatter("colour8")
    a = _vmult(op, src)
    op.set_cell_pairs(1)   # FP64: ignored
    assert torch.equal(a, _vmult(op, src))


@pytest.mark.parametrize("caching,formulation", VARIANTS)
@pytest.mark.parametrize("p", [1, 2, 4])
def test_single_cell_mesh(caching, formulation, p):
    # one cell: the only pair has no partner (pairs) and every node belongs
    # to exactly one cell (node sums)
    gm, om, cmask, mu, u, src = _setup(p=p, coarse=(1, 1, 1), level=0)
    op = _op(gm, mu, u, caching, formulation)
    ref = _oracle_op(om, cmask, mu, u, caching, formulation)
    want = ref.vmult(src)
    for pairs in (0, 1):
        op.set_cell_pairs(pairs)
        for scatter in ("atomic", "colour8", "nodesum"):
            op.set_scatter(scatter)
            got = _vmult(op, src).double().cpu().numpy()
            assert _rel(got, want) < 2e-5, (pairs, scatter)
