"""GPU tests of the node-sum scatter (LSMF_SCATTER_NODESUM): the vmult cell
loop stores every cell's results to a per-cell buffer and a node kernel adds
each node's cell contributions in increasing cell order.

* vmult / vmult_add are bit-identical from call to call, equal to the atomic
  path to rounding (1e-13 FP64, 2e-6 FP32) and to the oracle (1e-10 / 2e-5),
  for every variant at degrees 1 to 4, FP64 and FP32 (the FP32 pair
  kernel included where it is the default);
* constrained rows keep their identity entries;
* a V-cycle with node-sum level operators and a whole Newton solve repeat
  bit for bit, and the Newton solve agrees with the atomic one;
* the diagonal of a node-sum operator (colour launches) is reproducible.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
from test_gpu_operator import VARIANTS, _oracle_op, _rel, _setup  # noqa: E402
from test_gpu_scatter_and_waits import _newton_prm, _vmult  # noqa: E402


@pytest.mark.parametrize("caching,formulation", VARIANTS)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_nodesum_vmult_is_reproducible_and_matches(caching, formulation, precision, p):
    gm, om, cmask, mu, u, src = _setup(p=p, coarse=(3, 2, 2) if p < 3 else (2, 1, 2), level=1)
    ref = _oracle_op(om, cmask, mu, u, caching, formulation)
    op = lsmf.NeoHookOperator(gm, caching, formulation, precision)
    op.set_material(mu, 0.3)
    op.cache(torch.tensor(u, device="cuda", dtype=op.dtype))
    a1 = _vmult(op, src)
    op.set_scatter("nodesum")
    n1 = _vmult(op, src)
    assert torch.equal(n1, _vmult(op, src))          # bit-reproducible
    got = n1.double().cpu().numpy()
    assert _rel(got, a1.double().cpu().numpy()) < (1e-13 if precision == "fp64" else 2e-6)
    assert _rel(got, ref.vmult(src)) < (1e-10 if precision == "fp64" else 2e-5)
    assert np.array_equal(got[cmask == 1], src[cmask == 1].astype(np.float32 if precision == "fp32" else np.float64))
    # vmult_add accumulates through the node sums
    dsrc = torch.tensor(src, device="cuda", dtype=op.dtype)
    op.vmult_add(n1, dsrc)
    n2 = _vmult(op, src)
    op.vmult_add(n2, dsrc)
    assert torch.equal(n1, n2)
    assert _rel(n1.double().cpu().numpy(), 2 * got) < (1e-13 if precision == "fp64" else 2e-6)
    # the diagonal runs the colours: reproducible
    op.compute_diagonal()
    d1 = op.get_matrix_diagonal()
    op.compute_diagonal()
    assert torch.equal(d1, op.get_matrix_diagonal())


def test_nodesum_vcycle_is_reproducible():
    gm, om, cmask, mu, u, src = _setup(p=2, coarse=(2, 2, 2), level=2)
    b = src.copy()
    b[cmask == 1] = 0
    db = torch.tensor(b, device="cuda")
    du = torch.tensor(u, device="cuda")
    out = {}
    for mode in ("atomic", "nodesum"):
        g = lsmf.GMG(gm, "tensor4", 1, "fp32")
        g.set_scatter(mode)
        g.set_material(mu, 0.3)
        g.setup(du)
        r = []
        for _ in range(2):
            x = torch.empty_like(db)
            g.vmult(x, db)
            torch.cuda.synchronize()
            r.append(x)
        out[mode] = r
    assert torch.equal(out["nodesum"][0], out["nodesum"][1])
    assert _rel(out["nodesum"][0].cpu().numpy(), out["atomic"][0].cpu().numpy()) < 1e-4


def test_nodesum_newton_is_reproducible():
    runs = []
    for _ in range(2):
        pb = lsmf.Problem(_newton_prm("nodesum"))
        res = pb.run()
        runs.append(([s["newton_iterations"] for s in res["steps"]], [s["cg_iterations"] for s in res["steps"]],
                     pb.solution()))
    assert runs[0][0] == runs[1][0] and runs[0][1] == runs[1][1]
    assert np.array_equal(runs[0][2], runs[1][2])
    pa = lsmf.Problem(_newton_prm("atomic"))
    ra = pa.run()
    assert [s["newton_iterations"] for s in ra["steps"]] == runs[0][0]
    ua = pa.solution()
    assert np.max(np.abs(ua - runs[0][2])) <= 1e-7 * np.max(np.abs(ua))


def test_nodesum_option_values():
    gm = lsmf.Mesh("box", (1, 1, 1), 0, degree=2)
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    op.set_scatter("nodesum")
    op.set_scatter("atomic")
    with pytest.raises(lsmf.LsmfError) as e:
        op.set_scatter(3)
    assert e.value.status == 1
    assert lsmf.prm_validate(_newton_prm("nodesum"))[0] == 0
