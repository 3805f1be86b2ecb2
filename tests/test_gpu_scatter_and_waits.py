"""GPU tests of the colour8 scatter, the bounded bulk-copy wait, and the small
operator surface (n, el, memory_consumption), through the C ABI.

colour8 (LSMF_OPT_SCATTER = 1) processes the cells in the 8 parity colours
of the lattice, one launch per colour with plain adds: vmult, diagonal,
transfers and the residual must be bit-identical from call to call, agree
with the atomic path to rounding, and a whole Newton solve must repeat with
identical iteration counts and an identical solution.

The wait test sets the pipelined kernel's try limit to 0, so that every
wait for a cell record runs out at once: the copies still land (each warp
drains its stages before it ends), the operator reports LSMF_ERR_TIMEOUT
once, and the next vmult with the default bound is correct.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
import oracle as O  # noqa: E402
from prm_util import prm_text  # noqa: E402
from test_gpu_operator import _oracle_op, _rel, _setup  # noqa: E402


def _vmult(op, src):
    dsrc = torch.tensor(src, device="cuda", dtype=op.dtype)
    ddst = torch.empty_like(dsrc)
    op.vmult(ddst, dsrc)
    torch.cuda.synchronize()
    return ddst


@pytest.mark.parametrize("caching,formulation", [("tensor4", 1), ("tensor2", 1), ("scalar", 1), ("scalar", 0),
                                                 ("scalar_referential", 1), ("tensor4_ns", 1)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("p", [1, 2, 4])
def test_colour8_vmult_is_reproducible_and_matches(caching, formulation, precision, p):
    gm, om, cmask, mu, u, src = _setup(p=p, coarse=(3, 2, 2) if p < 4 else (2, 1, 2), level=1)
    ref = _oracle_op(om, cmask, mu, u, caching, formulation)
    op = lsmf.NeoHookOperator(gm, caching, formulation, precision)
    op.set_material(mu, 0.3)
    du = torch.tensor(u, device="cuda", dtype=op.dtype)
    op.cache(du)
    a1 = _vmult(op, src)
    op.set_scatter("colour8")
    c1 = _vmult(op, src)
    c2 = _vmult(op, src)
    assert torch.equal(c1, c2)                  # bit-reproducible
    tol = 1e-13 if precision == "fp64" else 2e-6
    assert _rel(c1.double().cpu().numpy(), a1.double().cpu().numpy()) < tol
    want = ref.vmult(src)
    assert _rel(c1.double().cpu().numpy(), want) < (1e-10 if precision == "fp64" else 2e-5)
    # every kernel form takes the colour lists
    for kernel in ("plain", "basic"):
        if kernel == "basic":
            op.set_basic_kernel(True)
        else:
            op.set_pipeline(0)
        k1 = _vmult(op, src)
        assert torch.equal(k1, _vmult(op, src))
        assert _rel(k1.double().cpu().numpy(), want) < (1e-10 if precision == "fp64" else 2e-5)
    # the diagonal too
    op.compute_diagonal()
    d1 = op.get_matrix_diagonal()
    op.compute_diagonal()
    assert torch.equal(d1, op.get_matrix_diagonal())
    dref, _ = ref.diagonal()
    assert _rel(d1.double().cpu().numpy(), dref) < (1e-10 if precision == "fp64" else 2e-5)


def test_colour8_vcycle_is_reproducible():
    gm, om, cmask, mu, u, src = _setup(p=2, coarse=(2, 2, 2), level=2)
    b = src.copy()
    b[cmask == 1] = 0
    db = torch.tensor(b, device="cuda")
    du = torch.tensor(u, device="cuda")
    out = {}
    for mode in ("atomic", "colour8"):
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
    assert torch.equal(out["colour8"][0], out["colour8"][1])
    assert _rel(out["colour8"][0].cpu().numpy(), out["atomic"][0].cpu().numpy()) < 1e-4


def _newton_prm(scatter):
    return prm_text({
        "Polynomial degree": 2, "Quadrature order": 3, "Dimension": 3, "Type": "Cook", "Elements per edge": 2,
        "Global refinement": 1, "Grid scale": 1, "Cook thickness": 10, "Poisson's ratio": 0.3,
        "Shear modulus": 80.194, "Formulation": 1, "Solver type": "MF_CG", "Residual": 1e-8,
        "Preconditioner type": "gmg", "MF caching": "tensor4", "MF level precision": "float", "MF scatter": scatter,
        "Dirichlet IDs and expressions": "1:0,0,0", "Dirichlet IDs and component mask": "1:true,true,true",
        "Neumann IDs and expressions": "11:0,6.25*t,0", "End time": 0.4, "Time step size": 0.2,
        "Output points": "48, 60, 5"})


def test_colour8_newton_is_reproducible():
    runs = []
    for _ in range(2):
        pb = lsmf.Problem(_newton_prm("colour8"))
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


def test_scatter_option_rejects_bad_values():
    gm = lsmf.Mesh("box", (1, 1, 1), 0, degree=2)
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    with pytest.raises(lsmf.LsmfError) as e:
        op.set_scatter(7)
    assert e.value.status == 1
    with pytest.raises(lsmf.LsmfError):
        op.set_wait_tries(-2)
    assert lsmf.prm_validate(_newton_prm("sometimes"))[0] == 9


def test_bounded_wait_run_out_reports_timeout_and_recovers():
    gm, om, cmask, mu, u, src = _setup(p=2, coarse=(4, 4, 4), level=1)
    ref = _oracle_op(om, cmask, mu, u, "tensor4", 1)
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    op.set_pipeline(1)              # the bulk-copy ring (its waits are bounded)
    op.set_material(mu, 0.3)
    du = torch.tensor(u, device="cuda")
    op.cache(du)
    op.set_wait_tries(0)            # every wait for a record runs out at once
    _vmult(op, src)
    with pytest.raises(lsmf.LsmfError) as e:
        op.sync()
    assert e.value.status == 8 and "timed out" in str(e.value)
    op.sync()                       # reported once: the device word was cleared
    op.set_wait_tries(-1)
    got = _vmult(op, src).cpu().numpy()
    op.sync()
    assert _rel(got, ref.vmult(src)) < 1e-10
    # a CG solve reports the run-out too
    op.set_wait_tries(0)
    b = torch.tensor(np.where(cmask == 1, 0.0, src), device="cuda")
    x = torch.zeros_like(b)
    with pytest.raises(lsmf.LsmfError) as e:
        lsmf.cg_solve(op, x, b, 1e-30, 3, "none")
    assert e.value.status == 8
    op.sync()                       # the solve reported (and cleared) it
    op.set_wait_tries(-1)


def test_el_n_and_memory_consumption():
    gm, om, cmask, mu, u, src = _setup(p=2, coarse=(2, 2, 2), level=1)
    nc, nn, nd = gm.info()
    # values per cell record: ncomp per quadrature point, padded at the end
    # to 16 bytes (tensor4, tensor2 and tensor4_ns fold JxW into their
    # coefficients: 51, 17 and 90 per point); scalar caching on these affine
    # cells keeps 11 per point and the reference inverse Jacobian once per
    # cell (11 * 27 + 9 = 306)
    for caching, rec in (("tensor4", 51 * 27 + 1), ("tensor2", 17 * 27 + 1), ("scalar", 306), ("tensor4_ns", 90 * 27)):
        op = lsmf.NeoHookOperator(gm, caching, 1, "fp64")
        assert op.m() == op.n() == nd
        # cache tables plus the index map and the node coordinates; diagonals
        # excluded
        assert op.memory_consumption() == nc * rec * 8 + nc * 27 * 4 + nn * 3 * 8
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    op.set_material(mu, 0.3)
    op.cache(torch.tensor(u, device="cuda"))
    with pytest.raises(lsmf.LsmfError) as e:
        op.el(3, 3)                 # no diagonal yet
    assert e.value.status == 4
    op.compute_diagonal()
    d = op.get_matrix_diagonal().cpu().numpy()
    for i in (0, 5, nd // 2, nd - 1):
        assert op.el(i, i) == d[i]
    with pytest.raises(lsmf.LsmfError) as e:
        op.el(1, 2)
    assert e.value.status == 10
    with pytest.raises(lsmf.LsmfError):
        op.el(nd, nd)
