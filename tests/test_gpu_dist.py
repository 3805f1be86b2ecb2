"""The distributed operator on one GPU: z-slab parts driven by one process
(lsmf_dist_create_group), each part's operator on its own CUDA stream, with
both interface exchanges: packed (update_ghost_values / compress(add)
through buffers moved between the parts' streams) and fused (the cell loops
read the owners' src values and add to the owners' dst directly, the
neighbours' streams ordered by events).

* vmult equals the whole-mesh vmult on every owned entry within 1e-12
  relative, for every caching variant and formulation;
* the owned-entry dot product equals the whole-mesh one;
* CG with the Jacobi preconditioner (diagonal summed across the interfaces)
  reaches the tolerance and its solution equals the whole-mesh CG solution
  within 1e-9 relative, with the same iteration count to within 2;
on a full box and on a box whose voids cut the interfaces, 2 and 3 parts.
The NCCL transport (one part per process) uses the same packing and
ownership; it is exercised where several GPUs are available.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
import oracle as O  # noqa: E402

COARSE = (4, 4, 4)
LEVEL = 1


def _problem(n_parts, voids, caching="tensor4", formulation=1):
    act = O.void_mask(COARSE, 3, 0.2, 5) if voids else None
    kw = dict(geometry="box", coarse=COARSE, n_refinements=LEVEL, degree=2, coarse_active=act)
    gm = lsmf.Mesh(**kw)
    spec = [(4, 7), (5, 4)]
    gm.set_dirichlet(spec)
    nc, nn, nd = gm.info()
    X, _, ijk = gm.arrays()
    rng = np.random.default_rng(11)
    mu = rng.choice([1.0, 10.0], nc)
    u = (0.01 * np.sin(np.pi * X[:, [1, 2, 0]])).reshape(-1)
    cell_of = {tuple(c): i for i, c in enumerate(ijk.tolist())}
    parts = []
    for r in range(n_parts):
        pm = lsmf.Mesh(n_parts=n_parts, part=r, **kw)
        pm.set_dirichlet(spec)
        lay = lsmf.partition_layout(n_parts, r, **kw)
        _, _, pijk = pm.arrays()
        pmu = mu[[cell_of[tuple(c)] for c in pijk.tolist()]]
        gd = (3 * lay["global_node"][:, None] + np.arange(3)).reshape(-1)
        owned = np.ones(lay["n_nodes"], dtype=bool)
        owned[lay["upper_shared"]] = False
        od = (3 * np.nonzero(owned)[0][:, None] + np.arange(3)).reshape(-1)
        assert np.array_equal(pm.constraint_mask(), gm.constraint_mask()[gd])
        op = lsmf.NeoHookOperator(pm, caching, formulation, "fp64")
        op.set_stream(torch.cuda.Stream())
        op.set_material(pmu, 0.3)
        du = torch.tensor(u[gd], device="cuda")
        op.cache(du)
        parts.append(dict(mesh=pm, op=op, u=du, gd=gd, od=od, lay=lay))
    gop = lsmf.NeoHookOperator(gm, caching, formulation, "fp64")
    gop.set_material(mu, 0.3)
    gu = torch.tensor(u, device="cuda")
    gop.cache(gu)
    return gm, gop, gu, parts, rng


@pytest.mark.parametrize("exchange", ["packed", "fused"])
@pytest.mark.parametrize("n_parts", [2, 3])
@pytest.mark.parametrize("voids", [False, True])
def test_group_vmult_dot_and_cg_equal_whole_mesh(n_parts, voids, exchange, parity):
    gm, gop, gu, parts, rng = _problem(n_parts, voids)
    nd = gm.info()[2]
    D = lsmf.Dist.group([p["op"] for p in parts])
    assert D.exchange() == "fused"  # the default for parts on one GPU
    D.set_exchange(exchange)
    assert D.exchange() == exchange
    src = rng.uniform(-1, 1, nd)
    dsrc = torch.tensor(src, device="cuda")
    want = torch.empty_like(dsrc)
    gop.vmult(want, dsrc)
    want = want.cpu().numpy()
    srcs, dsts = [], []
    for p in parts:
        s = torch.tensor(src[p["gd"]], device="cuda")
        s[torch.tensor(3 * p["lay"]["upper_shared"], device="cuda").long()] = 1e30  # ghosts are overwritten
        srcs.append(s)
        dsts.append(torch.full_like(s, 7.0))
    D.vmult(dsts, srcs)
    torch.cuda.synchronize()
    for p, d in zip(parts, dsts):
        got = d.cpu().numpy()
        parity("partitioned vmult, %d parts%s, %s exchange" % (n_parts, ", voids" if voids else "", exchange),
               np.max(np.abs(got[p["od"]] - want[p["gd"][p["od"]]])) / np.max(np.abs(want)), 1e-12)
        assert np.max(np.abs(got[p["od"]] - want[p["gd"][p["od"]]])) <= 1e-12 * np.max(np.abs(want))
        # ghost entries of the result are cleared
        ud = (3 * p["lay"]["upper_shared"][:, None] + np.arange(3)).reshape(-1)
        assert np.all(got[ud] == 0.0)
    # owned-entry dot product
    y = rng.uniform(-1, 1, nd)
    ys = [torch.tensor(y[p["gd"]], device="cuda") for p in parts]
    xs = [torch.tensor(src[p["gd"]], device="cuda") for p in parts]
    assert abs(D.dot(ys, xs) - float(np.dot(y, src))) <= 1e-12 * abs(float(np.dot(y, src)))
    # Jacobi-preconditioned CG against the whole-mesh CG
    cm = gm.constraint_mask()
    b = np.where(cm == 1, 0.0, rng.uniform(-1, 1, nd))
    db = torch.tensor(b, device="cuda")
    tol = 1e-10 * np.linalg.norm(b)
    gop.compute_diagonal()
    xg = torch.zeros_like(db)
    ig = lsmf.cg_solve(gop, xg, db, tol, 5000, "jacobi", omega=1.0)
    assert ig["converged"]
    bs = [torch.tensor(b[p["gd"]], device="cuda") for p in parts]
    xl = [torch.zeros_like(t) for t in bs]
    info = D.cg_solve(xl, bs, tol, 5000, "jacobi", omega=1.0)
    assert info["converged"] and info["residual"] <= tol
    assert abs(info["iterations"] - ig["iterations"]) <= 2, (info, ig)
    xg = xg.cpu().numpy()
    for p, x in zip(parts, xl):
        got = x.cpu().numpy()
        # the ghost entries carry the owners' values after the solve
        assert np.max(np.abs(got - xg[p["gd"]])) <= 1e-9 * np.max(np.abs(xg))


@pytest.mark.parametrize("caching,formulation", [("tensor2", 1), ("scalar", 1), ("scalar", 0),
                                                  ("scalar_referential", 1), ("tensor4_ns", 1)])
def test_fused_exchange_every_caching(caching, formulation, parity):
    # the scalar variants also gather the displacement at the ghost nodes
    # (from the owner's u in the fused form)
    gm, gop, gu, parts, rng = _problem(3, True, caching, formulation)
    nd = gm.info()[2]
    src = rng.uniform(-1, 1, nd)
    want = torch.empty(nd, dtype=torch.float64, device="cuda")
    gop.vmult(want, torch.tensor(src, device="cuda"))
    want = want.cpu().numpy()
    D = lsmf.Dist.group([p["op"] for p in parts])
    for exchange in ("fused", "packed"):
        D.set_exchange(exchange)
        srcs = [torch.tensor(src[p["gd"]], device="cuda") for p in parts]
        dsts = [torch.full_like(s, 7.0) for s in srcs]
        D.vmult(dsts, srcs)
        torch.cuda.synchronize()
        err = max(np.max(np.abs(d.cpu().numpy()[p["od"]] - want[p["gd"][p["od"]]])) for p, d in zip(parts, dsts))
        parity("partitioned vmult, 3 parts, voids, %s f%d, %s exchange" % (caching, formulation, exchange),
               err / np.max(np.abs(want)), 1e-12)
        assert err <= 1e-12 * np.max(np.abs(want)), (exchange, err)


def test_fused_exchange_parts_on_one_stream():
    # parts left on the default stream: every zeroing, wait and cell loop of
    # the fused exchange is ordered on the same stream (each wait follows its
    # event's record in that order)
    gm, gop, gu, parts, rng = _problem(3, True)
    for p in parts:
        p["op"].set_stream(None)
    nd = gm.info()[2]
    src = rng.uniform(-1, 1, nd)
    want = torch.empty(nd, dtype=torch.float64, device="cuda")
    gop.vmult(want, torch.tensor(src, device="cuda"))
    want = want.cpu().numpy()
    D = lsmf.Dist.group([p["op"] for p in parts])
    assert D.exchange() == "fused"
    srcs = [torch.tensor(src[p["gd"]], device="cuda") for p in parts]
    dsts = [torch.empty_like(s) for s in srcs]
    for _ in range(2):
        D.vmult(dsts, srcs)
    torch.cuda.synchronize()
    for p, d in zip(parts, dsts):
        assert np.max(np.abs(d.cpu().numpy()[p["od"]] - want[p["gd"][p["od"]]])) <= 1e-12 * np.max(np.abs(want))


def test_exchange_option():
    gm, gop, gu, parts, rng = _problem(2, False)
    D = lsmf.Dist.group([p["op"] for p in parts])
    nd = gm.info()[2]
    src = rng.uniform(-1, 1, nd)
    want = torch.empty(nd, dtype=torch.float64, device="cuda")
    gop.vmult(want, torch.tensor(src, device="cuda"))
    want = want.cpu().numpy()
    with pytest.raises(lsmf.LsmfError):
        D.set_exchange(5)
    # a deterministic scatter on one part: the vmult falls back to the packed
    # exchange and stays right
    parts[0]["op"].set_scatter("colour8")
    assert D.exchange() == "packed"
    srcs = [torch.tensor(src[p["gd"]], device="cuda") for p in parts]
    dsts = [torch.empty_like(s) for s in srcs]
    D.vmult(dsts, srcs)
    torch.cuda.synchronize()
    for p, d in zip(parts, dsts):
        assert np.max(np.abs(d.cpu().numpy()[p["od"]] - want[p["gd"][p["od"]]])) <= 1e-12 * np.max(np.abs(want))
    parts[0]["op"].set_scatter("atomic")
    assert D.exchange() == "fused"


def test_group_rejects_mismatched_parts():
    kw = dict(geometry="box", coarse=COARSE, n_refinements=LEVEL, degree=2)
    a = lsmf.Mesh(n_parts=2, part=0, **kw)
    b = lsmf.Mesh(n_parts=3, part=1, **kw)
    ops = [lsmf.NeoHookOperator(a, "tensor4", 1, "fp64"), lsmf.NeoHookOperator(b, "tensor4", 1, "fp64")]
    with pytest.raises(lsmf.LsmfError):
        lsmf.Dist.group(ops)
    with pytest.raises(lsmf.LsmfError):
        lsmf.Mesh(n_parts=5, part=0, **kw)  # fewer coarse z-layers than parts


def test_nccl_transport_single_part():
    """The NCCL transport with one part (the one-GPU case of a sharded run):
    libnccl is loaded at run time, the communicator is built from the
    128-byte id, the CG scalars go through ncclAllReduce; vmult and CG equal
    the plain operator's."""
    gm = lsmf.Mesh("box", COARSE, LEVEL, degree=2)
    gm.set_dirichlet([(4, 7)])
    nc, nn, nd = gm.info()
    X, _, _ = gm.arrays()
    rng = np.random.default_rng(5)
    mu = rng.choice([1.0, 10.0], nc)
    op = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    op.set_material(mu, 0.3)
    du = torch.tensor((0.01 * np.sin(np.pi * X[:, [1, 2, 0]])).reshape(-1), device="cuda")
    op.cache(du)
    uid = lsmf.Dist.nccl_unique_id()
    assert len(uid) == 128
    D = lsmf.Dist.nccl(op, uid)
    # one part per process: the interface data go through NCCL buffers
    assert D.exchange() == "packed"
    with pytest.raises(lsmf.LsmfError) as e:
        D.set_exchange("fused")
    assert e.value.status == 10  # LSMF_ERR_UNSUPPORTED
    src = torch.tensor(rng.uniform(-1, 1, nd), device="cuda")
    want, got = torch.empty_like(src), torch.empty_like(src)
    op.vmult(want, src)
    D.vmult([got], [src])
    torch.cuda.synchronize()
    # (the atomic scatter makes two vmults equal to rounding, not bitwise)
    assert (torch.max(torch.abs(got - want)) / torch.max(torch.abs(want))).item() < 1e-13
    b = torch.where(torch.tensor(gm.constraint_mask() == 1, device="cuda"), 0.0, src)
    tol = 1e-10 * torch.linalg.norm(b).item()
    op.compute_diagonal()
    x1, x2 = torch.zeros_like(b), torch.zeros_like(b)
    i1 = lsmf.cg_solve(op, x1, b, tol, 5000, "jacobi", omega=1.0)
    i2 = D.cg_solve([x2], [b], tol, 5000, "jacobi", omega=1.0)
    assert i1["converged"] and i2["converged"] and abs(i1["iterations"] - i2["iterations"]) <= 1
    assert (torch.max(torch.abs(x1 - x2)) / torch.max(torch.abs(x1))).item() < 1e-9
