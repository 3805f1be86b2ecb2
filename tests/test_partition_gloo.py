"""The z-slab partition of the distributed operator on the CPU: gloo ranks
(world size 2 and 3), each holding one part.

Each rank takes its part's layout from the library (lsmf_partition_layout,
host only: whole-mesh node numbers and the interface lists), builds the
oracle's operator on the part's cells, and runs the exchange protocol of
lsmf_dist_vmult with torch.distributed point-to-point messages:
update_ghost_values (the owners' values of the upper interface arrive from
part + 1), the part's cell loop, compress(add) (the ghosts' partial sums,
constrained entries dropped, are added on part + 1 and cleared here).  The
owned entries must equal the whole-mesh oracle vmult, every node must be
owned by exactly one part, and the all-reduced owned-entry dot product
must equal the whole-mesh one; on a full box and on a box with voids that
cut the interfaces.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

COARSE = (4, 4, 4)
LEVEL = 1


def _mask(voids):
    import oracle as O
    return O.void_mask(COARSE, 3, 0.2, 5) if voids else None


def _rank_main(rank, world, port, voids, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import lsmf
    import oracle as O
    act = _mask(voids)
    lay = lsmf.partition_layout(world, rank, geometry="box", coarse=COARSE, n_refinements=LEVEL, degree=2,
                                coarse_active=act)
    # the whole mesh and its operator (every rank builds it as the reference answer)
    og = O.Mesh(O.GEOM_BOX, COARSE, LEVEL, (0, 0, 0), (1, 1, 1), 1.0, 2, 3, coarse_active=act)
    assert lay["n_global_nodes"] == og.n_nodes
    cm_g = og.constraints([(4, 7), (5, 4)])
    rng = np.random.default_rng(3)
    mu_g = rng.choice([1.0, 10.0], og.n_cells)
    u_g = 0.01 * np.sin(np.pi * og.X[:, [1, 2, 0]]).reshape(-1)
    src_g = rng.uniform(-1, 1, og.n_dofs)
    ref = O.Operator(og, "tensor4", 1)
    ref.set_material(mu_g, 0.3)
    ref.set_constraints(cm_g)
    ref.cache(u_g)
    want = ref.vmult(src_g)
    # this part's cells: coarse z-layers [k0, k1) of the whole mesh
    nz = COARSE[2]
    k0, k1 = nz * rank // world, nz * (rank + 1) // world
    sub_act = None if act is None else act.reshape(nz, COARSE[1], COARSE[0])[k0:k1].reshape(-1)
    om = O.Mesh(O.GEOM_BOX, (COARSE[0], COARSE[1], k1 - k0), LEVEL, (0, 0, k0 / nz), (1, 1, k1 / nz), 1.0, 2, 3,
                coarse_active=sub_act)
    gn = lay["global_node"]
    assert om.n_nodes == lay["n_nodes"]
    assert np.max(np.abs(om.X - og.X[gn])) < 1e-14
    gd = (3 * gn[:, None] + np.arange(3)).reshape(-1)       # local dof -> whole-mesh dof
    # cell -> whole-mesh cell (through the nodes) for the per-cell mu
    key = {tuple(sorted(c)): i for i, c in enumerate(og.cell_nodes.tolist())}
    mu = np.array([mu_g[key[tuple(sorted(gn[c].tolist()))]] for c in om.cell_nodes])
    op = O.Operator(om, "tensor4", 1)
    op.set_material(mu, 0.3)
    cm = cm_g[gd]
    op.set_constraints(cm)
    op.cache(u_g[gd])
    lower, upper = lay["lower_shared"], lay["upper_shared"]
    ldofs = (3 * lower[:, None] + np.arange(3)).reshape(-1)
    udofs = (3 * upper[:, None] + np.arange(3)).reshape(-1)
    # local source: owned entries from the global vector, ghosts garbage
    src = src_g[gd].copy()
    src[udofs] = 1e30
    # update_ghost_values: owners (part + 1) send their lower interface values
    reqs = []
    if rank > 0:
        reqs.append(dist.isend(torch.tensor(src[ldofs]), rank - 1))
    if rank < world - 1:
        buf = torch.empty(len(udofs), dtype=torch.float64)
        dist.recv(buf, rank + 1)
        src[udofs] = buf.numpy()
    for r in reqs:
        r.wait()
    dst = op.vmult(src)
    # compress(add): ghosts' partial sums (constrained entries dropped) to part + 1
    reqs = []
    if rank < world - 1:
        send = dst[udofs].copy()
        send[cm[udofs] == 1] = 0.0
        reqs.append(dist.isend(torch.tensor(send), rank + 1))
        dst[udofs] = 0.0
    if rank > 0:
        buf = torch.empty(len(ldofs), dtype=torch.float64)
        dist.recv(buf, rank - 1)
        dst[ldofs] += buf.numpy()
    for r in reqs:
        r.wait()
    owned = np.ones(om.n_nodes, dtype=bool)
    owned[upper] = False
    od = (3 * np.nonzero(owned)[0][:, None] + np.arange(3)).reshape(-1)
    err = np.max(np.abs(dst[od] - want[gd[od]])) / np.max(np.abs(want))
    # owned-entry dot product, all-reduced
    x_g = rng.uniform(-1, 1, og.n_dofs)
    part_dot = torch.tensor([float(np.dot(x_g[gd[od]], src_g[gd[od]]))], dtype=torch.float64)
    dist.all_reduce(part_dot)
    count = np.zeros(og.n_nodes, dtype=np.int64)
    count[gn[owned]] = 1
    cnt = torch.tensor(count)
    dist.all_reduce(cnt)
    out[rank] = (float(err), float(part_dot.item()), float(np.dot(x_g, src_g)), bool(np.all(cnt.numpy() == 1)))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("voids", [False, True])
def test_partitioned_vmult_equals_whole_mesh(world, voids):
    port = 31000 + (os.getpid() + 17 * world + 3 * int(voids)) % 1000
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(world, port, voids, out), nprocs=world, join=True)
    for r in range(world):
        err, dot, dot_g, once = out[r]
        assert err < 1e-12, (r, err)
        assert abs(dot - dot_g) <= 1e-12 * abs(dot_g)
        assert once


@pytest.mark.parametrize("world", [2, 3, 4])
@pytest.mark.parametrize("voids", [False, True])
def test_interface_lists_pair_the_same_nodes(world, voids):
    """The fused exchange renumbers part r's ghost nodes (upper_shared[j])
    as part r + 1's nodes lower_shared[j]: both lists must name the same
    whole-mesh nodes in the same order, within each part's node range and
    below the peer bit (2^28) of the index map, and the ghosts must lie on
    the part's top node plane."""
    import lsmf
    act = _mask(voids)
    lays = [lsmf.partition_layout(world, r, geometry="box", coarse=COARSE, n_refinements=LEVEL, degree=2,
                                  coarse_active=act) for r in range(world)]
    for r in range(world):
        lay = lays[r]
        n = lay["n_nodes"]
        assert n < 2 ** 28
        for lst in (lay["lower_shared"], lay["upper_shared"]):
            assert lst.size == 0 or (lst.min() >= 0 and lst.max() < n)
        if r + 1 < world:
            up, lo = lay["upper_shared"], lays[r + 1]["lower_shared"]
            assert up.size == lo.size > 0
            assert np.array_equal(lay["global_node"][up], lays[r + 1]["global_node"][lo])
        else:
            assert lay["upper_shared"].size == 0
        if r == 0:
            assert lay["lower_shared"].size == 0
    # ghosts sit on the part's top plane z = k1 / nz (whole-mesh coordinates
    # from the oracle's mesh; node numbers are compacted around voids)
    import oracle as O
    og = O.Mesh(O.GEOM_BOX, COARSE, LEVEL, (0, 0, 0), (1, 1, 1), 1.0, 2, 3, coarse_active=act)
    for r in range(world - 1):
        z = og.X[lays[r]["global_node"][lays[r]["upper_shared"]], 2]
        assert np.max(np.abs(z - (COARSE[2] * (r + 1) // world) / COARSE[2])) < 1e-14
