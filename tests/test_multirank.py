"""Multi-process paths of bench.py on the CPU (gloo, world size 2): the
max-over-ranks timing and whole-job rate of the replicas, and the reference
arm launched under torchrun, where rank 0 alone runs and prints."""
import json
import os
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = 10.0 + 5.0 * rank  # rank 1 is the slow one
    tmax = bench.max_over_ranks(t, dist, "cpu")
    out[rank] = (tmax, bench.job_rate(world, 1000, 4, tmax))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_time_is_max_over_ranks():
    port = 29000 + os.getpid() % 1000
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
    assert out[0][0] == out[1][0] == 15.0
    # 2 replicas x 1000 dofs x 4 steps in 15 ms
    assert abs(out[0][1] - 2 * 1000 * 4 / 15e-3 / 1e9) < 1e-15


def test_reference_arm_under_torchrun_prints_once():
    port = 30000 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--cells", "4", "--steps", "2", "--warmup", "1"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
