"""One FP32 V-cycle of the voids-free 15^3 -> 30^3 Q2 hierarchy (tensor4,
Chebyshev degree 4, reference coarse solver), launched kernel by kernel
between cudaProfilerStart / Stop so that an ncu launch list
(--profile-from-start off) covers exactly that V-cycle.

    python profiles/vcycle_launches.py && \\
    ncu --metrics gpu__time_duration.sum --clock-control none --profile-from-start off \\
        --csv --log-file vcycle_launches.csv python profiles/vcycle_launches.py
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "large-strain-matrix-free_b200"))

import numpy as np  # noqa: E402
import torch  # noqa: E402

import bench  # noqa: E402
import lsmf  # noqa: E402

mesh = lsmf.Mesh("box", (15, 15, 15), 1, degree=2)
mesh.set_dirichlet([(4, 7)])
nc, nn, nd = mesh.info()
X, _, _ = mesh.arrays()
u = torch.tensor(bench.smooth_field(X, 1).reshape(-1), device="cuda")
g = lsmf.GMG(mesh, "tensor4", 1, "fp32", degree=4)
g.set_material(np.ones(nc), 0.3)
g.set_graph(False)
g.setup(u)
b = torch.tensor(np.random.default_rng(0).uniform(-1, 1, nd), device="cuda")
b[torch.tensor(mesh.constraint_mask() == 1, device="cuda")] = 0
x = torch.empty_like(b)
g.vmult(x, b)
torch.cuda.synchronize()
torch.cuda.profiler.start()
g.vmult(x, b)
torch.cuda.synchronize()
torch.cuda.profiler.stop()
print("coarse level:", g.level_info(0).tolist())
