"""Benchmark of the matrix-free Neo-Hookean tangent operator on B200.

Workload (one "step"): one tangent vmult, tensor4 caching, FP64, on the
64^3-cell Q2 unit cube (6,440,067 DoFs): per-cell mu drawn from {1, 10} by
seed, nu = 0.3, bottom face clamped, a seeded smooth displacement field
bounded by 0.01 (det F > 0.5 checked) and a seeded source vector
uniform in [-1, 1].  The cache tables (2.9 GB) are larger than L2, so no
L2 flush is needed between timed steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl lsmf|reference]

N > 1 runs N independent replicas (one per GPU, launched with torchrun):
the operator has no exchange step in this configuration.  Rank 0 prints one
JSON line.  --impl reference times the CPU implementation of the same
operator (the oracle restatement of the reference, OpenMP over all host
cores) on the same configuration.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "large-strain-matrix-free_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

N_CELLS_1D = 64
DEGREE = 2
NU = 0.3
METRIC = "Tangent vmult GDoF/s & Newton-step time, FP32-GMG vs FP64, same 1e-8 residual"


def alg_bytes(variant, S, n_nodes, n_qp, n_cells):
    """Algorithmic bytes per vmult (values counted once, index maps excluded):
    scalar S(9N + 11Q + 10C), tensor2 S(6N + 17Q), tensor4 S(6N + 51Q);
    the referential variants: scalar_referential S(6N + 14Q) (c, the point
    displacement, metric), tensor4_ns S(6N + 90Q) (dP/dF, inverse Jacobian).
    tensor4, tensor2 and tensor4_ns cache their coefficients times JxW, so
    their records carry no JxW value."""
    if variant == "tensor4":
        return S * (6 * n_nodes + 51 * n_qp)
    if variant == "tensor2":
        return S * (6 * n_nodes + 17 * n_qp)
    if variant == "scalar_referential":
        return S * (6 * n_nodes + 14 * n_qp)
    if variant == "tensor4_ns":
        return S * (6 * n_nodes + 90 * n_qp)
    return S * (9 * n_nodes + 11 * n_qp + 10 * n_cells)


def smooth_field(X, seed, amp=0.01, modes=3):
    """Seeded smooth displacement, |u_c| <= amp: sums of sines of low wave numbers."""
    rng = np.random.default_rng(seed)
    u = np.zeros_like(X)
    for c in range(3):
        for _ in range(modes):
            k = rng.integers(1, 3, size=3)
            a = rng.uniform(-1, 1) * amp / modes
            ph = rng.uniform(0, 2 * np.pi)
            u[:, c] += a * np.sin(np.pi * (X @ k) + ph)
    return u


def min_det_f(seed, amp=0.01, modes=3, n=24):
    """Smallest det(I + grad u) of smooth_field on a sample grid (analytic gradient)."""
    rng = np.random.default_rng(seed)
    g = np.linspace(0, 1, n)
    X = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    G = np.zeros((X.shape[0], 3, 3))
    for c in range(3):
        for _ in range(modes):
            k = rng.integers(1, 3, size=3)
            a = rng.uniform(-1, 1) * amp / modes
            ph = rng.uniform(0, 2 * np.pi)
            G[:, c, :] += (a * np.pi * np.cos(np.pi * (X @ k) + ph))[:, None] * k[None, :]
    F = G + np.eye(3)[None]
    return float(np.linalg.det(F).min())


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.proc = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([s.strip() for s in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(s[0]) for s in self.samples if len(s) >= 8 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) >= 8 and s[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            if len(s) < 8:
                continue
            for nm, v in zip(names, s[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def read_traffic():
    """DRAM bytes (read + write) per launch of the tensor4 FP64 apply kernel
    at the benchmark size, from the ncu figures kept in
    profiles/ncu_traffic.json (captured on a smaller case and scaled by the
    algorithmic bytes, as recorded there)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return float(json.load(f)["apply_tensor4_fp64_64cube"]["traffic_bytes_per_launch"])


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------- CPU (oracle)
def cpu_vmult_rate(n_cells_1d, variant, fp32, steps, seed=1234):
    """Time the oracle's OpenMP vmult (the CPU implementation of the same
    operator) on the same mesh and inputs; returns (GDoF/s, seconds, n_dofs)."""
    import oracle as O
    m = O.Mesh(O.GEOM_BOX, (n_cells_1d,) * 3, 0, (0, 0, 0), (1, 1, 1), 1.0, DEGREE, DEGREE + 1)
    rng = np.random.default_rng(seed)
    mu = rng.choice([1.0, 10.0], size=m.n_cells)
    u = smooth_field(m.X, seed).reshape(-1)
    src = np.random.default_rng(seed + 1).uniform(-1, 1, m.n_dofs)
    op = O.Operator(m, variant, 1, fp32=fp32)
    op.set_material(mu, NU)
    op.set_constraints(m.constraints([(4, 7)]))
    op.cache(u.astype(np.float32) if fp32 else u)
    op.vmult(src)  # warm-up
    ts = []
    for _ in range(steps):
        t = time.perf_counter()
        op.vmult(src)
        ts.append(time.perf_counter() - t)
    t = float(np.median(ts))
    return m.n_dofs / t / 1e9, t, m.n_dofs


def omp_binding():
    """The OpenMP thread placement the CPU leg ran with."""
    bind = os.environ.get("OMP_PROC_BIND")
    places = os.environ.get("OMP_PLACES")
    if not bind and not places:
        return "no explicit pinning: OMP_PROC_BIND / OMP_PLACES unset"
    return "OMP_PROC_BIND=%s OMP_PLACES=%s" % (bind, places)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    rate, t, n_dofs = cpu_vmult_rate(args.cells, "tensor4", False, max(1, args.steps))
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "GDoF/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": "tangent vmult, tensor4 caching, FP64, %d^3-cell Q2 unit cube" % args.cells,
                       "n_dofs": n_dofs, "parallelism": "OpenMP over host cores"},
            "cpu_baseline": {"value": rate, "unit": "GDoF/s", "cores": threads, "kind": "port",
                             "sample": "%d vmults of the full %d^3 Q2 workload (median), OpenMP over all %d host "
                                       "threads (%s)" % (args.steps, args.cells, threads, omp_binding())},
            "e2e": {"value": rate, "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------- Newton step (GPU)
def voids_prm(level_precision, cells=15, refinements=2, degree=4, end_time=0.1):
    """Heterogeneous voids problem: unit cube with 16 seeded spherical voids
    of radius 0.08 removed on the coarse mesh (15^3 coarse cells, 2
    refinements: 60^3 Q2 cells, ~5 M DoFs), mu = 1, nu = 0.3, bottom face
    clamped, top face displaced by -0.01 in z (the first of 10 load steps of
    -0.1 in total), FP64 outer CG to 1e-8 relative residual, Chebyshev
    smoother of the given degree on FP32 or FP64 level operators."""
    return "\n".join([
        "subsection Finite element system", "  set Polynomial degree = 2", "  set Quadrature order = 3", "end",
        "subsection Geometry", "  set Dimension = 3", "  set Type = Box", "  set Box cells = %d, %d, %d" % ((cells,) * 3),
        "  set Global refinement = %d" % refinements, "  set Void spheres = 16, 0.08, 2024", "end",
        "subsection Material properties", "  set Shear modulus = 1", "  set Poisson's ratio = 0.3",
        "  set Formulation = 1", "end",
        "subsection Linear solver", "  set Solver type = MF_CG", "  set Residual = 1e-8",
        "  set Preconditioner type = gmg", "  set MF caching = tensor4", "  set MF level precision = %s" % level_precision,
        "  set MF Chebyshev degree = %d" % degree, "end",
        "subsection Boundary conditions", "  set Dirichlet IDs and expressions = 4:0,0,0;5:0,0,-0.01",
        "  set Dirichlet IDs and component mask = 4:true,true,true;5:false,false,true", "end",
        "subsection Time", "  set End time = %g" % end_time, "  set Time step size = 0.1", "end", ""])


def compare_level_precisions(prm_of, repeats=3, device_index=0, mu=None):
    """Solve the first load step of the problem prm_of(level_precision) with
    FP32 and with FP64 GMG levels: one untimed solve per form (the first
    solve of a problem also instantiates its V-cycle and eigenvalue-CG
    graphs and allocates work buffers, which later load steps reuse), then
    `repeats` device-timed solves per form, the two forms alternating so that
    neither always runs first after other work.  Returns per-form medians of
    the time per Newton iteration (residual + set-up + CG), the clocks seen,
    the speed-up and the relative difference of the two solutions."""
    import lsmf
    forms = (("fp32_gmg", "float"), ("fp64_gmg", "double"))
    pbs = {}
    for form, prec in forms:
        pbs[form] = lsmf.Problem(prm_of(prec))
        if mu is not None:
            pbs[form].set_mu(mu)
    for form, _ in forms:
        pbs[form].run()
    runs = {form: [] for form, _ in forms}
    sampler = ClockSampler(device_index)
    sampler.start()
    for _ in range(repeats):
        for form, _ in forms:
            res = pbs[form].run()
            st = res["steps"][0]
            total = res["time_residual"] + res["time_setup"] + res["time_solve"]
            runs[form].append((total / max(1, st["newton_iterations"]), res, st))
    clocks = sampler.stop()
    out, sols = {}, {}
    for form, _ in forms:
        rs = sorted(runs[form], key=lambda r: r[0])
        per_step, res, st = rs[len(rs) // 2]
        out[form] = {"n_dofs": pbs[form].n_dofs, "newton_iterations": st["newton_iterations"],
                     "cg_iterations": st["cg_iterations"], "s_per_newton_step": round(per_step, 4),
                     "residual_s": round(res["time_residual"], 4), "setup_s": round(res["time_setup"], 4),
                     "solve_s": round(res["time_solve"], 4), "repeats": repeats,
                     "all_s_per_newton_step": [round(r[0], 4) for r in runs[form]]}
        sols[form] = pbs[form].solution()
    del pbs
    out["clocks"] = clocks
    a, b = sols["fp32_gmg"], sols["fp64_gmg"]
    out["speedup_fp32_over_fp64"] = round(out["fp64_gmg"]["s_per_newton_step"] / out["fp32_gmg"]["s_per_newton_step"], 3)
    out["solution_rel_diff"] = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    return out


def load_steps_times(cells=15, refinements=2, device_index=0, end_time=1.0):
    """All 10 load steps of the voids problem (top face displaced by -0.1 in
    total) with FP32 and with FP64 GMG levels: one untimed run per form, then
    one device-timed run per form (FP32 first).  Reports the total time
    (residual + set-up + CG over every Newton iteration), the Newton and CG
    iteration counts of every load step, whether the counts of the two forms
    agree, and the relative difference of the final displacements."""
    import lsmf
    forms = (("fp32_gmg", "float"), ("fp64_gmg", "double"))
    pbs = {form: lsmf.Problem(voids_prm(prec, cells, refinements, end_time=end_time)) for form, prec in forms}
    for form, _ in forms:
        pbs[form].run()
    out, sols = {}, {}
    sampler = ClockSampler(device_index)
    sampler.start()
    for form, _ in forms:
        res = pbs[form].run()
        total = res["time_residual"] + res["time_setup"] + res["time_solve"]
        nits = [s["newton_iterations"] for s in res["steps"]]
        out[form] = {"load_steps": len(res["steps"]), "total_s": round(total, 4),
                     "newton_iterations": nits, "cg_iterations": [s["cg_iterations"] for s in res["steps"]],
                     "s_per_newton_step": round(total / max(1, sum(nits)), 4),
                     "residual_s": round(res["time_residual"], 4), "setup_s": round(res["time_setup"], 4),
                     "solve_s": round(res["time_solve"], 4)}
        sols[form] = pbs[form].solution()
    out["clocks"] = sampler.stop()
    del pbs
    a, b = sols["fp32_gmg"], sols["fp64_gmg"]
    out["speedup_fp32_over_fp64"] = round(out["fp64_gmg"]["total_s"] / out["fp32_gmg"]["total_s"], 3)
    out["newton_counts_equal"] = out["fp32_gmg"]["newton_iterations"] == out["fp64_gmg"]["newton_iterations"]
    out["solution_rel_diff"] = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    out["workload"] = ("voids: 60^3 Q2 cube minus 16 spheres r=0.08, tensor4, all 10 load steps (top face "
                       "-0.1 in total), CG to 1e-8")
    return out


def stage_split(mesh, mu, u64, src64, variant, reps=5):
    """MFMask breakdown of one FP64 vmult (mf_nh_operator.h:74-106, the
    reference's timing block mf_elasticity.h:2384-2435): device time of the
    basic kernel with the stages read/write (RW: gather + scatter), + sum
    factorisation (SF), + quadrature (QD: cache stream + physics), and of the
    production kernel."""
    import torch
    import lsmf
    op = lsmf.NeoHookOperator(mesh, variant, 1, "fp64")
    op.set_material(mu, NU)
    op.cache(u64)
    stream = torch.cuda.current_stream()
    op.set_stream(stream)
    dst = torch.empty_like(src64)
    out = {}

    def timed(mask):
        for _ in range(2):
            op.vmult(dst, src64, mask)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            op.vmult(dst, src64, mask)
        b.record(stream)
        torch.cuda.synchronize()
        return round(a.elapsed_time(b) / reps, 4)
    z = lsmf.MASK_ZERO
    out["rw_ms"] = timed(z | lsmf.MASK_RW)
    out["rw_sf_ms"] = timed(z | lsmf.MASK_RW | lsmf.MASK_SF)
    op.set_basic_kernel(True)
    out["rw_sf_qd_basic_ms"] = timed(lsmf.MASK_DEFAULT)
    op.set_basic_kernel(False)
    out["production_ms"] = timed(lsmf.MASK_DEFAULT)
    del op
    return out


def newton_step_times(cells=15, refinements=2, repeats=3, device_index=0):
    """One load step of the voids problem with FP32 and with FP64 level
    operators (compare_level_precisions)."""
    import lsmf
    # warm-up on a small mesh so that module loading and first-launch costs
    # are not charged to the first form
    for prec in ("float", "double"):
        lsmf.Problem(voids_prm(prec, 4, 1)).run()
    out = compare_level_precisions(lambda prec: voids_prm(prec, cells, refinements), repeats, device_index)
    out["workload"] = "voids: 60^3 Q2 cube minus 16 spheres r=0.08, tensor4, first load step, CG to 1e-8"
    return out


def adjoint_prm(cells=8, refinements=2, formulation=1, level_precision="float", scatter="atomic", voids=True):
    """Adjoint workload: the heterogeneous-voids mesh reduced to ~1 M DoFs
    (unit cube, cells^3 coarse cells minus those whose centre lies in one of
    the 16 seeded spheres of radius 0.08, refined twice: 32^3 Q2 cells less
    14 x 64, 808,587 DoFs; voids=False: the full cube, 823,875 DoFs),
    bottom clamped, traction (0.02 t, 0, -0.05 t) on
    the top face, one load step solved to a tight Newton tolerance (relative
    residual 1e-11 and update 1e-10, no absolute stop: the relative residual
    levels off near 1e-13 while the update keeps falling, so both tests pass
    with a wide margin) with GMG levels of the given precision and an FP64
    outer CG to 1e-10 of the current residual (the last Newton iteration
    starts near the residual's rounding floor, which a stricter CG cannot
    always reduce further)."""
    keys = [("Finite element system", [("Polynomial degree", 2), ("Quadrature order", 3)]),
            ("Geometry", [("Dimension", 3), ("Type", "Box"), ("Box cells", "%d, %d, %d" % ((cells,) * 3)),
                          ("Global refinement", refinements)] + ([("Void spheres", "16, 0.08, 2024")] if voids else [])),
            ("Material properties", [("Shear modulus", 1.0), ("Poisson's ratio", 0.3), ("Formulation", formulation)]),
            ("Linear solver", [("Solver type", "MF_CG"), ("Residual", 1e-10), ("Preconditioner type", "gmg"),
                               ("MF caching", "tensor4" if formulation == 1 else "scalar"),
                               ("MF level precision", level_precision), ("MF scatter", scatter)]),
            ("Nonlinear solver", [("Max iterations Newton-Raphson", 25), ("Tolerance force", 1e-11),
                                  ("Tolerance displacement", 1e-10), ("Absolute tolerance force", 1e-17),
                                  ("Absolute tolerance displacement", 1e-17)]),
            ("Boundary conditions", [("Dirichlet IDs and expressions", "4:0,0,0"),
                                     ("Dirichlet IDs and component mask", "4:true,true,true"),
                                     ("Neumann IDs and expressions", "5:0.02*t,0,-0.05*t")]),
            ("Time", [("End time", 1), ("Time step size", 1)])]
    out = []
    for sub, kv in keys:
        out.append("subsection %s" % sub)
        out += ["  set %s = %s" % (k, v) for k, v in kv]
        out.append("end")
    return "\n".join(out) + "\n"


def adjoint_times(seed=4321, fd_directions=20, h=1e-6):
    """Adjoint gradient of J = 1/2 ||u - u_target||^2 on the top face with
    respect to log mu per cell (log mu ~ N(0, 0.3^2), seeded): device-synced
    times of the forward solve and the backward (adjoint) pass, and the
    difference to central finite differences (step 1e-6 in every cell's log
    mu, seeded +-1 directions), max |fd - adjoint| / max |fd| over the
    directions."""
    import torch
    import lsmf
    pb = lsmf.Problem(adjoint_prm())
    rng = np.random.default_rng(seed)
    theta = rng.normal(0.0, 0.3, pb.n_cells)
    target = rng.uniform(-1e-3, 1e-3, pb.n_dofs)
    pb.adjoint_forward(theta, target, 5)  # warm-up
    pb.adjoint_backward()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pb.adjoint_forward(theta, target, 5)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    grad = pb.adjoint_backward()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    fd, ad = fd_check(pb, theta, target, grad, rng, fd_directions, h)
    err = float(np.max(np.abs(fd - ad)) / np.max(np.abs(fd)))
    return {"workload": "voids mesh reduced to ~1 M DoFs: 8^3 coarse cells minus 16 seeded spheres r = 0.08, refined "
                        "twice (%d Q2 cells, %d DoFs), log mu ~ N(0, 0.3^2) per cell, top-face objective"
                        % (pb.n_cells, pb.n_dofs),
            "n_dofs": pb.n_dofs, "n_cells": pb.n_cells, "forward_s": round(t1 - t0, 4),
            "backward_s": round(t2 - t1, 4), "fd_directions": fd_directions, "fd_step": h,
            "fd_rel_err": err, "fd_rel_err_definition": "max_k |fd_k - g.v_k| / max_k |fd_k|",
            "fd_directions_kind": "seeded, entries +-1 (every cell's log mu moves by the step)"}


def fd_check(pb, theta, target, grad, rng, directions, h, obj_id=5):
    """Central differences of the objective along seeded directions v_k with
    entries +-1 (every cell's log mu moves by the step h) and the adjoint's
    directional derivatives g . v_k (two arrays).  Directions of unit 2-norm
    would move each of the n cells by only h / sqrt(n): on 32^3 cells the
    objective then changes by ~1e-10 of its value over the step, below what
    the forward solves resolve (~1e-14 relative), and the difference
    quotient measures the solves' rounding instead of the derivative."""
    fd, ad = [], []
    for _ in range(directions):
        v = rng.choice([-1.0, 1.0], size=pb.n_cells)
        jp = pb.adjoint_forward(theta + h * v, target, obj_id)
        jm = pb.adjoint_forward(theta - h * v, target, obj_id)
        fd.append((jp - jm) / (2 * h))
        ad.append(grad @ v)
    return np.array(fd), np.array(ad)


def vmult_rate(cells, degree, variant, prec, reps=10, seed=77):
    """Device-timed vmult rate of one caching variant on a cells^3 unit cube
    (mu in {1, 10} per cell, smooth displacement bounded by 0.01, bottom
    clamped): GDoF/s and the fraction of the measured HBM bandwidth for the
    variant's algorithmic bytes."""
    import torch
    import lsmf
    mesh = lsmf.Mesh("box", (cells,) * 3, 0, degree=degree)
    mesh.set_dirichlet([(4, 7)])
    n_cells, n_nodes, n_dofs = mesh.info()
    X, _, _ = mesh.arrays()
    dt = torch.float64 if prec == "fp64" else torch.float32
    u = torch.tensor(smooth_field(X, seed).reshape(-1), device="cuda", dtype=dt)
    op = lsmf.NeoHookOperator(mesh, variant, 1, prec)
    op.set_material(np.random.default_rng(seed).choice([1.0, 10.0], size=n_cells), NU)
    op.cache(u)
    src = torch.tensor(np.random.default_rng(seed + 1).uniform(-1, 1, n_dofs), device="cuda", dtype=dt)
    dst = torch.empty_like(src)
    stream = torch.cuda.current_stream()
    op.set_stream(stream)
    for _ in range(3):
        op.vmult(dst, src)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        op.vmult(dst, src)
    b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    by = alg_bytes(variant, 8 if prec == "fp64" else 4, n_nodes, n_cells * (degree + 1) ** 3, n_cells)
    peak, _ = measured_peak()
    del op
    return {"n_dofs": n_dofs, "ms": round(ms, 4), "gdofs": round(n_dofs / (ms * 1e-3) / 1e9, 3),
            "frac_hbm": round(by / (ms * 1e-3) / 1e9 / peak, 3)}


def inclusions_prm(level_precision, cells=16, refinements=3, fe_degree=2):
    """128^3 Q2 unit cube (50,923,779 DoFs; fe_degree 4 with 12^3 coarse
    cells refined twice: 48^3 Q4, 21,567,171 DoFs): bottom clamped, top
    displaced by -0.01 in z (first of 10 load steps), FP64 outer CG to 1e-8,
    Chebyshev degree 4 smoother on FP32 or FP64 levels of the same element
    degree; mu is set per cell afterwards."""
    return voids_prm(level_precision, cells, refinements).replace(
        "  set Void spheres = 16, 0.08, 2024\n", "").replace(
        "  set Polynomial degree = 2", "  set Polynomial degree = %d" % fe_degree).replace(
        "  set Quadrature order = 3", "  set Quadrature order = %d" % (fe_degree + 1))


def inclusion_mu(coarse=16, refinements=3, seed=99, n_spheres=32, target_fraction=0.2):
    """mu = 10 in seeded spheres covering 20 % of the volume, 1 elsewhere,
    per fine cell of the structured unit cube (cell centres), in the cell
    order of the problem's mesh (the same coarse cells and refinements).  The
    common radius is found by bisection so that the covered fraction of the
    cells (overlaps and the parts outside the cube do not count) reaches the
    target."""
    import lsmf
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, 1, (n_spheres, 3))
    mesh = lsmf.Mesh("box", (coarse,) * 3, refinements, degree=1)
    _, _, ijk = mesh.arrays()
    xc = (ijk + 0.5) / (coarse << refinements)
    d2 = np.full(len(xc), np.inf)
    for c in centres:
        np.minimum(d2, np.sum((xc - c) ** 2, axis=1), out=d2)
    lo, hi = 0.0, 1.0
    for _ in range(60):
        r = 0.5 * (lo + hi)
        if np.mean(d2 <= r * r) < target_fraction:
            lo = r
        else:
            hi = r
    inside = d2 <= hi * hi
    return np.where(inside, 10.0, 1.0), float(inside.mean())


def c5_measurements(repeats=3):
    """The large configurations: vmult rates at 128^3 Q2 and 48^3 Q4
    (tensor4, FP64 and FP32), and one Newton iteration of the 128^3 Q2
    inclusion problem with FP32 and with FP64 GMG levels."""
    out = {"vmult": {}}
    for cells, degree in ((128, 2), (48, 4)):
        for prec in ("fp64", "fp32"):
            out["vmult"]["%d^3_Q%d_tensor4_%s" % (cells, degree, prec)] = vmult_rate(cells, degree, "tensor4", prec)
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    mu, frac = inclusion_mu()
    out.update(compare_level_precisions(inclusions_prm, repeats, dev, mu))
    out["workload"] = ("inclusions: 128^3 Q2 unit cube, mu = 10 in 32 seeded spheres (%.1f %% of the cells), "
                       "tensor4, first load step, CG to 1e-8" % (100 * frac))
    # the same inclusion field on 48^3 Q4 cells (Q4 multigrid levels 12^3, 24^3, 48^3)
    mu4, frac4 = inclusion_mu(coarse=12, refinements=2)
    q4 = compare_level_precisions(lambda prec: inclusions_prm(prec, 12, 2, fe_degree=4), repeats, dev, mu4)
    q4["workload"] = ("inclusions: 48^3 Q4 unit cube, mu = 10 in 32 seeded spheres (%.1f %% of the cells), "
                      "tensor4, first load step, CG to 1e-8" % (100 * frac4))
    out["q4_newton"] = q4
    return out


def dist_vmult_times(cells=N_CELLS_1D, n_parts_list=(2, 4), seed=1234, reps=20):
    """The distributed operator at the benchmark size on one GPU: the
    cells^3 Q2 cube split into n z-slab parts (each part's operator on its
    own stream, in-process group), tensor4 FP64, with both interface
    exchanges: packed (ghost update and compress(add) through buffers) and
    fused (the cell loops read and add to the neighbours' vectors); host
    wall-clock per vmult over `reps` after 3 warm-ups (several streams:
    synchronised on both sides), against the whole-mesh vmult timed the same
    way, and the largest difference on the owned entries."""
    import torch
    import lsmf
    kw = dict(geometry="box", coarse=(cells,) * 3, n_refinements=0, degree=DEGREE)
    gm = lsmf.Mesh(**kw)
    gm.set_dirichlet([(4, 7)])
    nc, nn, nd = gm.info()
    X, _, ijk = gm.arrays()
    rng = np.random.default_rng(seed)
    mu = rng.choice([1.0, 10.0], nc)
    u = smooth_field(X, seed).reshape(-1)
    src = rng.uniform(-1, 1, nd)
    gop = lsmf.NeoHookOperator(gm, "tensor4", 1, "fp64")
    gop.set_material(mu, NU)
    gop.cache(torch.tensor(u, device="cuda"))
    dsrc = torch.tensor(src, device="cuda")
    want = torch.empty_like(dsrc)

    def wall(f):
        for _ in range(3):
            f()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(reps):
            f()
        torch.cuda.synchronize()
        return (time.perf_counter() - t) / reps * 1e3

    out = {"workload": "%d^3 Q2 cube, tensor4 FP64, z-slab parts on one GPU" % cells, "n_dofs": nd,
           "whole_ms": round(wall(lambda: gop.vmult(want, dsrc)), 4), "timing": "host wall-clock, synchronised"}
    want_h = want.cpu().numpy()
    del gop
    cell_of = {tuple(c): i for i, c in enumerate(ijk.tolist())}
    for n_parts in n_parts_list:
        parts = []
        for r in range(n_parts):
            pm = lsmf.Mesh(n_parts=n_parts, part=r, **kw)
            pm.set_dirichlet([(4, 7)])
            lay = lsmf.partition_layout(n_parts, r, **kw)
            _, _, pijk = pm.arrays()
            gd = (3 * lay["global_node"][:, None] + np.arange(3)).reshape(-1)
            owned = np.ones(lay["n_nodes"], dtype=bool)
            owned[lay["upper_shared"]] = False
            op = lsmf.NeoHookOperator(pm, "tensor4", 1, "fp64")
            op.set_stream(torch.cuda.Stream())
            op.set_material(mu[[cell_of[tuple(c)] for c in pijk.tolist()]], NU)
            op.cache(torch.tensor(u[gd], device="cuda"))
            s_ = torch.tensor(src[gd], device="cuda")
            parts.append(dict(op=op, gd=gd, od=(3 * np.nonzero(owned)[0][:, None] + np.arange(3)).reshape(-1),
                              src=s_, dst=torch.empty_like(s_)))
        D = lsmf.Dist.group([p["op"] for p in parts])
        rec = {}
        for mode in ("packed", "fused"):
            D.set_exchange(mode)
            t = wall(lambda: D.vmult([p["dst"] for p in parts], [p["src"] for p in parts]))
            err = max(float(np.max(np.abs(p["dst"].cpu().numpy()[p["od"]] - want_h[p["gd"][p["od"]]])))
                      for p in parts)
            rec[mode] = {"ms": round(t, 4), "overhead": round(t / out["whole_ms"] - 1.0, 4),
                         "rel_err_owned": err / float(np.max(np.abs(want_h)))}
        out["parts_%d" % n_parts] = rec
        del D, parts
        torch.cuda.empty_cache()
    return out


def max_over_ranks(t_ms, dist, device):
    """The slowest rank's time (every rank takes part; a single process
    returns its own)."""
    if not dist:
        return t_ms
    import torch
    tt = torch.tensor([float(t_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def job_rate(world, n_dofs, steps, t_ms):
    """Whole-job GDoF/s: every rank (replica) applies the operator to its own
    n_dofs vector once per step; t_ms is the max-over-ranks time of `steps`
    steps."""
    return world * n_dofs * steps / (t_ms * 1e-3) / 1e9


def profile_vcycle(cells=15, refinements=1):
    """One FP32 V-cycle of the cells^3 -> (cells 2^refinements)^3 Q2 hierarchy
    (tensor4, Chebyshev degree 4, reference coarse solver) launched kernel by
    kernel between cudaProfilerStart / Stop, so that a profiler started with
    profiling off (ncu --profile-from-start off) records exactly that V-cycle."""
    import torch
    import lsmf
    mesh = lsmf.Mesh("box", (cells,) * 3, refinements, degree=2)
    mesh.set_dirichlet([(4, 7)])
    nc, nn, nd = mesh.info()
    X, _, _ = mesh.arrays()
    u = torch.tensor(smooth_field(X, 1).reshape(-1), device="cuda")
    g = lsmf.GMG(mesh, "tensor4", 1, "fp32", degree=4)
    g.set_material(np.ones(nc), NU)
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
    print(json.dumps({"profile_vcycle": "done", "coarse_level": g.level_info(0).tolist()}), flush=True)
    return 0


def profile_setup(cells=15, refinements=2, precision="fp32"):
    """One multigrid set-up (level caches, diagonals, Chebyshev eigenvalue
    estimates, the coarse solver's accurate estimate) of the cells^3 ->
    (cells 2^refinements)^3 Q2 tensor4 hierarchy, Chebyshev degree 4, between
    cudaProfilerStart / Stop after one untimed set-up; prints its
    event-timed duration."""
    import torch
    import lsmf
    mesh = lsmf.Mesh("box", (cells,) * 3, refinements, degree=2)
    mesh.set_dirichlet([(4, 7)])
    nc, nn, nd = mesh.info()
    X, _, _ = mesh.arrays()
    u = torch.tensor(smooth_field(X, 1).reshape(-1), device="cuda")
    g = lsmf.GMG(mesh, "tensor4", 1, precision, degree=4)
    g.set_material(np.ones(nc), NU)
    g.setup(u)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.profiler.start()
    a.record(stream)
    g.setup(u)
    b.record(stream)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"profile_setup": "done", "ms": round(a.elapsed_time(b), 3),
                      "levels": [g.level_info(l).tolist() for l in range(mesh.n_levels)]}), flush=True)
    return 0


def profile_pairs(sizes=(48, 15)):
    """One FP32 vmult per (cells^3 Q2 cube, tensor4 / tensor2, one cell per
    warp / cell pairs), plain record loads, no warm-up: the launches that an
    ncu capture of apply_fast_kernel and apply_pair_kernel compares."""
    import torch
    import lsmf
    for n in sizes:
        mesh = lsmf.Mesh("box", (n,) * 3, 0, degree=2)
        mesh.set_dirichlet([(4, 7)])
        nc, nn, nd = mesh.info()
        X, _, _ = mesh.arrays()
        mu = np.random.default_rng(1).choice([1.0, 10.0], nc)
        u = torch.tensor(smooth_field(X, 3).reshape(-1), device="cuda").float()
        src = torch.tensor(np.random.default_rng(2).uniform(-1, 1, nd), device="cuda").float()
        for variant in ("tensor4", "tensor2"):
            op = lsmf.NeoHookOperator(mesh, variant, 1, "fp32")
            op.set_material(mu, NU)
            op.cache(u)
            op.set_pipeline(0)
            for pairs in (0, 1):
                op.set_cell_pairs(pairs)
                dst = torch.empty_like(src)
                op.vmult(dst, src)
            torch.cuda.synchronize()
            del op
    print(json.dumps({"profile_pairs": "done", "sizes": list(sizes)}), flush=True)
    return 0


# ---------------------------------------------------------------- GPU (lsmf)
def run_lsmf(args):
    import torch
    import lsmf

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        # replicas: every rank runs the headline vmult and the end-to-end
        # pass; the single-GPU diagnostics (variants, large meshes, Newton,
        # adjoint) and the CPU baseline belong to the N = 1 run
        args.no_variants = args.no_large = args.no_newton = args.no_adjoint = args.no_cpu = True

    seed = 1234
    assert min_det_f(seed) > 0.5
    mesh = lsmf.Mesh("box", (args.cells,) * 3, 0, degree=DEGREE)
    mesh.set_dirichlet([(4, 7)])
    n_cells, n_nodes, n_dofs = mesh.info()
    X, _, _ = mesh.arrays()
    rng = np.random.default_rng(seed)
    mu = rng.choice([1.0, 10.0], size=n_cells)
    u_h = smooth_field(X, seed).reshape(-1)
    src_h = np.random.default_rng(seed + 1).uniform(-1, 1, n_dofs)
    n_qp = n_cells * (DEGREE + 1) ** 3
    u64 = torch.tensor(u_h, device="cuda")
    u32 = u64.float()
    src64 = torch.tensor(src_h, device="cuda")
    src32 = src64.float()

    def make(variant, prec):
        op = lsmf.NeoHookOperator(mesh, variant, 1, prec)
        op.set_material(mu, NU)
        op.cache(u64 if prec == "fp64" else u32)
        return op

    op = make("tensor4", "fp64")
    dst = torch.empty_like(src64)
    stream = torch.cuda.current_stream()
    lib = lsmf.lib()
    lib.lsmf_operator_set_stream(op.h, lsmf.vp(stream.cuda_stream))

    for _ in range(args.warmup):
        op.vmult(dst, src64)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        op.vmult(dst, src64)
    e1.record(stream)
    torch.cuda.synchronize()
    t_ms = e0.elapsed_time(e1)
    # kernel-level timing for the roofline (apply kernel + constrained rows)
    ts = []
    for _ in range(args.steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        op.vmult_add(dst, src64)
        b.record(stream)
        ts.append((a, b))
    torch.cuda.synchronize()
    apply_ms = float(np.mean([a.elapsed_time(b) for a, b in ts]))
    clocks = sampler.stop()
    t_ms = max_over_ranks(t_ms, dist, "cuda")
    value = job_rate(world, n_dofs, args.steps, t_ms)

    # per-variant rates (same mesh / inputs)
    variants = {}
    peak, peak_kind = measured_peak()
    for variant in () if args.no_variants else ("tensor4", "tensor2", "scalar", "scalar_referential", "tensor4_ns"):
        for prec in ("fp64", "fp32"):
            if variant == "tensor4" and prec == "fp64":
                v_op, s_in = op, src64
            else:
                v_op = make(variant, prec)
                s_in = src64 if prec == "fp64" else src32
                lib.lsmf_operator_set_stream(v_op.h, lsmf.vp(stream.cuda_stream))
            d_out = torch.empty_like(s_in)
            for _ in range(2):
                v_op.vmult(d_out, s_in)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = 5
            a.record(stream)
            for _ in range(reps):
                v_op.vmult(d_out, s_in)
            b.record(stream)
            torch.cuda.synchronize()
            ms = a.elapsed_time(b) / reps
            by = alg_bytes(variant, 8 if prec == "fp64" else 4, n_nodes, n_qp, n_cells)
            variants["%s_%s" % (variant, prec)] = {
                "gdofs": round(n_dofs / (ms * 1e-3) / 1e9, 3), "ms": round(ms, 4),
                "alg_GBps": round(by / (ms * 1e-3) / 1e9, 1), "frac_hbm": round(by / (ms * 1e-3) / 1e9 / peak, 3)}
            if v_op is not op:
                del v_op
    if not args.no_variants:
        # the bit-reproducible scatters beside the atomic default, tensor4
        # FP64: 8 colour launches with plain adds, and one cell loop into a
        # per-cell buffer followed by per-node sums in cell order
        for mode in ("colour8", "nodesum"):
            op.set_scatter(mode)
            d_out = torch.empty_like(src64)
            for _ in range(2):
                op.vmult(d_out, src64)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(5):
                op.vmult(d_out, src64)
            b.record(stream)
            torch.cuda.synchronize()
            ms = a.elapsed_time(b) / 5
            by = alg_bytes("tensor4", 8, n_nodes, n_qp, n_cells)
            variants["tensor4_fp64_" + mode] = {
                "gdofs": round(n_dofs / (ms * 1e-3) / 1e9, 3), "ms": round(ms, 4),
                "alg_GBps": round(by / (ms * 1e-3) / 1e9, 1), "frac_hbm": round(by / (ms * 1e-3) / 1e9 / peak, 3)}
        op.set_scatter("atomic")

    # end to end through the public API with host buffers: every step copies
    # its source from pinned host memory and its result back; the copies of
    # neighbouring steps run on their own streams and overlap the vmult
    # (double-buffered device vectors, event-ordered)
    nbuf = 2
    src_pin = [torch.tensor(src_h).pin_memory() for _ in range(nbuf)]
    dst_pin = [torch.empty(n_dofs, dtype=torch.float64).pin_memory() for _ in range(nbuf)]
    d_src = [torch.empty_like(src64) for _ in range(nbuf)]
    d_dst = [torch.empty_like(src64) for _ in range(nbuf)]
    # non-blocking streams for the copies and the vmult (the legacy default
    # stream would serialise with both copy streams)
    s_h2d, s_d2h, s_cmp = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    lib.lsmf_operator_set_stream(op.h, lsmf.vp(s_cmp.cuda_stream))
    ev_in = [torch.cuda.Event() for _ in range(nbuf)]
    ev_done = [torch.cuda.Event() for _ in range(nbuf)]
    ev_out = [torch.cuda.Event() for _ in range(nbuf)]

    def e2e_steps(k):
        for i in range(k):
            j = i % nbuf
            with torch.cuda.stream(s_h2d):
                if i >= nbuf:
                    s_h2d.wait_event(ev_done[j])  # vmult i-2 finished reading d_src[j]
                d_src[j].copy_(src_pin[j], non_blocking=True)
                ev_in[j].record(s_h2d)
            s_cmp.wait_event(ev_in[j])
            if i >= nbuf:
                s_cmp.wait_event(ev_out[j])      # D2H i-2 finished reading d_dst[j]
            op.vmult(d_dst[j], d_src[j])
            ev_done[j].record(s_cmp)
            with torch.cuda.stream(s_d2h):
                s_d2h.wait_event(ev_done[j])
                dst_pin[j].copy_(d_dst[j], non_blocking=True)
                ev_out[j].record(s_d2h)

    e2e_steps(2 * nbuf)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s_h2d)
    e2e_steps(args.steps)
    s_h2d.wait_stream(s_d2h)
    s_h2d.wait_stream(s_cmp)
    b.record(s_h2d)
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b) / args.steps
    assert torch.allclose(d_dst[(args.steps - 1) % nbuf], dst_pin[(args.steps - 1) % nbuf].cuda())
    e2e_ms = max_over_ranks(e2e_ms, dist, "cuda")
    # the bound of the e2e step: the same two copies (one each way, the
    # same pinned buffers) running concurrently with no vmult
    def duplex_ms(k=10):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(s_h2d)
        s_d2h.wait_stream(s_h2d)
        for i in range(k):
            with torch.cuda.stream(s_h2d):
                d_src[i % nbuf].copy_(src_pin[i % nbuf], non_blocking=True)
            with torch.cuda.stream(s_d2h):
                dst_pin[i % nbuf].copy_(d_dst[i % nbuf], non_blocking=True)
        s_h2d.wait_stream(s_d2h)
        b.record(s_h2d)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / k
    duplex_ms()
    link_ms = duplex_ms()
    e2e = {"value": job_rate(world, n_dofs, 1, e2e_ms), "unit": "GDoF/s",
           "h2d_bytes_per_step": n_dofs * 8, "d2h_bytes_per_step": n_dofs * 8,
           "pipelining": "H2D(i+1) and D2H(i-1) overlap vmult(i), double-buffered",
           "link_ms_per_step": round(link_ms, 4),
           "link_GBps_each_way": round(n_dofs * 8 / (link_ms * 1e-3) / 1e9, 1),
           "frac_of_link": round(link_ms / e2e_ms, 3),
           "link_definition": "the step's H2D and D2H copies run concurrently without the vmult (measured here)"}
    lib.lsmf_operator_set_stream(op.h, lsmf.vp(stream.cuda_stream))
    # release the section's pinned buffers, device vectors and streams
    torch.cuda.synchronize()
    del src_pin, dst_pin, d_src, d_dst, s_h2d, s_d2h, s_cmp, ev_in, ev_done, ev_out

    alg = alg_bytes("tensor4", 8, n_nodes, n_qp, n_cells)
    achieved = alg / (apply_ms * 1e-3) / 1e9
    traffic = read_traffic()
    chunks = op.get_option(8)
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "peak_kind": peak_kind, "alg_bytes_per_launch": alg,
                "kernel": "apply_fast_kernel<2,3,double,tensor4,1 stage>",
                "chunks": chunks,
                "timed": "the cell loop of one vmult_add (its %d concurrent chunks forked from and joined back into "
                         "the timing stream) plus the identity rows, CUDA events on that stream" % chunks}

    # MFMask stage breakdown (RW / SF / QD) of the FP64 variants
    stages = {}
    if not args.no_variants:
        for variant in ("tensor4", "tensor2", "scalar"):
            stages[variant] = stage_split(mesh, mu, u64, src64, variant)

    # the large single-GPU configurations: tensor4 vmults at 48^3 Q4 and
    # 128^3 Q2 (24.4 GB of FP64 records)
    large = {}
    dist_parts = None
    if not args.no_variants and not args.no_large:
        del op
        torch.cuda.empty_cache()
        # the z-slab distributed operator at the benchmark size, on this GPU
        dist_parts = dist_vmult_times(args.cells)
        torch.cuda.empty_cache()
        for cells, degree in ((48, 4), (128, 2)):
            for prec in ("fp64", "fp32"):
                large["%d^3_Q%d_tensor4_%s" % (cells, degree, prec)] = vmult_rate(cells, degree, "tensor4", prec)
                torch.cuda.empty_cache()

    newton = None
    load_steps = None
    if not args.no_newton:
        torch.cuda.synchronize()
        newton = newton_step_times(device_index=local)
        load_steps = load_steps_times(device_index=local)

    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_times()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        rate, t, _ = cpu_vmult_rate(args.cells, "tensor4", False, 5)
        cpu = {"value": rate, "unit": "GDoF/s", "cores": threads, "kind": "port",
               "sample": "5 vmults (median) of the full %d^3 Q2 tensor4 FP64 workload, OpenMP over all %d host "
                         "threads (%s)" % (args.cells, threads, omp_binding())}

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 4), "unit": "GDoF/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_ms / args.steps, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded mu field, smooth displacement, random source)",
                "config": {"workload": "tangent vmult, tensor4 caching, FP64, %d^3-cell Q2 unit cube" % args.cells,
                           "n_dofs": n_dofs, "n_cells": n_cells, "degree": DEGREE,
                           "parallelism": "replicas" if world > 1 else "single GPU",
                           "l2": "inputs larger than L2 (2.9 GB cache tables), no flush"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                # per vmult: one apply launch per chunk and one identity-row
                # launch (the clamped bottom face lies in the first chunk)
                "gpu_launches": (chunks + 1) * args.steps, "clocks": clocks, "variants": variants,
                "stage_split_fp64": stages, "large_vmults": large, "dist_vmult_one_gpu": dist_parts,
                "newton_step": newton, "newton_load_steps": load_steps, "adjoint": adjoint}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lsmf", choices=["lsmf", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-variants", action="store_true", help="skip the per-variant table")
    ap.add_argument("--no-newton", action="store_true", help="skip the FP32-GMG vs FP64 Newton-step comparison")
    ap.add_argument("--newton-only", action="store_true", help="only the Newton-step comparison")
    ap.add_argument("--newton-cells", type=int, default=15, help="coarse cells per direction of the voids mesh")
    ap.add_argument("--newton-refinements", type=int, default=2)
    ap.add_argument("--cells", type=int, default=N_CELLS_1D, help="cells per direction (64 = the benchmark)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-gradient timing")
    ap.add_argument("--no-large", action="store_true", help="skip the 48^3 Q4 / 128^3 Q2 vmults")
    ap.add_argument("--profile-vcycle", action="store_true",
                    help="only one FP32 V-cycle between cudaProfilerStart / Stop (for ncu --profile-from-start off)")
    ap.add_argument("--profile-cells", type=int, default=15, help="coarse cells per direction of --profile-vcycle")
    ap.add_argument("--profile-refinements", type=int, default=1, help="refinements of --profile-vcycle")
    ap.add_argument("--profile-setup", action="store_true",
                    help="only one FP32 multigrid set-up of the 15^3 -> 60^3 hierarchy between cudaProfilerStart / Stop")
    ap.add_argument("--profile-pairs", action="store_true",
                    help="only one FP32 vmult per (48^3 / 15^3, tensor4 / tensor2, one cell / cell pairs) for ncu")
    ap.add_argument("--c5", action="store_true",
                    help="only the large configurations (128^3 Q2, 48^3 Q4 vmults; 128^3 inclusion Newton step)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_vcycle:
        return profile_vcycle(args.profile_cells, args.profile_refinements)
    if args.profile_pairs:
        return profile_pairs()
    if args.profile_setup:
        return profile_setup()
    if args.c5:
        print(json.dumps(c5_measurements()), flush=True)
        return 0
    if args.newton_only:
        print(json.dumps(newton_step_times(args.newton_cells, args.newton_refinements,
                                           device_index=int(os.environ.get("LOCAL_RANK", "0")))), flush=True)
        return 0
    return run_lsmf(args)


if __name__ == "__main__":
    sys.exit(main())
