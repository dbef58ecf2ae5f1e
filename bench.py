"""Throughput of the element loop: incompatible-mode Hex8 tangent + residual +
assembly, element updates per second, FP64.

Workload (one step): NonlinearSystem.evaluate(u, 0, want_tangent=True) on
the element-kernel microbenchmark - a 1000 x 500 x 2 sheet of 0.04 x 0.04 x
0.5 mm cells (1,000,000 incompatible-mode Hex8, 8 points each), Hill48 +
two-term Chaboche with Voce hardening, logarithmic strain, a committed
plastic history and an increment that makes about 40 % of the points yield
(springback-precomp_b200/workload.py). One step is the element kernel
(local Newton, condensation), the gather of f_int / gross / energy / yield
count and the gather of the tangent into the 283.8M-entry CSC pattern.

`value` is elements / s with the inputs resident on the device; `e2e` the
same through the C ABI with host buffers: u copied in from pinned memory
and f_int plus the tangent values copied back, every step. Under torchrun
every rank evaluates its own part (independent meshes, no collective on the
data path; weak scaling); the time is the max over ranks.

--workload partition measures the free-free block of a Dirichlet partition
(PartitionedFactor): its gather from the full tangent, and the device
factorisation and solve it feeds.

--workload adjoint measures the adjoint springback sensitivity: a sheet part
with a frozen end-of-forming history released onto 3-2-1 supports, the
gradient of the RMS springback of its top face with respect to a 20 x 20
bicubic grid of commanded heights (torch.autograd through the release
solve), its cost against one release solve, and its agreement with central
differences (h = 1e-6 mm) along seeded random directions.

--impl reference times the reference's CPU algorithm - the oracle's
restatement of it (the reference needs Eigen, which this image lacks) - on
all host cores, on a bounded sample of the same workload per step.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "springback-precomp_b200"
METRIC = "Hex8 tangent+residual+assembly elem/s (FP64)"
# DRAM bytes (read + write) per element of one evaluation's K1: ncu's
# dram__bytes_read.sum + dram__bytes_write.sum summed over the phase kernels
# of one evaluation of the same construction at 80,000 elements (200 x 200 x
# 2): 16.57 GB (pre 4.48, return 5.41, log map 2.09, post 2.94, control
# 0.48, condense 0.81, the single kernel's share 0.36); the traffic grows
# with the elements, so an evaluation of ne elements moves about ne times
# this.
K1_DRAM_BYTES_PER_ELEMENT = 16.57e9 / 80000
# The single kernel (--local-iteration single): 0.69 + 5.28 GB in one launch
# at 80,000 elements.
K1_SINGLE_DRAM_BYTES_PER_ELEMENT = (0.692594688e9 + 5.275133e9) / 80000
# The same for the standard Hex8 kernel: 0.192 GB read + 1.610 GB written in
# one launch at 80,000 elements.
K1S_DRAM_BYTES_PER_ELEMENT = (0.191949568e9 + 1.610487e9) / 80000
# DRAM bytes per block entry of one free-free gather (assemble): the same ncu
# metrics over one launch on the 200 x 200 x 2 sheet's block, 271.0 MB read +
# 139.0 MB written for 22,528,485 entries.
GATHER_DRAM_BYTES_PER_ENTRY = (271.010304e6 + 139.048192e6) / 22528485
UNIT = "elem/s"


def oracle_module():
    """The oracle (test infrastructure), for the CPU-baseline legs only."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.build()
    return oracle


def oracle_problem(orc, nx, ny, nz, seed):
    """A sample problem of the same construction, built with the oracle on
    the CPU (no GPU on the reference arm's path)."""
    wl = importlib.import_module(PKG + ".workload")
    device_to_oracle, oracle_to_device = orc.device_to_oracle, orc.oracle_to_device

    def evaluate(mesh, mat, u, state, alpha, want_yield=False):
        nt = mat.kinematic_terms
        r = orc.elements(mat.as_dict(), mesh.element_coordinates(), mesh.gather(u), device_to_oracle(state, nt),
                         alpha, want_tangent=False)
        out = (oracle_to_device(r["states"], nt), r["alpha"], r["status"])
        return out + ((r["yield_flags"],) if want_yield else ())

    prob = wl.make_problem(nx, ny, nz, seed=seed, evaluate=evaluate, sample=min(1024, nx * ny * nz))
    return prob, device_to_oracle(prob.state, prob.material.kinematic_terms)


def time_oracle(orc, prob, committed, threads, min_seconds):
    """elements/s of the oracle's NonlinearSystem::evaluate (element loop on
    `threads` OpenMP threads, serial gather and scatter) on the sample."""
    mesh, mat = prob.mesh, prob.material
    pat = orc.pattern(mesh.num_nodes, mesh.connectivity)
    orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, prob.u, committed, prob.alpha,
                        threads=threads, pat=pat)
    times = []
    t_end = time.perf_counter() + min_seconds
    while time.perf_counter() < t_end or len(times) < 3:
        t0 = time.perf_counter()
        r = orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, prob.u, committed, prob.alpha,
                                threads=threads, pat=pat)
        times.append(time.perf_counter() - t0)
        assert r["code"] == 0
    return mesh.num_elements / statistics.median(times), len(times)


def cpu_count():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def __enter__(self):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=self.file,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()

    def summary(self):
        self.file.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def fp64_peak_tflops(torch, dev):
    """Measured FP64 peak of this GPU: a cuBLAS DGEMM (8192^3, best of 5)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def run_reference(args, rank, world):
    """The reference arm: the oracle port (the reference's CPU algorithm:
    OpenMP static schedule over elements, serial scatter in element order)
    built -O3 -march=native for this host's CPU, on all host cores, one
    evaluation of a bounded sample of the same workload per step; beside it
    the same on one thread on a smaller sample."""
    if rank != 0:
        return 0
    orc = oracle_module()
    orc.use_variant("fast")
    nx, ny, nz = args.ref_nx, args.ref_ny, args.nz
    prob, committed = oracle_problem(orc, nx, ny, nz, seed=7)
    cores = cpu_count()
    mesh, mat = prob.mesh, prob.material
    pat = orc.pattern(mesh.num_nodes, mesh.connectivity)
    std = args.element == "standard"
    with orc.element(std, True):
        for _ in range(args.warmup):
            orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, prob.u, committed, prob.alpha,
                                threads=cores, pat=pat)
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            r = orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, prob.u, committed, prob.alpha,
                                    threads=cores, pat=pat)
            times.append(time.perf_counter() - t0)
            assert r["code"] == 0
    dt = sum(times) / len(times)
    value = mesh.num_elements / dt
    # One thread, on the small sample (bounded to a few seconds).
    small, small_committed = oracle_problem(orc, args.sample_nx, args.sample_ny, nz, seed=7)
    with orc.element(std, True):
        one_rate, n_one = time_oracle(orc, small, small_committed, 1, 4.0)
    sample = (f"{mesh.num_elements} elements ({nx}x{ny}x{nz} of the same sheet, law and history construction) "
              f"per step, {cores} threads; single thread on {small.mesh.num_elements} elements "
              f"({args.sample_nx}x{args.sample_ny}x{nz}), median of {n_one} runs")
    cpu = {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
           "single_thread": one_rate, "median_step_ms": statistics.median(times) * 1e3,
           "build": orc.FAST_FLAGS, "cpu": cpu_model()}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(args, world), "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_baseline_subprocess(args):
    """The reference arm's measurement, run as its own process before this
    process touches the GPU (so that no CUDA or torch thread shares the host
    cores with it), with fewer steps; its cpu_baseline object."""
    cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--steps", str(args.cpu_steps),
           "--warmup", "3", "--nz", str(args.nz), "--ref-nx", str(args.ref_nx), "--ref-ny", str(args.ref_ny),
           "--sample-nx", str(args.sample_nx), "--sample-ny", str(args.sample_ny), "--element", args.element]
    env = dict(os.environ)
    env["CUDA_VISIBLE_DEVICES"] = ""
    out = subprocess.run(cmd, check=True, capture_output=True, text=True, env=env).stdout
    line = json.loads([ln for ln in out.splitlines() if ln.startswith("{")][-1])
    cpu = line["cpu_baseline"]
    cpu["sample"] += f"; {args.cpu_steps} timed steps in a separate process before the GPU work"
    return cpu


def run_batched(args, rank, world):
    """The batched design sweep: the parts of the sweep configuration - a
    scrambled Sobol sequence over four families (dome, truncated cone,
    elliptic cone of axis ratio 1.0-1.6, pyramid), footprint 15-20 mm, depth
    2-4 mm, wall 30-55 degrees, 20k-150k Hex8 each in two layers - with the
    microbenchmark's material. One sweep = `sweep_increments` forming
    increments of every part towards its shape (to 15 % of its depth, the
    sheet laid on the scaled surface): each increment two Newton iterations'
    evaluations with the tangent, then the commit - the element loop's work
    of the parts' forming runs; the solves are the reference's own and stay
    out. Timed one part at a time (each part's system made, its increments
    timed on the device, released), against all parts as one batched system
    whose thread mapping the autotuner picks first. Reported: parts per hour
    of both."""
    import torch

    if world > 1 and rank != 0:
        return 0
    pkg = importlib.import_module(PKG)
    batch_mod = importlib.import_module(PKG + ".batch")
    wl = importlib.import_module(PKG + ".workload")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    mat = pkg.material.hill_chaboche_sheet()
    parts = wl.sweep_parts(args.parts)
    meshes = [m for _, m in parts]
    K, depth = args.sweep_increments, 0.15
    total = sum(m.num_elements for m in meshes)
    stream = torch.cuda.current_stream()

    # The increments' displacements, once for both runs (host memory).
    disps = [[(wl.formed_positions(m, part, (k + 1) * depth / K) - m.coords).reshape(-1) for k in range(K)]
             for part, m in parts]

    def run_increments(system, us):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        yielding = 0
        for k in range(K):
            for _ in range(2):
                ev = system.evaluate(us[k], 0.0, True)
            yielding = ev.yielding_points
            system.commit()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), yielding

    # One part at a time.
    seq_ms, per_part = 0.0, []
    for (part, mesh), dp in zip(parts, disps):
        sy = pkg.NonlinearSystem(mesh, mat)
        us = [torch.tensor(d, device=dev) for d in dp]
        ms, _ = run_increments(sy, us)
        seq_ms += ms
        per_part.append(ms)
        sy.close()
        del us
    torch.cuda.empty_cache()
    # All parts as one system.
    t0 = time.perf_counter()
    batch = batch_mod.PartBatch(meshes, mat)
    ub = [torch.tensor(np.concatenate([dp[k] for dp in disps]), device=dev) for k in range(K)]
    build_s = time.perf_counter() - t0
    tune = batch.autotune(ub[0])
    bat_ms, yielding = run_increments(batch.system, ub)
    line = {"metric": "batched design sweep: parts/h of the element loop (FP64)",
            "value": args.parts / (bat_ms / 1e3) * 3600.0,
            "unit": "parts/h", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": bat_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.parts} parts (Sobol over dome, truncated cone, elliptic cone, pyramid; "
                                   f"footprint 15-20 mm, depth 2-4 mm, wall 30-55 deg), {total} IM Hex8 in all "
                                   f"(20k-150k each, 2 layers), Hill48 + Chaboche + Voce, logarithmic strain; one "
                                   f"step = {K} forming increments of every part, each 2 evaluations with the "
                                   "tangent and a commit"},
            "sequential_parts_per_hour": args.parts / (seq_ms / 1e3) * 3600.0,
            "sequential_ms": seq_ms, "batched_ms": bat_ms, "speedup": seq_ms / bat_ms,
            "elements_per_s_batched": 2 * K * total / (bat_ms / 1e3),
            "elements_per_s_sequential": 2 * K * total / (seq_ms / 1e3),
            "autotune_ms": {f"{m}/{e}": t for (m, e), t in tune.items()}, "chosen": list(batch.chosen),
            "batch_build_s": build_s, "yielding_fraction": yielding / (8.0 * total),
            "part_ms_min_max": [min(per_part), max(per_part)]}
    print(json.dumps(line), flush=True)
    return 0


def sheet_partition(pkg, torch, nx, ny, dev):
    """A nx x ny x 2 sheet of 1 mm x 1 mm x 0.5 mm cells (aluminium, Swift
    law, 2 x 2 x 2 points) under a small bending field, held on its two x
    edges: the system, the tangent values and the free DOFs."""
    mat = pkg.material.aluminium_swift()
    m = pkg.structured_hex_mesh(nx, ny, 2, nx * 1e-3, ny * 1e-3, 1e-3)
    x = m.coords
    sysm = pkg.NonlinearSystem(m, mat)
    u = np.zeros_like(x)
    u[:, 2] = -1e-4 * (x[:, 0] / x[:, 0].max()) ** 2
    ev = sysm.evaluate(torch.tensor(u.reshape(-1), device=dev), 0.0, True)
    edge = np.flatnonzero((x[:, 0] == x[:, 0].min()) | (x[:, 0] == x[:, 0].max()))
    held = np.zeros(m.num_dofs, dtype=bool)
    for c in range(3):
        held[3 * edge + c] = True
    return sysm, ev.tangent.clone(), np.flatnonzero(~held).astype(np.int32)


def run_adjoint(args, rank, world):
    """The adjoint springback sensitivity on one GPU: the frozen release of
    an adj_nx x adj_ny x 2 IM Hex8 sheet part carrying the committed history
    of the microbenchmark's loading (Hill48 + Chaboche), J = the RMS vertical
    deviation of its top face from the formed heights, p = the 20 x 20
    bicubic grid of height offsets over the footprint. One step = one
    gradient dJ/dp: the release solve (forward) and the adjoint (backward:
    points re-evaluated at u*, one factorisation, one transposed solve, the
    shape-derivative kernel). Reported: the gradient's cost over one release
    solve, and central differences of J along `directions` seeded random
    directions of p."""
    import torch

    if world > 1 and rank != 0:
        return 0
    pkg = importlib.import_module(PKG)
    wl = importlib.import_module(PKG + ".workload")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nx, ny = args.adj_nx, args.adj_ny
    if args.adj_part == "cone":
        # The fine-mesh part: the truncated cone formed to 35 % of its depth,
        # its committed history from the element kernel; the grid over the
        # cone's footprint.
        csys, cprob = wl.make_cone_problem(args.adj_cone_n, 4, device=dev)
        mesh, material = cprob.mesh, cprob.material
        committed, modes = csys.committed_all(), csys.internal_all()
        csys.close()
        u_np = cprob.u0
        r = wl.CONE["footprint_radius"]
        box = (-r, r, -r, r)
        part_desc = (f"truncated cone (18 mm footprint, 3 mm deep, 50 deg wall) formed to 35 % in a "
                     f"{args.adj_cone_n}x{args.adj_cone_n}x4 IM Hex8 sheet, its imbalance released in 8 increments")
        # Its history is loaded by imposed displacements, far from
        # equilibrium: full Newton steps from it overshoot onto another
        # equilibrium of the supported sheet or invert elements.
        increments = 8
    else:
        prob = wl.make_problem(nx, ny, 2, seed=5, sample=min(4096, nx * ny * 2))
        mesh, material, committed, modes, u_np = prob.mesh, prob.material, prob.state, prob.alpha, prob.u
        lo, hi = mesh.coords.min(axis=0), mesh.coords.max(axis=0)
        box = (lo[0], hi[0], lo[1], hi[1])
        part_desc = (f"{nx}x{ny}x2 IM Hex8 sheet part carrying the microbenchmark's committed Hill48 + Chaboche "
                     f"history")
        increments = 1
    x0 = torch.tensor(mesh.coords, device=dev)
    zmax = mesh.coords[:, 2].max()
    grid = pkg.BicubicHeights(box[0], box[1], box[2], box[3], n=20)
    stencil = grid.stencil(mesh.coords[:, :2], device=dev)
    top = torch.tensor(np.flatnonzero(np.isclose(mesh.coords[:, 2], zmax)), device=dev)
    u_formed = torch.tensor(u_np, device=dev)
    target = x0[top, 2] + u_formed.reshape(-1, 3)[top, 2]
    release = pkg.Release(mesh, material, committed, modes, pkg.supports_321(mesh), increments=increments)

    def coords_of(p):
        lift = torch.zeros_like(x0)
        lift[:, 2] = grid.heights(p, stencil)
        return x0 + lift

    def gradient():
        p = torch.zeros((20, 20), dtype=torch.float64, device=dev, requires_grad=True)
        c = coords_of(p)
        u = pkg.released(c, release, u_formed)
        j = pkg.springback_rms(c, u, top, target)
        j.backward()
        return float(j.detach()), p.grad.detach(), u.detach()

    stream = torch.cuda.current_stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    for w in range(args.warmup):
        t0 = time.perf_counter()
        j, grad, u_star = gradient()
        print(f"adjoint warm-up {w}: {time.perf_counter() - t0:.1f} s, {release.iterations} Newton iterations",
              file=sys.stderr, flush=True)
    # The backward alone: the adjoint at the released state, dJ/du of the RMS.
    c0 = coords_of(torch.zeros((20, 20), dtype=torch.float64, device=dev))
    dj = torch.zeros_like(u_star)
    dj.reshape(-1, 3)[top, 2] = (u_star.reshape(-1, 3)[top, 2] + c0[top, 2] - target) / (len(top) * j)
    lam = torch.tensor(np.random.default_rng(4).standard_normal(mesh.num_dofs), device=dev)
    release_ms, grad_ms, adjoint_ms, adjoint_cold_ms, vjp_ms = [], [], [], [], []
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            release_ms.append(timed(lambda: release.solve(x0, u_formed))[0])
            iterations = release.iterations
            grad_ms.append(timed(gradient)[0])
            adjoint_ms.append(timed(lambda: release.adjoint(c0, u_star, dj))[0])
            release.forget_factorization()
            adjoint_cold_ms.append(timed(lambda: release.adjoint(c0, u_star, dj))[0])
            vjp_ms.append(timed(lambda: release.system.vjp_x(u_star, lam, frozen=True))[0])
    rel_ms, g_ms, a_ms = statistics.median(release_ms), statistics.median(grad_ms), statistics.median(adjoint_ms)
    g = grad.cpu().numpy()
    h = 1e-9
    rng = np.random.default_rng(32)
    errors = []
    t0 = time.perf_counter()
    for _ in range(args.directions):
        d = rng.uniform(-1.0, 1.0, size=(20, 20))
        jd = []
        for sign in (1.0, -1.0):
            c = coords_of(torch.tensor(sign * h * d, device=dev))
            jd.append(float(pkg.springback_rms(c, release.solve(c, u_star, increments=1), top, target)))
        fd = (jd[0] - jd[1]) / (2.0 * h)
        errors.append(abs(float((g * d).sum()) - fd) / abs(fd))
    fd_s = time.perf_counter() - t0
    line = {"metric": "adjoint springback gradient (400 commanded heights): cost relative to one release solve",
            "value": g_ms / rel_ms, "unit": "x", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": g_ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"frozen release of a {part_desc} ({mesh.num_elements} elements, "
                                   f"{len(release.free)} free DOFs), 3-2-1 supports; J = RMS springback of "
                                   "the top face; p = 20x20 bicubic height grid; one step = dJ/dp by "
                                   "torch.autograd (release solve + adjoint)"},
            "release_solve_ms": rel_ms, "newton_iterations": iterations, "gradient_ms": g_ms,
            "adjoint_ms": a_ms, "adjoint_over_release": a_ms / rel_ms, "springback_rms_m": j,
            "adjoint_refactorised_ms": statistics.median(adjoint_cold_ms),
            "per_step_ms": {"release": release_ms, "gradient": grad_ms, "adjoint": adjoint_ms,
                            "adjoint_refactorised": adjoint_cold_ms, "vjp_x": vjp_ms},
            "vjp_x_elements_per_s": mesh.num_elements / (statistics.median(vjp_ms) / 1e3),
            "central_differences": {"directions": args.directions, "h_mm": 1e-6,
                                    "max_relative_difference": max(errors) if errors else None,
                                    "median_relative_difference": statistics.median(errors) if errors else None,
                                    "seconds": fd_s},
            "factor_kind": release.part.kind, "clocks": clocks.summary()}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = (cpu_adjoint(pkg, 16, "cone") if args.adj_part == "cone"
                                else cpu_adjoint(pkg, args.adj_sample))
    print(json.dumps(line))
    release.close()
    return 0


def run_forming(args, rank, world):
    """The CPU-runnable forming run on one GPU, start to finish: the 40 x 40
    x 2 IM sheet (Swift J2, logarithmic strain) clamped in its outer band,
    one 3 mm sphere on the spiral to a 10 mm, 2 mm deep dome in 0.5 mm
    step-downs, then the unload in the clamp and the release onto 3-2-1
    supports (workload.cfg1_deck). The Newton driver around this package's
    element loop, contact and device factorisations is the test harness's
    restatement of the reference's forming driver (tests/forming_harness.py:
    its increment schedule, cuts, contact anticipation and line search). A
    throughput and robustness run: the reference committed no output for
    it. Reported: wall time per step, increments, cuts, the formed and
    released heights."""
    import torch

    if world > 1 and rank != 0:
        return 0
    pkg = importlib.import_module(PKG)
    wl = importlib.import_module(PKG + ".workload")
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests"))
    from forming_harness import FormingRun

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    deck = wl.cfg1_deck()
    times = deck["tools"][0]["trajectory"]["times"]
    if args.forming_stations > 0:
        # The form step cut short after that many points of the path (then
        # the unload and the release as usual).
        deck["steps"][0]["deck"]["time"][1] = min(deck["steps"][0]["deck"]["time"][1],
                                                  times[min(args.forming_stations, len(times) - 1)])
    # The increments grow back after a cut as the reference's driver lets
    # them: by the iterations to its own tolerance.
    run = FormingRun(pkg, deck, dev, growth_test="reference", tolerance="reference")
    top = np.flatnonzero(np.isclose(run.nodes[:, 2], run.nodes[:, 2].max()))
    steps = []
    with ClockSampler(0) as clocks:
        for k, st in enumerate(deck["steps"]):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = run.run_step(k, None)
            torch.cuda.synchronize()
            z = run.nodes[top, 2] + res.u.reshape(-1, 3)[top, 2]
            steps.append({"name": st["deck"]["name"], "seconds": time.perf_counter() - t0,
                          "increments": res.increments, "cuts": res.cuts, "pole_height_m": float(z.min()),
                          "max_eq_plastic_strain": float(res.eq_plastic_strain.max()),
                          "max_tool_force_n": float(max((abs(f) for f in res.tool_fz), default=0.0))})
            print(json.dumps(steps[-1]), file=sys.stderr, flush=True)
    total = sum(s["seconds"] for s in steps)
    form = steps[0]
    line = {"metric": "CPU-runnable forming run: wall time on one GPU", "value": total, "unit": "s", "n_gpus": 1,
            "steps": 1, "warmup": 0, "ms_per_step": total * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "20x20x1 mm sheet, 40x40x2 IM Hex8, outer 1 mm clamped; J2 + Swift (E 70 GPa, "
                                   "nu 0.33, K 425 MPa, eps0 0.003, n 0.29) through from_swift; sphere R 3 mm, "
                                   "penalty 10, mu 0.1, spiral to a 10 mm x 2 mm dome in 0.5 mm step-downs; "
                                   "unload; 3-2-1 release; logarithmic strain"},
            "per_step": steps, "tool_path_points": len(deck["tools"][0]["trajectory"]["points"]),
            "form_end_time": deck["steps"][0]["deck"]["time"][1],
            "form_seconds_per_increment": form["seconds"] / max(form["increments"], 1), "clocks": clocks.summary()}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = forming_cpu_baseline(pkg, wl, FormingRun)
    print(json.dumps(line), flush=True)
    return 0


def forming_cpu_baseline(pkg, wl, FormingRun, stations=5):
    """The same deck's first `stations` path points through the same
    harness on the host cores, the oracle's system and contact in place of
    the package's and scipy's solves: seconds per converged increment."""
    from oracle_backend import OracleBackend

    orc = oracle_module()
    orc.use_variant("fast")
    deck = wl.cfg1_deck()
    deck["steps"][0]["deck"]["time"][1] = deck["tools"][0]["trajectory"]["times"][stations]
    run = FormingRun(OracleBackend(pkg, orc), deck, "cpu", solver="host", growth_test="reference",
                     tolerance="reference")
    t0 = time.perf_counter()
    res = run.run_step(0, None)
    seconds = time.perf_counter() - t0
    return {"value": seconds / max(res.increments, 1), "unit": "s per increment", "cores": cpu_count(),
            "kind": "port", "sample": f"the form step to the path's point {stations} ({res.increments} increments, "
                                      f"{res.cuts} cuts), the oracle through the harness, scipy's solves",
            "seconds": seconds}


def cpu_adjoint(pkg, n, part="sheet"):
    """The same release and gradient with the oracle on the host cores (the
    oracle's release Newton with scipy's sparse LU, its adjoint with the
    transposed block and its per-element shape derivative) on an n x n x 2
    sample part whose history the oracle loads, or an n x n x 4 cone part of
    the fine-mesh construction (released in 8 increments, as on the GPU)."""
    orc = oracle_module()
    if part == "cone":
        wl = importlib.import_module(PKG + ".workload")
        mesh, mat, committed, alpha, _ = cone_sample(orc, n)
        u0 = (wl.formed_positions(mesh, wl.cone_part(), 0.35) - mesh.coords).reshape(-1)
        increments, desc = 8, f"{n}x{n}x4 cone part ({mesh.num_elements} elements) released in 8 increments"
    else:
        prob, committed = oracle_problem(orc, n, n, 2, 5)
        mesh, mat, alpha, u0 = prob.mesh, prob.material, prob.alpha, prob.u
        increments, desc = 1, f"{n}x{n}x2 part ({mesh.num_elements} elements)"
    m = mat.as_dict()
    m["yield_stress"] = 1e300  # frozen
    free = pkg.supports_321(mesh)
    top = np.flatnonzero(np.isclose(mesh.coords[:, 2], mesh.coords[:, 2].max()))
    t0 = time.perf_counter()
    u, iterations = orc.release_solve(m, mesh.coords, mesh.connectivity, committed, alpha, free, u0,
                                      increments=increments)
    release_s = time.perf_counter() - t0
    d = u.reshape(-1, 3)[top, 2] - u0.reshape(-1, 3)[top, 2]
    j = float(np.sqrt(np.mean(d * d)))
    dj = np.zeros(mesh.num_dofs)
    dj[3 * top + 2] = d / (len(top) * j)
    t0 = time.perf_counter()
    orc.release_adjoint(m, mesh.coords, mesh.connectivity, committed, alpha, free, u, dj)
    adjoint_s = time.perf_counter() - t0
    return {"value": (release_s + adjoint_s) / release_s, "unit": "x", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{desc}, the oracle's history, one release and one gradient",
            "release_solve_ms": release_s * 1e3, "newton_iterations": iterations, "adjoint_ms": adjoint_s * 1e3}


def run_cone(args, rank, world):
    """The fine-mesh part: the truncated cone (18 mm footprint, 3 mm deep, 50
    degree wall) in a 1 mm sheet of cone_n x cone_n x 4 IM Hex8 (224 x 224 x
    4 = 200,704 elements by default), Hill48 + Chaboche, formed to 35 % of
    its depth in committed increments, with the two tools of double-sided
    forming on its wall. One step = one Newton iteration's device work:
    NonlinearSystem.evaluate with the tangent, ToolContact.evaluate of both
    tools with their blocks, and the blocks added into the tangent. Beside
    it: the contact's share (K3), the candidate search of an increment by
    the uniform-grid hash and by the flat scan, the candidate and active
    counts."""
    import torch

    if world > 1 and rank != 0:
        return 0
    pkg = importlib.import_module(PKG)
    wl = importlib.import_module(PKG + ".workload")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cpu = None
    if not args.no_cpu_baseline:
        cpu = cone_cpu_baseline(args)
    peaks = measured_peaks()
    fp64_peak = fp64_peak_tflops(torch, dev)
    t_setup = time.perf_counter()
    sysm, prob = wl.make_cone_problem(args.cone_n, 4, device=dev)
    mesh = prob.mesh
    ne = mesh.num_elements
    contact = pkg.ToolContact(mesh, [pkg.Tool(**t) for t in prob.tools], friction_tangent="exact")
    u0 = torch.tensor(prob.u0, device=dev)
    u = torch.tensor(prob.u, device=dev)
    margin = 2.0e-3 + float(np.abs(prob.u - prob.u0).max()) + float(np.sqrt(prob.tools[0]["area"].min()))
    contact.begin_increment(u0, 0.0, 1.0, [True, True], margin)
    sysm.set_timing(True)
    setup_s = time.perf_counter() - t_setup
    stream = torch.cuda.current_stream()

    def step():
        ev = sysm.evaluate(u, 0.0, True)
        cev = contact.evaluate(u, 1.0, True)
        sysm.add_node_blocks(cev.nodes, cev.blocks)
        return ev, cev

    for _ in range(args.warmup):
        ev, cev = step()
    torch.cuda.synchronize()
    elem_ms, k3_ms = [], []
    with ClockSampler(0) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("timed_steps")
        e0.record(stream)
        for _ in range(args.steps):
            ev = sysm.evaluate(u, 0.0, True)
            elem_ms.append(sysm.last_timings()["element"])
            c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            c0.record(stream)
            cev = contact.evaluate(u, 1.0, True)
            c1.record(stream)
            sysm.add_node_blocks(cev.nodes, cev.blocks)
            c1.synchronize()
            k3_ms.append(c0.elapsed_time(c1))
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = e0.elapsed_time(e1) / args.steps

    def begin_ms(mode, reps=10):
        contact.set_search(mode)
        contact.begin_increment(u0, 0.0, 1.0, [True, True], margin)
        torch.cuda.synchronize()
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for _ in range(reps):
            contact.begin_increment(u0, 0.0, 1.0, [True, True], margin)
        b1.record(stream)
        torch.cuda.synchronize()
        return b0.elapsed_time(b1) / reps, [contact.candidates(k) for k in range(2)]

    grid_ms, grid_cand = begin_ms("grid")
    scan_ms, scan_cand = begin_ms("scan")
    assert grid_cand == scan_cand, (grid_cand, scan_cand)
    contact.set_search("grid")
    # End to end through the public calls with host buffers (the tangent
    # double-buffered, read back on a copy stream while the next step runs).
    u_host = u.cpu().pin_memory()
    f_host = torch.empty(sysm.num_dofs, dtype=torch.float64).pin_memory()
    v_host = [torch.empty(sysm.nnz, dtype=torch.float64).pin_memory() for _ in range(2)]
    v_dev = [torch.empty(sysm.nnz, dtype=torch.float64, device=dev) for _ in range(2)]
    copied = [torch.cuda.Event() for _ in range(2)]
    copy_stream = torch.cuda.Stream(device=dev)
    u_dev = torch.empty_like(u)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s0.record(stream)
    for k in range(args.steps):
        b = k % 2
        stream.wait_event(copied[b])
        u_dev.copy_(u_host, non_blocking=True)
        sysm.set_values_buffer(v_dev[b])
        ev = sysm.evaluate(u_dev, 0.0, True)
        cev = contact.evaluate(u_dev, 1.0, True)
        sysm.add_node_blocks(cev.nodes, cev.blocks)
        f_host.copy_(ev.internal, non_blocking=True)
        copy_stream.wait_stream(stream)
        with torch.cuda.stream(copy_stream):
            v_host[b].copy_(v_dev[b], non_blocking=True)
            copied[b].record(copy_stream)
    stream.wait_stream(copy_stream)
    s1.record(stream)
    torch.cuda.synchronize()
    sysm.set_values_buffer(None)
    e2e_ms = s0.elapsed_time(s1) / args.steps
    el_ms = statistics.mean(elem_ms)
    flops = None
    if not args.no_cpu_baseline:
        flops = cone_flops_per_element(args)
    roofline = None
    if flops:
        achieved = flops * ne / (el_ms / 1e3) / 1e12
        roofline = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp64_peak, "traffic": None, "kernel": "K1 (phase kernels)",
                    "kernel_ms": el_ms, "flops_per_element": flops,
                    "peak_source": "measured in this run: cuBLAS FP64 GEMM 8192^3 burst"}
    line = {"metric": METRIC + " with two-tool contact", "value": ne / (ms / 1e3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"fine-mesh part: truncated cone (18 mm footprint, 3 mm deep, 50 deg wall) in a "
                                   f"1 mm sheet of {args.cone_n}x{args.cone_n}x4 IM Hex8 ({ne} elements), Hill48 + "
                                   "Chaboche, formed to 35% of its depth; forming and support balls (R 2 mm) on the "
                                   "wall; one step = evaluate with tangent + both tools' contact + their blocks",
                       "l2": "inputs larger than L2"},
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": ne / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 8 * sysm.num_dofs,
                    "d2h_bytes_per_step": 8 * (sysm.num_dofs + sysm.nnz), "ms_per_step": e2e_ms},
            "phases_ms": {"element": el_ms, "contact_evaluate": statistics.mean(k3_ms)},
            "contact": {"begin_grid_ms": grid_ms, "begin_scan_ms": scan_ms, "candidates": grid_cand,
                        "active": [int(cev.tools[k][6]) for k in range(2)],
                        "slaves": [int(len(t["nodes"])) for t in prob.tools], "margin_m": margin},
            # K1's phase kernels (26 rounds of 5, the condensation, the
            # single kernel's list), K2b + finish, K2a; per tool 7 contact
            # kernels (moved points, evaluate, the ordered compaction's 3,
            # scatter, resultants), the norms' two stages over both tools,
            # and the blocks' add.
            "gpu_launches": args.steps * ((26 * 5 + 2) + 3 + 2 * 7 + 2 + 1), "clocks": clocks.summary(),
            "yielding_fraction": ev.yielding_points / (8.0 * ne),
            "setup_s": setup_s}
    print(json.dumps(line), flush=True)
    contact.close()
    return 0


def cone_sample(orc, n):
    """A small cone part of the same construction on the CPU (the oracle's
    element routines load its history)."""
    wl = importlib.import_module(PKG + ".workload")
    mesh = wl.cone_sheet(n, 4)
    mat = importlib.import_module(PKG + ".material").hill_chaboche_sheet()
    cone = wl.cone_part()
    steps, s = 7, 0.35
    committed = np.zeros((mesh.num_elements, 8, orc.NF))
    alpha = np.zeros((mesh.num_elements, 9))
    X = mesh.element_coordinates()
    for k in range(1, steps + 1):
        uk = (wl.formed_positions(mesh, cone, k * s / steps) - mesh.coords).reshape(-1)
        r = orc.elements(mat.as_dict(), X, mesh.gather(uk), committed, alpha, want_tangent=False)
        ok = r["status"] == 0
        committed = np.where(ok[:, None, None], r["states"], committed)
        alpha = np.where(ok[:, None], r["alpha"], alpha)
    u = (wl.formed_positions(mesh, cone, s + 0.25 * s / steps) - mesh.coords).reshape(-1)
    return mesh, mat, committed, alpha, u


def cone_cpu_baseline(args):
    """The oracle (-O3 -march=native, all host threads) on a cone_sample_n x
    cone_sample_n x 4 part of the same construction: elements / s of its
    NonlinearSystem::evaluate with the tangent."""
    orc = oracle_module()
    orc.use_variant("fast")
    try:
        mesh, mat, committed, alpha, u = cone_sample(orc, args.cone_sample_n)
        cores = cpu_count()
        pat = orc.pattern(mesh.num_nodes, mesh.connectivity)
        orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, u, committed, alpha, threads=cores,
                            pat=pat)
        times = []
        for _ in range(3):
            t0 = time.perf_counter()
            r = orc.system_evaluate(mat.as_dict(), mesh.coords, mesh.connectivity, u, committed, alpha, threads=cores,
                                    pat=pat)
            times.append(time.perf_counter() - t0)
        value = mesh.num_elements / statistics.median(times)
        return {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "build": orc.FAST_FLAGS,
                "sample": f"{mesh.num_elements} elements ({args.cone_sample_n}x{args.cone_sample_n}x4 cone part of the "
                          f"same construction), median of 3 evaluations with the tangent (code {r['code']})"}
    finally:
        orc.use_variant("strict")


def cone_flops_per_element(args):
    orc = oracle_module()
    mesh, mat, committed, alpha, u = cone_sample(orc, min(args.cone_sample_n, 24))
    cnt = orc.count_flops(mat.as_dict(), mesh.element_coordinates(), mesh.gather(u), committed, alpha)
    return cnt / mesh.num_elements


def run_partition(args, rank, world):
    """The free-free block of a Dirichlet partition (PartitionedFactor,
    Forming.cpp:59-241): one step = the gather of the block's values from
    the full tangent (assemble), the kernel the roofline covers; beside it
    the factorisation (sparse Cholesky) and solve the block feeds, and the
    CPU: the oracle's restatement of the gather and scipy's SuperLU (the
    reference's CHOLMOD / UMFPACK are not in this image) on a bounded
    sample."""
    import torch

    if world > 1 and rank != 0:
        return 0
    pkg = importlib.import_module(PKG)
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    peaks = measured_peaks()
    nx, ny = args.part_nx, args.part_ny
    sysm, values, free = sheet_partition(pkg, torch, nx, ny, dev)
    t0 = time.perf_counter()
    part = pkg.PartitionedFactor.for_system(sysm, free)
    torch.cuda.synchronize()
    create_ms = (time.perf_counter() - t0) * 1e3
    kff = torch.empty(part.nnz, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        part.assemble(values, kff)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            part.assemble(values, kff)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    entries = part.nnz
    alg_bytes = entries * (8 + 4 + 8)  # value read, source index read, block value written
    achieved = alg_bytes / (ms / 1e3) / 1e9
    # Through the public call with host buffers: the full tangent copied in
    # from pinned memory, the block's values copied back, every step.
    host_vals = values.cpu().pin_memory()
    host_kff = torch.empty(entries, dtype=torch.float64).pin_memory()
    dev_vals = torch.empty_like(values)
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        dev_vals.copy_(host_vals, non_blocking=True)
        part.assemble(dev_vals, kff)
        host_kff.copy_(kff, non_blocking=True)
    e3.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e2.elapsed_time(e3) / args.steps
    # The factorisation the block feeds.
    part.factorize(values, True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        part.factorize(values, True)
    torch.cuda.synchronize()
    factor_ms = (time.perf_counter() - t0) / 3 * 1e3
    b = torch.ones(part.num_free, dtype=torch.float64, device=dev)
    part.solve(b)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        part.solve(b)
    torch.cuda.synchronize()
    solve_ms = (time.perf_counter() - t0) / 3 * 1e3
    line = {"metric": "free-free block entries gathered/s (FP64)", "value": entries / (ms / 1e3),
            "unit": "entries/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"free-free block of a {nx}x{ny}x2 IM Hex8 sheet held on its x edges "
                                   f"({part.num_free} free DOFs, {entries} block entries of "
                                   f"{sysm.nnz}); one step = PartitionedFactor.assemble",
                       "l2": "inputs larger than L2 (full values, source map and block values "
                             f"{alg_bytes / 1e6:.0f} MB per step)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                         "frac": achieved / peaks.get("hbm_gbs", 6650.0),
                         "traffic": GATHER_DRAM_BYTES_PER_ENTRY * entries,
                         "peak_source": peaks.get("source", "MEASURED_PEAKS.json")},
            "e2e": {"value": entries / (e2e_ms / 1e3), "unit": "entries/s", "h2d_bytes_per_step": values.numel() * 8,
                    "d2h_bytes_per_step": entries * 8},
            "gpu_launches": args.steps, "clocks": clocks.summary(),
            "create_ms": create_ms, "cholesky_factor_ms": factor_ms, "cholesky_solve_ms": solve_ms,
            "counts": part.counts()}
    if not args.no_cpu_baseline:
        orc = oracle_module()
        snx, sny = args.sample_nx, args.sample_ny
        ssys, svals, sfree = sheet_partition(pkg, torch, snx, sny, dev)
        pat = {"outer": ssys.outer.cpu().numpy(), "inner": ssys.inner.cpu().numpy()}
        v = svals.cpu().numpy()
        t0 = time.perf_counter()
        _, _, src, sk = orc.free_free_block(pat, v, sfree)
        cpu_s = time.perf_counter() - t0
        import scipy.sparse as sp
        import scipy.sparse.linalg as spl
        n = ssys.num_dofs
        K = sp.csc_matrix((v, pat["inner"], pat["outer"]), shape=(n, n))[sfree][:, sfree].tocsc()
        t0 = time.perf_counter()
        spl.splu(K).solve(np.ones(len(sfree)))
        lu_s = time.perf_counter() - t0
        spart = pkg.PartitionedFactor.for_system(ssys, sfree)
        spart.factorize(svals, True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        spart.factorize(svals, True)
        spart.solve(torch.ones(len(sfree), dtype=torch.float64, device=dev))
        torch.cuda.synchronize()
        gpu_fs = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": len(sk) / cpu_s, "unit": "entries/s", "cores": 1, "kind": "port",
                                "sample": f"the oracle's gather of the {snx}x{sny}x2 sheet's block ({len(sk)} "
                                          f"entries)",
                                "superlu_factor_solve_ms": lu_s * 1e3, "gpu_cholesky_factor_solve_ms": gpu_fs * 1e3,
                                "superlu_sample": f"{snx}x{sny}x2 sheet, {len(sfree)} free DOFs"}
    print(json.dumps(line), flush=True)
    return 0


def config(args, world):
    element = "IM Hex8" if args.element == "incompatible_modes" else "standard Hex8 (B-bar)"
    return {"workload": f"element-kernel microbenchmark: {args.nx}x{args.ny}x{args.nz} {element} sheet "
                        f"(0.04x0.04x0.5 mm cells), 2x2x2 points, Hill48 r=(0.73,0.80,0.70) + Chaboche "
                        f"(8000 MPa/200, 1200 MPa/20) + Voce, logarithmic strain, ~40% of points yielding; "
                        f"one step = NonlinearSystem.evaluate with tangent",
            "elements_per_rank": args.nx * args.ny * args.nz, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (1.7 GB committed state, 4.6 GB element tangents, 2.3 GB CSC values "
                  "per rank)"}


def main():
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nx", type=int, default=1000)
    p.add_argument("--ny", type=int, default=500)
    p.add_argument("--nz", type=int, default=2)
    p.add_argument("--sample-nx", type=int, default=50)
    p.add_argument("--sample-ny", type=int, default=40)
    p.add_argument("--ref-nx", type=int, default=160, help="the CPU baseline's all-core sample: ref-nx x ref-ny x nz")
    p.add_argument("--ref-ny", type=int, default=160)
    p.add_argument("--cpu-steps", type=int, default=5, help="timed steps of the in-run CPU baseline")
    p.add_argument("--epb", type=int, default=0, help="elements per block of the element kernel (0: default)")
    p.add_argument("--local-iteration", default="phases", choices=["phases", "single"],
                   help="the local iteration as phase kernels over the mesh (default) or one kernel per element")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--cone-n", type=int, default=224)
    p.add_argument("--cone-sample-n", type=int, default=48)
    p.add_argument("--workload", default="microbench",
                   choices=["microbench", "batched", "partition", "adjoint", "cone", "forming"],
                   help="batched: the design-sweep batch (64 parts of 20k-150k elements) in one launch against the "
                        "same parts evaluated one at a time; partition: the free-free block of a Dirichlet "
                        "partition gathered from the full tangent, and the factorisation it feeds; adjoint: the "
                        "springback gradient with respect to 400 commanded heights against one release solve and "
                        "central differences; cone: the fine-mesh truncated cone (200k elements) with the two tools "
                        "of double-sided forming; forming: the CPU-runnable forming run (a 40x40x2 sheet, a spiral "
                        "to a dome, unload, release) start to finish")
    p.add_argument("--element", default="incompatible_modes", choices=["incompatible_modes", "standard"],
                   help="standard: the standard Hex8 with mean dilatation on the same sheet and history")
    p.add_argument("--part-nx", type=int, default=200)
    p.add_argument("--part-ny", type=int, default=200)
    p.add_argument("--parts", type=int, default=64)
    p.add_argument("--sweep-increments", type=int, default=4)
    p.add_argument("--adj-nx", type=int, default=100)
    p.add_argument("--adj-ny", type=int, default=100)
    p.add_argument("--directions", type=int, default=32)
    p.add_argument("--adj-sample", type=int, default=40)
    p.add_argument("--forming-stations", type=int, default=0,
                   help="forming: end the form step at this point of the tool path (0: the whole path)")
    p.add_argument("--adj-part", default="sheet", choices=["sheet", "cone"],
                   help="the part of the adjoint workload: a flat sheet with the microbenchmark's history, or the "
                        "fine-mesh cone")
    p.add_argument("--adj-cone-n", type=int, default=32,
                   help="the adjoint's cone part: adj-cone-n x adj-cone-n x 4. Each release is ~43 Newton "
                        "iterations, each a factorisation of its free-free block: ~0.24 s at 32 (16,329 DOFs), "
                        "~14 s at 64 (63k DOFs)")
    args = p.parse_args()
    args.warmup = max(args.warmup, 3)

    replicas = importlib.import_module(PKG + ".replicas")
    rank, world, local = replicas.rank_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "batched":
        return run_batched(args, rank, world)
    if args.workload == "partition":
        return run_partition(args, rank, world)
    if args.workload == "adjoint":
        return run_adjoint(args, rank, world)
    if args.workload == "cone":
        return run_cone(args, rank, world)
    if args.workload == "forming":
        return run_forming(args, rank, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_subprocess(args)

    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    replicas.init(world, "nccl", dev)

    wl = importlib.import_module(PKG + ".workload")
    peaks = measured_peaks()
    fp64_peak = fp64_peak_tflops(torch, dev)

    t_setup = time.perf_counter()
    sysm, u, s, mesh = wl.make_system_problem(args.nx, args.ny, args.nz, seed=replicas.replica_seed(7, rank),
                                              device=dev)
    ne = mesh.num_elements
    if args.element == "standard":
        # The standard Hex8 from the same committed history.
        sysm.set_element("standard", "auto")
    if args.epb:
        sysm.set_elements_per_block(args.epb)
    sysm.set_local_iteration(args.local_iteration)
    sysm.set_timing(True)
    setup_s = time.perf_counter() - t_setup

    def barrier():
        replicas.barrier(world)

    for _ in range(args.warmup):
        ev = sysm.evaluate(u, 0.0, True)
    yielding = ev.yielding_points
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    elem_ms, force_ms, value_ms = [], [], []
    with ClockSampler(local) as clocks:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        # The NVTX range names the timed launches for a profiler's filter.
        torch.cuda.nvtx.range_push("timed_steps")
        start.record(stream)
        for _ in range(args.steps):
            ev = sysm.evaluate(u, 0.0, True)
            t = sysm.last_timings()
            elem_ms.append(t["element"])
            force_ms.append(t["forces"])
            value_ms.append(t["values"])
        end.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    barrier()
    torch.cuda.synchronize()
    ms = replicas.max_over_ranks(start.elapsed_time(end) / args.steps, world, dev)
    value = replicas.job_rate(ne, world, ms / 1e3)

    # End to end through the C ABI with host buffers: every step u copied in
    # from pinned memory, f_int and the 2.3 GB of tangent values read back.
    # The tangent alternates between two device buffers
    # (sbk_system_set_values_buffer), so that one step's values travel to
    # the host on a copy stream while the next step evaluates.
    e2e = None
    if not args.no_e2e:
        u_host = u.cpu().pin_memory()
        f_host = torch.empty(sysm.num_dofs, dtype=torch.float64).pin_memory()
        v_host = [torch.empty(sysm.nnz, dtype=torch.float64).pin_memory() for _ in range(2)]
        v_dev = [torch.empty(sysm.nnz, dtype=torch.float64, device=dev) for _ in range(2)]
        copied = [torch.cuda.Event() for _ in range(2)]
        copy_stream = torch.cuda.Stream(device=dev)
        u_dev = torch.empty_like(u)
        barrier()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for k in range(args.steps):
            b = k % 2
            stream.wait_event(copied[b])  # the buffer's last read-back has finished
            u_dev.copy_(u_host, non_blocking=True)
            sysm.set_values_buffer(v_dev[b])
            ev = sysm.evaluate(u_dev, 0.0, True)
            f_host.copy_(ev.internal, non_blocking=True)
            copy_stream.wait_stream(stream)
            with torch.cuda.stream(copy_stream):
                v_host[b].copy_(v_dev[b], non_blocking=True)
                copied[b].record(copy_stream)
        stream.wait_stream(copy_stream)
        s1.record(stream)
        torch.cuda.synchronize()
        sysm.set_values_buffer(None)
        barrier()
        e_ms = replicas.max_over_ranks(s0.elapsed_time(s1) / args.steps, world, dev)
        e2e = {"value": replicas.job_rate(ne, world, e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 8 * sysm.num_dofs,
               "d2h_bytes_per_step": 8 * (sysm.num_dofs + sysm.nnz), "ms_per_step": e_ms,
               "overlap": "tangent values read back on a copy stream while the next step evaluates"}

    line = None
    if rank == 0:
        flops_per_element = None
        if world == 1 and not args.no_cpu_baseline:
            orc = oracle_module()
            prob, committed = oracle_problem(orc, args.sample_nx, args.sample_ny, args.nz, seed=7)
            std = orc.element(args.element == "standard", True)
            # Algorithmic flops per element (counting scalar) on a sample.
            with std:
                cnt = orc.count_flops(prob.material.as_dict(), prob.mesh.element_coordinates(),
                                      prob.mesh.gather(prob.u), committed, prob.alpha)
            flops_per_element = cnt / prob.mesh.num_elements
        el_ms = statistics.mean(elem_ms)
        # Kernels of one step: K1 (the phase kernels: 26 rounds of 5 launches,
        # the condensation, the single kernel for the elements it takes; or
        # one launch), then the force gather and its finish (2), the value
        # gather, and for the single kernel the schedule (count, CUB's scan,
        # place).
        phases = args.element == "incompatible_modes" and args.local_iteration == "phases"
        launches_per_step = (26 * 5 + 2 if phases else 1 + 3) + 3
        k1_name = ("K1: the local iteration as phase kernels (wave_pre / wave_return / wave_log / wave_post / "
                   "wave_control x 26 rounds, wave_condense, element_list)" if phases else
                   "element_kernel (K1)" if args.element == "incompatible_modes" else "standard_kernel (K1s)")
        roofline = None
        if flops_per_element:
            achieved = flops_per_element * ne / (el_ms / 1e3) / 1e12
            roofline = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                        "frac": achieved / fp64_peak,
                        "traffic": (K1S_DRAM_BYTES_PER_ELEMENT if args.element != "incompatible_modes"
                                    else K1_DRAM_BYTES_PER_ELEMENT if phases
                                    else K1_SINGLE_DRAM_BYTES_PER_ELEMENT) * ne,
                        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of K1's launches in "
                                          "one evaluation of the 200x200x2 sheet (80,000 elements), scaled by "
                                          "elements",
                        "kernel": k1_name, "kernel_ms": el_ms,
                        "flops_per_element": flops_per_element,
                        "peak_source": "measured in this run: cuBLAS FP64 GEMM 8192^3 burst (FP64 has no entry in "
                                       "MEASURED_PEAKS.json)"}
        # Assembly (K2) is bandwidth bound: its algorithmic bytes per step.
        nnz = sysm.nnz
        asm_bytes = ne * 576 * 8 + nnz * 8 + ne * 64 * 4 + (nnz // 9) * (4 + 8 + 4 + 4)
        asm_ms = statistics.mean(value_ms)
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config(args, world),
                "roofline": roofline,
                "roofline_assembly": {"bound": "hbm", "achieved": asm_bytes / (asm_ms / 1e3) / 1e9,
                                      "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                                      "frac": asm_bytes / (asm_ms / 1e3) / 1e9 / peaks.get("hbm_gbs", 6650.0),
                                      "kernel": "assemble_values (K2)", "kernel_ms": asm_ms,
                                      "traffic": None},
                "phases_ms": {"element": el_ms, "forces": statistics.mean(force_ms), "values": asm_ms},
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches_per_step * args.steps,
                "clocks": clocks.summary(), "yielding_fraction": yielding / (8.0 * ne), "increment_s": s,
                "setup_s": setup_s}
        print(json.dumps(line), flush=True)
    replicas.finish(world)
    return 0


if __name__ == "__main__":
    sys.exit(main())
