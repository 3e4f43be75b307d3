#!/usr/bin/env python
"""Benchmark: Yee/CPML time-step throughput (Mcell/s) and HBM-roofline fraction on B200.

Workload (the bandwidth-roofline configuration): 512³ FP32 grid, dl = 1 mm,
npml = 16, εr ~ U[1, 12] per 8³-cell block (seeded), a Jx point source at the
centre driven by a Gaussian pulse, and one z-plane DFT monitor of Ex at 4
frequencies, fused into the step.  A "step" is one full leapfrog update of that
grid.  Inputs are ~9 GB per step, far larger than the 126 MB L2, so no L2 flush
is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

For N > 1 the script runs under torchrun with one rank per GPU; each rank runs an
independent replica of the workload (the path is one grid per GPU here), timing
is the max over ranks, and ``value`` is the total cell updates of all ranks per
second ("scaling": "weak").

The line also carries ``n2f``: the near-to-far contraction of a 320³ box
(614,400 face samples x 4 currents x 32 frequencies, complex64) onto 361 x 181
directions in split-BF16 and TF32 on the tensor cores, timed by CUDA events, with
its error against the float64 direct sum on every 64th direction.
``fp64`` is the same construction at 384³ in FP64 mode (the FP64 throughput
figure, 136 B/cell of algorithmic traffic).  It also carries ``adjoint``: the ε-gradient leg at 160×160×96 FP32 (npml 12,
96×96×16 design box, Jx sheet at 30 GHz, 3000 steps, checkpoints every 100 steps,
objective Σ|Ex(30 GHz)|² over a 32×32 patch): ``t_grad / t_forward`` by CUDA events,
and the gradient against central differences (h = 1e-3) at 16 seeded voxels in FP64.

``--impl reference`` times the reference's own Yee/source kernels
(``opencl_fdtd_solver/kernels/yee_update.cl``, ``sources.cl``) compiled as C with
OpenMP on all host cores (``oracle/_ref``; the C restatement in ``oracle/`` when
that library is absent), on a bounded number of steps of the same grid.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FREQS = (20e9, 25e9, 30e9, 35e9)
METRIC = "Mcell/s (Yee+CPML step, 512^3 FP32, % of HBM roofline)"
FALLBACK_HBM_GBS = 6650.0


def alg_bytes_per_cell(shape, npml, item=4, dft_planes=((2, 1, 4),)):
    """Algorithmic bytes per cell-step: 6 fields read+write, 3 ce reads, ψ on the
    stripes (4 arrays per axis, read+write), plane DFT accumulators (complex128
    read+write per plane cell, component and frequency)."""
    nx, ny, nz = shape
    cells = nx * ny * nz
    b = 15 * item
    if npml > 0:
        frac = sum(min(2 * npml, n) / n for n in shape)
        b += frac * 4 * 2 * item
    for axis, ncomp, nfreq in dft_planes:
        plane_cells = cells // shape[axis]
        b += plane_cells * ncomp * nfreq * 32 / cells
    return b


def measured_hbm():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def blocky_eps(shape, block=8, lo=1.0, hi=12.0, seed=1234):
    rng = np.random.default_rng(seed)
    nb = [-(-n // block) for n in shape]
    vals = rng.uniform(lo, hi, nb).astype(np.float32)
    e = np.repeat(np.repeat(np.repeat(vals, block, 0), block, 1), block, 2)
    return np.ascontiguousarray(e[: shape[0], : shape[1], : shape[2]])


def gaussian_pulse(t, fwidth=20e9):
    t0 = 5.0 / (np.pi * fwidth)
    sigma = 1.0 / (np.pi * fwidth)
    return float(np.exp(-0.5 * ((t - t0) / sigma) ** 2))


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus, backend="nccl"):
    """One process per GPU (torchrun's RANK/LOCAL_RANK/WORLD_SIZE); the only
    collectives are a barrier and a max-reduction of the device time."""
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def reduce_max(x, world):
    """Max of x over the ranks (the job's time is its slowest replica's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, cells, steps, max_ms):
    """Whole-job Mcell/s of `world` replicas that each advanced `cells` cells
    `steps` steps, timed by the slowest replica."""
    return world * cells * steps / (max_ms / 1e3) / 1e6


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def make_engine(size, npml, dtype, fused=True):
    from opencl_fdtd_solver_b200 import CUDAFDTD, CUDAPlaneDFTMonitor

    shape = (size, size, size)
    g = CUDAFDTD(shape, 1e-3, npml=npml, dtype=dtype, fused=fused)
    c = size // 2
    g.add_source(lambda f: f.add_source_Jx(c, gaussian_pulse(f.t), i0=c, i1=c + 1, j0=c, j1=c + 1))
    mon = CUDAPlaneDFTMonitor(g, "z", c, FREQS, ("Ex",))
    return g, mon


def cpu_engine(size, npml, dtype, backend):
    """The same grid and step on the CPU (reference kernels compiled as C, or the
    oracle port), with the same z-plane DFT of Ex at 4 frequencies (the oracle's
    plane-DFT monitor: the reference has no plane-DFT kernel)."""
    from oracle.cpu_fdtd import OracleFDTD
    from oracle.dft_oracle import OraclePlaneDFTMonitor

    shape = (size, size, size)
    o = OracleFDTD(shape, 1e-3, npml=npml, dtype=dtype, backend=backend)
    o.set_epsilon(blocky_eps(shape))
    c = size // 2
    o.add_source(lambda f: f.add_source_Jx(c, gaussian_pulse(f.t), i0=c, i1=c + 1, j0=c, j1=c + 1))
    o._bench_dft = OraclePlaneDFTMonitor(o, "z", c, FREQS, ("Ex",))
    return o


def cpu_reference_rate(size, npml, dtype, seconds, backend):
    """Mcell/s of the CPU Yee step over ~``seconds`` of steps after one warm-up step."""
    from oracle.cpu_fdtd import num_threads

    o = cpu_engine(size, npml, dtype, backend)
    o.step()  # warm-up (page-in)
    n, t0 = 0, time.perf_counter()
    while True:
        o.step()
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 50:
            break
    return size**3 * n / el / 1e6, n, el, num_threads()


def workload_config(size, npml, world):
    """The workload both arms time (identical dicts, so the two lines compare)."""
    return {"workload": f"yee_cpml_{size}^3_fp32_npml{npml}_blocky_eps_jx_point_zdft4",
            "grid": [size] * 3, "npml": npml, "plane_dft_freqs_hz": list(FREQS),
            "eps_seed": 1234, "l2": "inputs (~9 GB/step) exceed L2; no flush",
            "parallelism": f"replicas{world}"}


def run_reference_arm(args, rank, world):
    """Each timed step is one Yee step of the grid on all host cores; warm-up and timed
    steps stop early once ``--cpu-budget`` seconds are spent, so the run stays bounded."""
    if rank != 0:
        return None
    from oracle.cpu_fdtd import num_threads, ref_available

    backend = "ref" if ref_available() else "oracle"
    kind = "reference" if backend == "ref" else "port"
    o = cpu_engine(args.size, args.npml, np.float32, backend)
    t_start = time.perf_counter()
    for _ in range(args.warmup):
        o.step()
        if time.perf_counter() - t_start > 0.2 * args.cpu_budget:
            break
    per = []
    t_start = time.perf_counter()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.step()
        per.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > args.cpu_budget:
            break
    value = args.size**3 * len(per) / sum(per) / 1e6
    thr = num_threads()
    sample = (f"{len(per)} of {args.steps} requested Yee steps of the {args.size}^3 FP32 grid "
              f"(time budget {args.cpu_budget:.0f} s), {thr} OpenMP threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": "Mcell/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(args.size**3 / value / 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.size, args.npml, world),
        "arm": "the reference's Yee/CPML and source kernels on the host cores, with the same "
               "z-plane DFT of Ex at 4 frequencies (the oracle's plane-DFT monitor; the reference "
               "has no plane-DFT kernel)",
        "cpu_baseline": {"value": round(value, 2), "unit": "Mcell/s", "cores": thr, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 2), "unit": "Mcell/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    return line


def interior_alg_bytes(shape, npml, item=4):
    """Algorithmic bytes of one launch of the interior single-pass kernel: for every
    cell of the H box [npml, N-npml)^3 one read of E, H and ce and one write of E
    and H (15 arrays x item), with no ψ and no DFT (those run in the shell and
    plane-DFT kernels)."""
    n = 1
    for d in shape:
        n *= max(0, d - 2 * npml)
    return 15 * item * n


# The timed run's first steps are faster: until the pulse has filled the grid
# most field values are zero and the GPU stays below its power cap.  The bench
# line reports the rate before and after this many steps beside the average.
PHASE_SPLIT = 1000


def run_steps_timed(g, k):
    """Device time (ms) of k steps on the engine's stream (events on that stream),
    the library's per-launch times over the same steps, and its launch count."""
    import ctypes

    import torch

    from opencl_fdtd_solver_b200 import _capi as capi

    lib = capi.lib()
    st = g.queue
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    mid = torch.cuda.Event(enable_timing=True)
    split = min(k, PHASE_SPLIT)
    torch.cuda.synchronize()
    n0 = lib.fdtd_launch_count()
    capi.run("fdtd_profile_steps", 1)
    start.record(st)
    for n in range(k):
        if n == split:
            mid.record(st)
        g.step()
    if split == k:
        mid.record(st)
    end.record(st)
    torch.cuda.synchronize()
    capi.run("fdtd_profile_steps", 0)
    launches = lib.fdtd_launch_count() - n0
    ms = (ctypes.c_double * 5)()
    nsteps = ctypes.c_int32()
    capi.run("fdtd_profile_read", ms, ctypes.byref(nsteps))
    per_kernel = {name: ms[i] / max(1, nsteps.value)
                  for i, name in enumerate(("k_shell_H", "k_shell_E_side", "k_interior",
                                            "k_plane_dft_box", "k_shell_E"))}
    phases = {f"ms_per_step_first_{split}": round(start.elapsed_time(mid) / max(1, split), 4)}
    if k > split:
        phases[f"ms_per_step_after_{split}"] = round(mid.elapsed_time(end) / (k - split), 4)
    run_steps_timed.phases = phases
    return start.elapsed_time(end), per_kernel, launches


def run_b200_arm(args, rank, world, local):
    import torch

    size, npml = args.size, args.npml
    shape = (size, size, size)
    cells = size**3
    eps = blocky_eps(shape)
    g, mon = make_engine(size, npml, np.float32, fused=not args.split)
    g.set_epsilon(eps)
    for _ in range(args.warmup):
        g.step()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total_ms, per_kernel, launches = run_steps_timed(g, args.steps)
    phases = run_steps_timed.phases
    total_ms = reduce_max(total_ms, world)
    clocks = clk.summary()
    ms_per_step = total_ms / args.steps
    value = aggregate_rate(world, cells, args.steps, total_ms)
    fused = g._fused_enabled

    item = 4
    peak, peak_kind = measured_hbm()
    bpc = alg_bytes_per_cell(shape, npml, item, ((2, 1, len(FREQS)),))
    step_achieved = bpc * cells / (ms_per_step / 1e3) / 1e9
    if fused and per_kernel["k_interior"] > 0:
        # dominant kernel: the interior single-pass kernel (largest share of the step)
        k_ms = per_kernel["k_interior"]
        k_bytes = interior_alg_bytes(shape, npml, item)
        kname = "k_interior"
    else:
        kname, k_ms, k_bytes = "step (split kernels)", ms_per_step, bpc * cells
    achieved = k_bytes / (k_ms / 1e3) / 1e9
    traffic = None
    tp = ROOT / "profiles" / "yee_step_traffic.json"
    if tp.exists():
        try:
            tj = json.loads(tp.read_text())
            if tj.get("size") == size and tj.get("npml") == npml and tj.get("kernel") == kname:
                traffic = tj.get("bytes_per_launch")
        except Exception:
            traffic = None
    del g, mon
    torch.cuda.empty_cache()

    # end to end through the public API with host buffers: a new engine, εr
    # uploaded from the host (coefficients built on the device), the
    # configuration's full run (4000 steps by default) with the Python source
    # callback, the DFT plane and one field plane read back
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    g2, mon2 = make_engine(size, npml, np.float32, fused=not args.split)
    ev0.record(g2.queue)
    g2.set_epsilon(eps)
    e2e_steps = args.e2e_steps
    for _ in range(e2e_steps):
        g2.step()
    dft = mon2.dft("Ex")
    plane = g2.field_tensor("Ex")[:, :, size // 2].cpu().numpy()
    ev1.record(g2.queue)
    torch.cuda.synchronize()
    e2e_wall = time.perf_counter() - t0
    e2e_dev_ms = reduce_max(ev0.elapsed_time(ev1), world)
    e2e_value = aggregate_rate(world, cells, e2e_steps, e2e_dev_ms)
    h2d = eps.nbytes  # εr; the coefficients are built on the device
    d2h = dft.nbytes + plane.nbytes
    del g2, mon2
    torch.cuda.empty_cache()

    adjoint = None
    if not args.no_adjoint:
        barrier(world)
        adjoint = run_adjoint_leg(args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle.cpu_fdtd import ref_available

        backend = "ref" if ref_available() else "oracle"
        r, n, el, thr = cpu_reference_rate(size, npml, np.float32, args.cpu_seconds, backend)
        cpu = {"value": round(r, 2), "unit": "Mcell/s", "cores": thr,
               "kind": "reference" if backend == "ref" else "port",
               "sample": f"{n} steps of the same {size}^3 grid in {el:.1f} s (after 1 warm-up)"}
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mcell/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_config(size, npml, world),
        "fused_step": fused,
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1),
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic, "peak_source": peak_kind,
                     "alg_bytes_per_launch": int(k_bytes),
                     "ms_per_launch": round(k_ms, 4)},
        "step_roofline": {"alg_bytes_per_cell": round(bpc, 3),
                          "achieved": round(step_achieved, 1),
                          "frac": round(step_achieved / peak, 4),
                          "ms_per_launch": {k: round(v, 4) for k, v in per_kernel.items()},
                          "phases": phases},
        "e2e": {"value": round(e2e_value, 1), "unit": "Mcell/s",
                "h2d_bytes_per_step": int(h2d / e2e_steps),
                "d2h_bytes_per_step": int(d2h / e2e_steps), "steps": e2e_steps,
                "wall_s": round(e2e_wall, 3)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if adjoint is not None:
        line["adjoint"] = adjoint
    if not args.no_fp64:
        barrier(world)
        line["fp64"] = run_fp64_leg(args)
    if not args.no_n2f:
        barrier(world)
        line["n2f"] = run_n2f_leg(args)
    if not args.no_fp64_error:
        barrier(world)
        line["fp64_error"] = run_fp64_error_leg(args)
    if not args.no_huygens:
        barrier(world)
        line["huygens_box"] = run_huygens_leg(args)
    if rank == 0 and world == 1 and not args.no_cpu and not args.no_numpy:
        line["cpu_baseline_numpy"] = run_numpy_leg(args)
    return line


# ------------------------------------------------------------------ fp64 leg
def run_fp64_leg(args):
    """The same construction in FP64 mode (384³ by default): Mcell/s and the
    fraction of the HBM roofline from counted bytes per cell (FP64 fields)."""
    import torch

    size, npml = args.fp64_size, args.npml
    shape = (size, size, size)
    g, mon = make_engine(size, npml, np.float64)
    g.set_epsilon(blocky_eps(shape))
    for _ in range(3):
        g.step()
    torch.cuda.synchronize()
    k = args.fp64_steps
    total_ms, per_kernel, _ = run_steps_timed(g, k)
    ms = total_ms / k
    cells = size**3
    bpc = alg_bytes_per_cell(shape, npml, 8, ((2, 1, len(FREQS)),))
    peak, _ = measured_hbm()
    achieved = bpc * cells / (ms / 1e3) / 1e9
    del g, mon
    torch.cuda.empty_cache()
    return {"workload": f"yee_cpml_{size}^3_fp64_npml{npml}_blocky_eps_jx_point_zdft4",
            "value": round(cells * k / (total_ms / 1e3) / 1e6, 1), "unit": "Mcell/s",
            "steps": k, "ms_per_step": round(ms, 4), "alg_bytes_per_cell": round(bpc, 3),
            "achieved_gbs": round(achieved, 1), "frac": round(achieved / peak, 4),
            "ms_per_launch": {kk: round(v, 4) for kk, v in per_kernel.items()}}


# --------------------------------------------------------------- adjoint leg
ADJ_SHAPE = (160, 160, 96)
ADJ_NPML = 12
ADJ_DESIGN = ((32, 128), (32, 128), (40, 56))
ADJ_SHEET = dict(z=24, i0=12, i1=148, j0=12, j1=148)
ADJ_PLANE = 72
ADJ_PATCH = ((64, 96), (64, 96))
ADJ_FREQ = 30e9
ADJ_STEPS = 3000
ADJ_K = 100


def gaussian_sine(t, f0=30e9, fwidth=10e9):
    t0 = 5.0 / (np.pi * fwidth)
    sigma = 1.0 / (np.pi * fwidth)
    return float(np.exp(-0.5 * ((t - t0) / sigma) ** 2) * np.sin(2 * np.pi * f0 * t))


def design_eps(seed=2024, corr=6.0):
    """εr = 1 + 3·sigmoid(g) over the design box, g a seeded Gaussian random field
    (white noise smoothed by a Gaussian of σ = ``corr`` cells, periodic, unit variance)."""
    dims = tuple(hi - lo for lo, hi in ADJ_DESIGN)
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(dims)
    k = [np.fft.fftfreq(n) for n in dims]
    kk = sum(np.meshgrid(*[(2 * np.pi * v) ** 2 for v in k], indexing="ij"))
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * np.exp(-0.5 * corr**2 * kk)))
    g = (g - g.mean()) / g.std()
    return 1.0 + 3.0 / (1.0 + np.exp(-g))


def adjoint_problem(dtype, n_steps=ADJ_STEPS):
    from opencl_fdtd_solver_b200 import CUDAFDTD, DFTObjective, EpsilonAdjoint

    fd = CUDAFDTD(ADJ_SHAPE, 1e-3, npml=ADJ_NPML, dtype=dtype)
    s = ADJ_SHEET
    fd.add_source(lambda f: f.add_source_Jx(s["z"], gaussian_sine(f.t), s["i0"], s["i1"],
                                            s["j0"], s["j1"], rim_taper=True))
    obj = DFTObjective("z", ADJ_PLANE, ADJ_PATCH, [ADJ_FREQ], ("Ex",))
    return EpsilonAdjoint(fd, ADJ_DESIGN, n_steps, obj, checkpoint_every=ADJ_K)


def plain_forward(adj, eps_d):
    """One forward solve without checkpoints: set εr, run N steps with the DFT, read J."""
    import torch

    from opencl_fdtd_solver_b200 import CUDAPlaneDFTMonitor

    fd, o = adj.fdtd, adj.objective
    fd.set_epsilon(adj._eps_full(eps_d))
    fd.reset_state()
    saved = fd._monitors
    fd._monitors = []
    try:
        mon = CUDAPlaneDFTMonitor(fd, o.axis, o.index, o.freqs, o.components)
        fd.run(adj.n_steps)
    finally:
        fd._monitors = saved
    (a0, a1), (b0, b1) = o.patch
    D = torch.view_as_complex(mon.acc)[:, :, a0:a1, b0:b1]
    return float(o.fn(D))


def timed(fn, stream):
    import torch

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def run_adjoint_leg(args):
    """t_grad / t_forward at the adjoint configuration (FP32), and the gradient
    checked against central differences (h = 1e-3) at 16 seeded voxels in FP64."""
    import torch

    eps_d = design_eps()
    adj = adjoint_problem(np.float32, args.adj_steps)
    st = adj.fdtd.queue
    adj.value_and_grad(eps_d)  # warm-up
    plain_forward(adj, eps_d)
    t_fwd = min(timed(lambda: plain_forward(adj, eps_d), st)[0] for _ in range(3))
    t_grad, (J32, g32) = min((timed(lambda: adj.value_and_grad(eps_d), st) for _ in range(3)),
                             key=lambda r: r[0])
    # the two passes of the gradient apart: forward (with the captures) and the
    # reverse sweep alone, whose per-step time is the reverse step's
    t_fwd_cap = timed(lambda: adj.forward(eps_d), st)[0]
    t_bwd = timed(lambda: adj.backward(), st)[0]
    # the same reverse sweep with the interior plane march (the gradient is
    # bit-identical; the default is the per-cell sweep, measured faster here)
    adj.fused_reverse = True
    t_bwd_march = timed(lambda: adj.backward(), st)[0]
    adj.fused_reverse = False
    del adj
    torch.cuda.empty_cache()
    adj64 = adjoint_problem(np.float64, args.adj_steps)
    t64, (J64, g64) = timed(lambda: adj64.value_and_grad(eps_d), adj64.fdtd.queue)
    rng = np.random.default_rng(16)
    dims = g64.shape
    voxels = [tuple(int(rng.integers(0, d)) for d in dims) for _ in range(args.adj_fd_voxels)]
    h = 1e-3
    fd_g = []
    for v in voxels:
        ep = eps_d.copy()
        ep[v] += h
        jp = adj64.forward(ep)
        ep[v] -= 2 * h
        jm = adj64.forward(ep)
        fd_g.append((jp - jm) / (2 * h))
    fd_g = np.array(fd_g)
    ad64 = np.array([g64[v] for v in voxels])
    ad32 = np.array([g32[v] for v in voxels])
    n_design = int(np.prod(dims))
    del adj64
    torch.cuda.empty_cache()
    return {
        "workload": (f"adjoint_{ADJ_SHAPE[0]}x{ADJ_SHAPE[1]}x{ADJ_SHAPE[2]}_npml{ADJ_NPML}_"
                     f"design{dims[0]}x{dims[1]}x{dims[2]}_jx_sheet_30GHz_{args.adj_steps}steps_"
                     f"patch32x32_K{ADJ_K}"),
        "t_forward_ms": round(t_fwd, 2),
        "t_grad_ms": round(t_grad, 2),
        "grad_cost_forward_solves": round(t_grad / t_fwd, 3),
        "t_forward_with_captures_ms": round(t_fwd_cap, 2),
        "t_reverse_sweep_ms": round(t_bwd, 2),
        "reverse_step_us": round(1e3 * t_bwd / args.adj_steps, 2),
        "forward_step_us": round(1e3 * t_fwd / args.adj_steps, 2),
        "reverse_step_us_interior_march": round(1e3 * t_bwd_march / args.adj_steps, 2),
        "target_forward_solves": 4,
        "fd_gradient_cost_forward_solves": n_design + 1,
        "fd_gradient_ms_extrapolated": round((n_design + 1) * t_fwd, 1),
        "speedup_vs_fd_gradient": round((n_design + 1) * t_fwd / t_grad, 1),
        "fd_check": ({"voxels": len(voxels), "h": h, "dtype": "f64",
                      "rel_err": float(np.linalg.norm(ad64 - fd_g) / np.linalg.norm(fd_g)),
                      "rel_err_fp32_adjoint_vs_fd": float(np.linalg.norm(ad32 - fd_g)
                                                          / np.linalg.norm(fd_g))}
                     if voxels else None),
        "fp32_vs_fp64_grad_rel_err": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
        "J_fp32": J32, "J_fp64": J64, "t_grad_fp64_ms": round(t64, 2),
        "design_eps": "1 + 3 sigmoid(GRF), sigma 6 cells, seed 2024",
    }


# ------------------------------------------------------------------- n2f leg
def measured_tensor():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["bf16_tflops"]), "measured"
        except Exception:
            pass
    return 1590.0, "fallback"


def n2f_faces(n, nfreq, dl=1e-3, seed=4321, rho0=100.0):
    """Six faces of an n³ box: seeded complex Gaussian currents (complex64) under
    exp(-(ρ/ρ0)²), ρ the distance from the face centre in cells."""
    import torch

    from opencl_fdtd_solver_b200 import N2FFace

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    ra = torch.arange(n, device="cuda", dtype=torch.float32) - (n - 1) / 2
    env = torch.exp(-(ra[:, None] ** 2 + ra[None, :] ** 2) / rho0**2)
    faces = []
    for normal in range(3):
        for side in (0, 1):
            re = torch.randn((nfreq, n, n, 4), generator=g, device="cuda")
            im = torch.randn((nfreq, n, n, 4), generator=g, device="cuda")
            cur = torch.complex(re, im) * env[None, :, :, None]
            faces.append(N2FFace(normal=normal, x_n=(side - 0.5) * n * dl,
                                 o_p=(-n / 2 + 0.5) * dl, o_q=(-n / 2 + 0.5) * dl, pitch=dl,
                                 cur=cur.contiguous()))
    return faces


def n2f_directions(ntheta=361, nphi=181):
    th = np.linspace(0.0, np.pi, ntheta)
    ph = np.linspace(0.0, np.pi, nphi)
    T, P = np.meshgrid(th, ph, indexing="ij")
    return np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)


def run_n2f_leg(args):
    """The near-to-far contraction: 6 faces of an n³ box x 4 currents x nfreq
    frequencies onto 361 x 181 directions, split-BF16 and TF32 on the tensor cores,
    checked against the float64 direct sum on every 64th direction."""
    import torch

    from opencl_fdtd_solver_b200 import near2far_contract

    n, nfreq = args.n2f_size, args.n2f_freqs
    faces = n2f_faces(n, nfreq)
    dirs = n2f_directions()
    freqs = np.linspace(10e9, 40e9, nfreq)
    n_obs, ns = dirs.shape[0], 6 * n * n
    flops = 8.0 * n_obs * ns * 4 * nfreq
    peak, peak_kind = measured_tensor()
    st = torch.cuda.current_stream()
    out, modes = {}, {}
    for mode in ("bf16x3", "tf32"):
        near2far_contract(faces, freqs, dirs, mode=mode)
        best, res = None, None
        for _ in range(3):
            ms, r = timed(lambda: near2far_contract(faces, freqs, dirs, mode=mode), st)
            if best is None or ms < best:
                best, res = ms, r
        out[mode] = res
        modes[mode] = {"ms": round(best, 2), "alg_tflops": round(flops / best / 1e9, 1),
                       "frac_of_bf16_peak": round(flops / best / 1e9 / peak, 4),
                       "mma_products": 3 if mode == "bf16x3" else 1}
    sub = np.arange(0, n_obs, 64)
    t64, ref = timed(lambda: near2far_contract(faces, freqs, dirs[sub], mode="fp64"), st)
    ref = ref.cpu().numpy()
    for mode, res in out.items():
        o = res.cpu().numpy()[:, sub].astype(np.complex128)
        modes[mode]["rel_err_vs_fp64"] = float(np.linalg.norm(o - ref) / np.linalg.norm(ref))
        modes[mode]["max_err_over_peak"] = float(np.abs(o - ref).max() / np.abs(ref).max())
    t64_full = t64 * n_obs / sub.size
    return {
        "workload": f"n2f_box{n}^3_6faces_{ns}samples_x4_{nfreq}freqs_to_361x181_dirs",
        "alg_flops": flops, "peak_tflops": peak, "peak_source": peak_kind,
        "modes": modes,
        "fp64_direct_ms_subset": round(t64, 1), "fp64_subset_dirs": int(sub.size),
        "fp64_direct_ms_extrapolated": round(t64_full, 1),
        "speedup_bf16x3_vs_fp64_direct": round(t64_full / modes["bf16x3"]["ms"], 1),
    }


# ----------------------------------------------------------- host-monitor leg
def run_host_monitor_leg(args):
    """Per-step cost of the reference's host Huygens-box monitor on 256³ FP32
    (npml 12, box half-width 44 cells, one frequency): this package's
    ``NumPyNear2FarMonitor`` reading only its face slabs (``host_regions``)
    against the same monitor reading six full volumes per step, beside the bare
    step.  Wall-clock per step (the monitor runs on the host between steps)."""
    import torch

    from opencl_fdtd_solver_b200 import CUDAFDTD, NumPyNear2FarMonitor

    size, npml, dl, half = 256, 12, 1e-3, 44
    shape = (size,) * 3
    c = size // 2
    ctr = (c * dl,) * 3
    box = (2 * half * dl,) * 3

    class FullReads(NumPyNear2FarMonitor):
        host_regions = None

    def engine(mon_cls):
        g = CUDAFDTD(shape, dl, npml=npml)
        g.add_source(lambda f: f.add_source_Jx(c, gaussian_sine(f.t), i0=c, i1=c + 1, j0=c,
                                               j1=c + 1))
        m = mon_cls(g, ctr, box, ADJ_FREQ) if mon_cls else None
        return g, m

    def per_step(g, k):
        for _ in range(3):
            g.step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k):
            g.step()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / k * 1e3

    out = {"workload": f"host_n2f_monitor_{size}^3_fp32_npml{npml}_box{2 * half + 1}",
           "unit": "ms/step"}
    g, _ = engine(None)
    out["bare_step_ms"] = round(per_step(g, 200), 4)
    del g
    g, m = engine(NumPyNear2FarMonitor)
    out["windowed_ms"] = round(per_step(g, 100), 4)
    cells = sum((a1 - a0) * (b1 - b0) * (c1 - c0)
                for (a0, a1), (b0, b1), (c0, c1) in m.host_regions())
    out["windowed_d2h_bytes_per_step"] = 6 * 4 * cells
    del g, m
    g, m = engine(FullReads)
    out["full_reads_ms"] = round(per_step(g, 10), 4)
    out["full_reads_d2h_bytes_per_step"] = 6 * 4 * size**3
    del g, m
    torch.cuda.empty_cache()
    out["speedup"] = round(out["full_reads_ms"] / out["windowed_ms"], 2)
    return out


# ------------------------------------------------------- NumPy CPU baseline
def numpy_rate(size, npml, courant, eps, warm, windows, per_window):
    """Mcell/s of the NumPy face-CPML engine (the reference's NumPy algorithm,
    restated bit-identically in ``oracle/numpy_face_cpml.py``): warm-up steps,
    then ``windows`` timed windows of ``per_window`` steps, median
    (reference ``benchmarks/benchmark_vs_meep.py:108-122``)."""
    from oracle.numpy_face_cpml import NumPyFaceCPML

    shape = (size,) * 3
    o = NumPyFaceCPML(shape, 1e-3, npml=npml, courant=courant)
    if eps is not None:
        o.set_epsilon(eps)
    c = size // 2
    o.add_source(lambda f: f.add_source_Jx(c, gaussian_pulse(f.t), i0=c, i1=c + 1, j0=c, j1=c + 1))
    o.run(warm)
    rates = []
    for _ in range(windows):
        t0 = time.perf_counter()
        o.run(per_window)
        rates.append(size**3 * per_window / (time.perf_counter() - t0) / 1e6)
    return statistics.median(rates), rates


def run_numpy_leg(args):
    """The reference's NumPy engine (face-striped CPML) on the host: the small
    configuration's 64³ grid (2 warm-up steps, 3 windows of 10) and the 512³
    roofline grid (1 warm-up step, 3 windows of 1 step; full-length NumPy runs
    at 512³ take hours).  NumPy evaluates each array operation on one core."""
    r64, w64 = numpy_rate(64, 8, 0.5, None, 2, 3, 10)
    out = {"kind": "port", "engine": "NumPyFDTD_FaceCPML algorithm (oracle/numpy_face_cpml.py, "
                                      "bit-identical to the reference on its fixtures)",
           "threads": 1, "host_cpus": os.cpu_count(),
           "omp_num_threads": os.environ.get("OMP_NUM_THREADS"),
           "small_64^3": {"value": round(r64, 2), "unit": "Mcell/s",
                          "windows_mcells": [round(x, 2) for x in w64],
                          "sample": "64^3 FP32 vacuum, npml 8, Courant 0.5, 2 warm-up + 3 x 10 steps"}}
    if not args.numpy_small_only:
        shape = (args.size,) * 3
        r512, w512 = numpy_rate(args.size, args.npml, None, blocky_eps(shape), 1, 3, 1)
        out[f"roofline_{args.size}^3"] = {
            "value": round(r512, 2), "unit": "Mcell/s", "windows_mcells": [round(x, 2) for x in w512],
            "sample": f"{args.size}^3 FP32 blocky eps, npml {args.npml}, 1 warm-up + 3 x 1 step"}
    return out


# ------------------------------------------------------ FP32 vs FP64 errors
def _peak_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a.astype(np.complex128 if np.iscomplexobj(a) else np.float64) - b).max()
                 / np.abs(b).max())


def run_fp64_error_leg(args):
    """Each FP32 result's peak-normalised error against an FP64 run of the same
    configuration (``max|x32 - x64| / max|x64|``):
      * small (64³, npml 8, Courant 0.5, Jx point, 500 steps): Ex, Hy and their
        z = 32 plane DFTs at 25/30/35 GHz, against the FP64 NumPy face-CPML engine;
      * medium (256³ sphere, rim-tapered sheet, 2000 steps): the 8-frequency box
        DFTs and the far field at 20 and 40 GHz (direct and split-BF16), against
        the FP64 CUDA engine (itself within 1e-12 of FP64 NumPy on the parity tests);
      * roofline (512³ blocky εr): the six fields and the Ex plane DFT after
        ``--fp64-error-steps`` steps, against the FP64 CUDA engine.
    H errors are also given over η0 times the E peak: the sources leave a static
    charge field in E near them, H is a difference of those large E values, and
    its own peak is small once the pulse has left."""
    import torch

    from opencl_fdtd_solver_b200 import CUDAFDTD, CUDAPlaneDFTMonitor
    from oracle.numpy_face_cpml import NumPyFaceCPML

    out = {}
    # small configuration
    freqs = [25e9, 30e9, 35e9]
    g = CUDAFDTD((64,) * 3, 1e-3, npml=8, courant=0.5)
    src = lambda f: f.add_source_Jx(32, gaussian_sine(f.t, 30e9, 20e9), i0=32, i1=33, j0=32,
                                    j1=33)
    g.add_source(src)
    m = CUDAPlaneDFTMonitor(g, "z", 32, freqs, ("Ex", "Hy"))
    g.run(500)
    o = NumPyFaceCPML((64,) * 3, 1e-3, npml=8, dtype=np.float64, courant=0.5)
    o.add_source(src)
    om = 2 * np.pi * np.array(freqs)
    acc = {c: np.zeros((3, 64, 64), np.complex128) for c in ("Ex", "Hy")}
    st = {"p": None}

    def plane(f):
        st["p"] = (np.exp(1j * om * f.t) * f.dt if st["p"] is None
                   else st["p"] * np.exp(1j * om * f.dt))
        ph = st["p"] * np.exp(-0.5j * om * f.dt)
        acc["Ex"] += st["p"][:, None, None] * f.Ex[:, :, 32][None]
        acc["Hy"] += ph[:, None, None] * f.Hy[:, :, 32][None]

    o.add_monitor(plane)
    o.run(500)
    from opencl_fdtd_solver_b200 import ETA0

    e_peak = np.abs(o.Ex).max()
    out["small_64^3_500steps_vs_fp64_numpy"] = {
        "Ex": _peak_err(g.Ex, o.Ex), "Hy": _peak_err(g.Hy, o.Hy),
        "Hy_over_eta0_Ex_peak": float(ETA0 * np.abs(g.Hy.astype(np.float64) - o.Hy).max()
                                      / e_peak),
        "dft_Ex": _peak_err(m.dft("Ex"), acc["Ex"]), "dft_Hy": _peak_err(m.dft("Hy"), acc["Hy"])}
    del g, m, o
    torch.cuda.empty_cache()
    # medium configuration
    th = np.deg2rad(np.linspace(0.0, 180.0, 181))
    ph_ = np.deg2rad(np.linspace(0.0, 180.0, 91, endpoint=False))
    T, P = np.meshgrid(th, ph_, indexing="ij")
    pts = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    res = {}
    for dt_ in (np.float32, np.float64):
        gm, mon = medium_engine(box=True, dtype=dt_)
        gm.run(args.fp64_error_medium_steps)
        r = {"box": [mon.face_dft(fi) for fi in range(MED_FREQS.size)],
             "ff": {fi: mon.get_farfields(pts, fi) for fi in (0, MED_FREQS.size - 1)}}
        if dt_ == np.float32:
            r["ff_bf16x3"] = {fi: mon.get_farfields(pts, fi, method="bf16x3")
                              for fi in (0, MED_FREQS.size - 1)}
        res[dt_] = r
        del gm, mon
        torch.cuda.empty_cache()
    a, b = res[np.float32], res[np.float64]
    box_err = max(_peak_err(a["box"][fi][c], b["box"][fi][c])
                  for fi in range(MED_FREQS.size) for c in a["box"][fi])
    out[f"medium_{MED_N}^3_{args.fp64_error_medium_steps}steps_vs_fp64_cuda"] = {
        "box_dft_max_over_freqs_components": box_err,
        "farfield_direct": {f"{MED_FREQS[fi] / 1e9:.0f}GHz": _peak_err(a["ff"][fi], b["ff"][fi])
                            for fi in a["ff"]},
        "farfield_bf16x3": {f"{MED_FREQS[fi] / 1e9:.0f}GHz": _peak_err(a["ff_bf16x3"][fi],
                                                                       b["ff"][fi])
                            for fi in a["ff"]}}
    # roofline grid
    n, k = args.size, args.fp64_error_steps
    shape = (n,) * 3
    eps = blocky_eps(shape)
    ref = None
    errs = {}
    for dt_ in (np.float64, np.float32):  # FP64 first; its fields stay on the device
        gr, mr = make_engine(n, args.npml, dt_)
        gr.set_epsilon(eps)
        gr.run(k)
        cur = {f: gr.field_tensor(f).double() for f in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}
        dft = mr.dft("Ex")
        if ref is None:
            ref = ({f: t.clone() for f, t in cur.items()}, dft)
        else:
            from opencl_fdtd_solver_b200 import ETA0

            e_peak = max(float(ref[0][f].abs().max()) for f in ("Ex", "Ey", "Ez"))
            for f, t in cur.items():
                d = float((t - ref[0][f]).abs().max())
                errs[f] = d / float(ref[0][f].abs().max())
                if f[0] == "H":
                    errs[f + "_over_eta0_E_peak"] = ETA0 * d / e_peak
            errs["dft_Ex"] = _peak_err(dft, ref[1])
        del gr, mr, cur
        torch.cuda.empty_cache()
    del ref
    torch.cuda.empty_cache()
    out[f"roofline_{n}^3_{k}steps_vs_fp64_cuda"] = errs
    return out


# ------------------------------------------------------- medium-config legs
MED_N, MED_NPML, MED_HALF = 256, 12, 44
MED_FREQS = np.linspace(20e9, 40e9, 8)


def medium_engine(box=True, fused=True, dtype=np.float32):
    """The medium configuration: 256³ FP32, npml 12, εr = 4 sphere (r = 40
    cells), a rim-tapered Jx sheet at z = npml + 8 across the PML-free span, and
    (``box``) the 6-face Huygens DFT box of half-width 44 cells at 8 frequencies."""
    from opencl_fdtd_solver_b200 import CUDAFDTD, CUDANear2FarMonitor

    n, npml, dl = MED_N, MED_NPML, 1e-3
    shape = (n,) * 3
    ii, jj, kk = np.meshgrid(*[np.arange(n)] * 3, indexing="ij", sparse=True)
    eps = np.ones(shape, np.float32)
    eps[(ii - n // 2) ** 2 + (jj - n // 2) ** 2 + (kk - n // 2) ** 2 < 40**2] = 4.0
    g = CUDAFDTD(shape, dl, npml=npml, dtype=dtype, fused=fused)
    g.set_epsilon(eps)
    z = npml + 8
    g.add_source(lambda f: f.add_source_Jx(z, gaussian_sine(f.t, 30e9, 20e9), npml, n - npml,
                                           npml, n - npml, rim_taper=True))
    mon = None
    if box:
        mon = CUDANear2FarMonitor(g, (n // 2 * dl,) * 3, (2 * MED_HALF * dl,) * 3, MED_FREQS)
    return g, mon


def run_huygens_leg(args):
    """Cost of the Huygens-box face DFT (89³ box, 8 frequencies) on the medium
    configuration: ms per step with and without the box monitor, device time by
    CUDA events on the engine's stream and host wall time (the monitor's launch
    is issued from its Python callback after each step).  The two engines run
    alternately, three windows each, and the medians are compared, so that a
    drift of the board's clock between windows does not enter the difference.
    The reference quotes about 1.5 % for its fused 6-face DFT (README.md:192)."""
    import torch

    k = args.huygens_steps
    out = {"workload": f"medium_{MED_N}^3_fp32_npml{MED_NPML}_sphere_sheet_box"
                       f"{2 * MED_HALF + 1}^3_{MED_FREQS.size}freqs", "steps_per_window": k,
           "windows": 3}
    engines = {tag: medium_engine(box=box) for tag, box in (("no_box", False), ("box", True))}
    for g, _ in engines.values():
        for _ in range(args.warmup):
            g.step()
    torch.cuda.synchronize()
    times = {tag: {"wall": [], "device": []} for tag in engines}
    for _ in range(3):
        for tag, (g, _) in engines.items():
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e0.record(g.queue)
            for _ in range(k):
                g.step()
            e1.record(g.queue)
            torch.cuda.synchronize()
            times[tag]["wall"].append((time.perf_counter() - t0) / k * 1e3)
            times[tag]["device"].append(e0.elapsed_time(e1) / k)
    for tag in engines:
        for kind in ("wall", "device"):
            out[f"{tag}_{kind}_ms_per_step"] = round(float(np.median(times[tag][kind])), 4)
    del engines
    torch.cuda.empty_cache()
    for kind in ("wall", "device"):
        a, b = out[f"no_box_{kind}_ms_per_step"], out[f"box_{kind}_ms_per_step"]
        out[f"overhead_{kind}_pct"] = round(100.0 * (b - a) / a, 2)
    out["reference_claim_pct"] = 1.5
    return out


def run_kernels_leg(args):
    """One launch (after warm-up) of each auxiliary kernel at documented sizes,
    timed by CUDA events; the workload of the per-kernel ncu summaries.
      * medium configuration (256³, npml 12): one fused step with the Huygens box
        (k_shell_H, k_interior, k_plane_dft_box, k_shell_E, k_dft_faces) and one
        split step (k_update_H, k_update_E), with a z-plane DFT of Ex at 4 freqs;
      * the far field of the box at one frequency onto 181 x 91 directions
        (k_farfield_nl, k_farfield_eh);
      * the tensor-core contraction of a 160³ box (6 faces, 4 currents, 8 freqs)
        onto 361 x 181 directions in split-BF16 (k_n2f_pack, k_n2f_tc, k_n2f_combine)."""
    import torch

    from opencl_fdtd_solver_b200 import CUDAPlaneDFTMonitor, near2far_contract

    res = {}
    g, mon = medium_engine(box=True)
    CUDAPlaneDFTMonitor(g, "z", MED_N // 2, FREQS, ("Ex",))
    for _ in range(args.warmup):
        g.step()
    st = g.queue
    res["fused_step_with_box_ms"] = round(timed(g.step, st)[0], 4)
    g._fused_enabled = False
    res["split_step_with_box_ms"] = round(timed(g.step, st)[0], 4)
    th = np.deg2rad(np.linspace(0.0, 180.0, 181))
    ph = np.deg2rad(np.linspace(0.0, 180.0, 91, endpoint=False))
    T, P = np.meshgrid(th, ph, indexing="ij")
    pts = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    res["farfield_direct_16471_ms"] = round(timed(lambda: mon.get_farfields(pts, 3), st)[0], 3)
    del g, mon
    torch.cuda.empty_cache()
    faces = n2f_faces(160, 8)
    dirs = n2f_directions()
    freqs = np.linspace(10e9, 40e9, 8)
    res["n2f_bf16x3_box160_8freqs_ms"] = round(
        timed(lambda: near2far_contract(faces, freqs, dirs, mode="bf16x3"),
              torch.cuda.current_stream())[0], 3)
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4000,
                    help="timed steps (default: the configuration's full 4000-step run; the "
                         "step slows by ~3%% once the pulse has filled the grid, so a short "
                         "early window would overstate the rate)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--npml", type=int, default=16)
    ap.add_argument("--split", action="store_true", help="use the two-kernel half-step path")
    ap.add_argument("--e2e-steps", type=int, default=4000,
                    help="steps of the end-to-end run (the configuration's full length)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="CPU-baseline sample length beside the GPU arm")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint-gradient leg (t_grad / t_forward, FD check)")
    ap.add_argument("--no-n2f", action="store_true", help="skip the near-to-far contraction leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 throughput leg")
    ap.add_argument("--no-huygens", action="store_true", help="skip the Huygens-box overhead leg")
    ap.add_argument("--fp64-size", type=int, default=384)
    ap.add_argument("--fp64-steps", type=int, default=100)
    ap.add_argument("--only", choices=("n2f", "adjoint", "fp64", "host_monitor", "huygens",
                                       "kernels", "numpy", "fp64_error"),
                    help="run one auxiliary leg alone and print its object (profiling)")
    ap.add_argument("--n2f-size", type=int, default=320, help="box edge (samples per face side)")
    ap.add_argument("--n2f-freqs", type=int, default=32)
    ap.add_argument("--adj-steps", type=int, default=ADJ_STEPS, help="time steps per adjoint solve")
    ap.add_argument("--no-numpy", action="store_true", help="skip the NumPy CPU-baseline leg")
    ap.add_argument("--numpy-small-only", action="store_true",
                    help="NumPy CPU baseline at 64^3 only (skip the 512^3 sample)")
    ap.add_argument("--no-fp64-error", action="store_true",
                    help="skip the FP32-vs-FP64 error leg")
    ap.add_argument("--fp64-error-steps", type=int, default=1200,
                    help="steps of the 512^3 FP32-vs-FP64 comparison")
    ap.add_argument("--fp64-error-medium-steps", type=int, default=2000,
                    help="steps of the medium-configuration FP32-vs-FP64 comparison")
    ap.add_argument("--huygens-steps", type=int, default=500,
                    help="timed steps of each arm of the Huygens-box overhead leg")
    ap.add_argument("--adj-fd-voxels", type=int, default=16,
                    help="design voxels checked by central differences")
    ap.add_argument("--cpu-budget", type=float, default=60.0,
                    help="time budget of the --impl reference arm's timed steps")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        line = run_reference_arm(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0
    rank, world, local = dist_setup(args.gpus)
    if args.only:
        res = {"n2f": run_n2f_leg, "adjoint": run_adjoint_leg, "fp64": run_fp64_leg,
               "host_monitor": run_host_monitor_leg, "huygens": run_huygens_leg,
               "kernels": run_kernels_leg, "numpy": run_numpy_leg,
               "fp64_error": run_fp64_error_leg}[args.only](args)
        if rank == 0:
            print(json.dumps({args.only: res}), flush=True)
        return 0
    line = run_b200_arm(args, rank, world, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
