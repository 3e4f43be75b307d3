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


def dist_setup(n_gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def reduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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
    """The same grid on the CPU (reference kernels compiled as C, or the oracle port)."""
    from oracle.cpu_fdtd import OracleFDTD

    shape = (size, size, size)
    o = OracleFDTD(shape, 1e-3, npml=npml, dtype=dtype, backend=backend)
    o.set_epsilon(blocky_eps(shape))
    c = size // 2
    o.add_source(lambda f: f.add_source_Jx(c, gaussian_pulse(f.t), i0=c, i1=c + 1, j0=c, j1=c + 1))
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
        "config": {"workload": f"yee_cpml_{args.size}^3_fp32_npml{args.npml}_blocky_eps",
                   "cpu": True},
        "cpu_baseline": {"value": round(value, 2), "unit": "Mcell/s", "cores": thr, "kind": kind,
                         "sample": sample},
        "e2e": {"value": round(value, 2), "unit": "Mcell/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    return line


def time_steps(g, k, event_pairs=True):
    """Device time (ms) of k steps on the engine's stream, bracketed by events."""
    import torch

    st = g.queue
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    per = []
    torch.cuda.synchronize()
    start.record(st)
    evs = []
    for _ in range(k):
        if event_pairs:
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
        g.step()
        if event_pairs:
            b.record(st)
            evs.append((a, b))
    end.record(st)
    torch.cuda.synchronize()
    total = start.elapsed_time(end)
    per = [a.elapsed_time(b) for a, b in evs]
    return total, per


def run_b200_arm(args, rank, world, local):
    import torch

    from opencl_fdtd_solver_b200 import CUDAFDTD

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
        total_ms, per = time_steps(g, args.steps)
    total_ms = reduce_max(total_ms, world)
    clocks = clk.summary()
    ms_per_step = total_ms / args.steps
    value = world * cells * args.steps / (total_ms / 1e3) / 1e6
    fused = g._fused_enabled
    launches_per_step = 1 if fused else 2

    # roofline of the dominant kernel (the fused step: one launch per step)
    item = 4
    bpc = alg_bytes_per_cell(shape, npml, item, ((2, 1, len(FREQS)),))
    per_launch_ms = statistics.mean(per)
    achieved = bpc * cells / (per_launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_hbm()
    traffic = None
    tp = ROOT / "profiles" / "yee_step_traffic.json"
    if tp.exists():
        try:
            tj = json.loads(tp.read_text())
            if tj.get("size") == size and tj.get("fused") == fused:
                traffic = tj.get("bytes_per_launch")
        except Exception:
            traffic = None

    # end to end through the public API with host buffers: ε upload (host → ce on
    # device), K steps with the Python source callback, DFT plane + one field
    # plane read back to the host
    del g, mon
    torch.cuda.empty_cache()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    g2, mon2 = make_engine(size, npml, np.float32, fused=not args.split)
    ev0.record(g2.queue)
    g2.set_epsilon(eps)
    for _ in range(args.steps):
        g2.step()
    dft = mon2.dft("Ex")
    plane = g2.field_tensor("Ex")[:, :, size // 2].cpu().numpy()
    ev1.record(g2.queue)
    torch.cuda.synchronize()
    e2e_wall = time.perf_counter() - t0
    e2e_dev_ms = reduce_max(ev0.elapsed_time(ev1), world)
    e2e_s = max(e2e_dev_ms / 1e3, 0.0)
    e2e_value = world * cells * args.steps / e2e_s / 1e6
    h2d = 3 * cells * item  # ce arrays built from the host ε
    d2h = dft.nbytes + plane.nbytes
    del g2, mon2
    torch.cuda.empty_cache()

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
        "config": {"workload": f"yee_cpml_{size}^3_fp32_npml{npml}_blocky_eps_jx_point_zdft4",
                   "grid": list(shape), "npml": npml, "plane_dft_freqs_hz": list(FREQS),
                   "eps_seed": 1234, "fused_step": fused,
                   "l2": "inputs (~9 GB/step) exceed L2; no flush",
                   "parallelism": f"replicas{world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": peak_kind, "alg_bytes_per_cell": round(bpc, 3)},
        "e2e": {"value": round(e2e_value, 1), "unit": "Mcell/s",
                "h2d_bytes_per_step": int(h2d / args.steps),
                "d2h_bytes_per_step": int(d2h / args.steps),
                "wall_s": round(e2e_wall, 3)},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    return line


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--npml", type=int, default=16)
    ap.add_argument("--split", action="store_true", help="use the two-kernel half-step path")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="CPU-baseline sample length beside the GPU arm")
    ap.add_argument("--cpu-budget", type=float, default=150.0,
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
    line = run_b200_arm(args, rank, world, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
