"""Multi-process replica path of bench.py on CPU (gloo, world size 2).

The engine runs one grid per GPU, so N GPUs run N independent replicas; the
only collectives are a barrier and the max over ranks of the timed region.
These tests run that host logic with two gloo ranks on 127.0.0.1: rank set-up
from the torchrun environment, the max-reduction, the barrier, and the
whole-job rate computed from the slowest replica, each replica advancing a
small grid with the CPU oracle (no GPU needed).
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import json
    import time

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    from oracle.cpu_fdtd import OracleFDTD, set_num_threads

    set_num_threads(1)
    r, w, local = bench.dist_setup(world, backend="gloo")
    assert (r, w, local) == (rank, world, rank)
    shape, steps = (24, 20, 16), 6
    o = OracleFDTD(shape, 1e-3, npml=4, dtype=np.float32)
    o.add_source(lambda f: f.add_source_Jx(8, np.sin(2e10 * f.t), 10, 12, 9, 11))
    bench.barrier(w)
    t0 = time.perf_counter()
    o.run(steps)
    if rank == 1:
        time.sleep(0.05)  # the slower replica
    ms = (time.perf_counter() - t0) * 1e3
    worst = bench.reduce_max(ms, w)
    bench.barrier(w)
    rate = bench.aggregate_rate(w, int(np.prod(shape)), steps, worst)
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as fh:
        json.dump({"ms": ms, "worst": worst, "rate": rate, "ex_sum": float(np.abs(o.Ex).sum())}, fh)
    import torch.distributed as dist

    dist.destroy_process_group()


def test_two_gloo_replicas_max_reduce_and_rate(tmp_path):
    import json
    import sys
    from pathlib import Path

    root = str(Path(__file__).resolve().parents[1])
    if root not in sys.path:
        sys.path.insert(0, root)
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(2)]
    worst = max(r["ms"] for r in res)
    assert res[1]["ms"] >= 50.0
    for r in res:
        assert r["worst"] == pytest.approx(worst)       # every rank sees the slowest replica
    assert res[0]["rate"] == pytest.approx(res[1]["rate"])
    # the aggregate rate counts both replicas' cells over the slowest time
    assert res[0]["rate"] == pytest.approx(2 * 24 * 20 * 16 * 6 / (worst / 1e3) / 1e6)
    assert res[0]["ex_sum"] > 0 and res[1]["ex_sum"] > 0


def test_single_process_needs_no_process_group():
    import bench

    os.environ.pop("WORLD_SIZE", None)
    assert bench.reduce_max(3.5, 1) == 3.5
    bench.barrier(1)
    assert bench.aggregate_rate(1, 1000, 10, 1000.0) == pytest.approx(0.01)
