"""x-slab decomposition on CPU: partition rules and a gloo multi-rank run.

Each rank advances its slab of the grid (the NumPy face-CPML restatement of the
reference engine, with the x-CPML only on global faces and one ghost plane per
inner side) and exchanges ghost planes after every step over
``torch.distributed`` (gloo, 127.0.0.1).  The owned planes gathered from all
ranks must equal the single-domain run bit for bit: fields, with a rim-tapered
sheet that spans the slab boundary and a dielectric block across it.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from opencl_fdtd_solver_b200 import slabs
from oracle.numpy_face_cpml import NumPyFaceCPML
from tests.cases import gaussian_sine

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")

SHAPE, NPML, STEPS = (26, 14, 12), 3, 40
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _eps():
    eps = np.ones(SHAPE, np.float32)
    eps[9:17, 4:10, 3:9] = 3.5  # straddles the slab boundaries at 2 and 3 ranks
    return eps


def _source(f):
    f.add_source_Jx(6, gaussian_sine(f.t, 60e9, 40e9), i0=5, i1=21, j0=3, j1=11,
                    rim_taper=True)


def _single():
    o = NumPyFaceCPML(SHAPE, 1e-3, npml=NPML)
    o.set_epsilon(_eps())
    o.add_source(_source)
    o.run(STEPS)
    return {n: getattr(o, n).copy() for n in FIELDS}


def test_partition_rules():
    p = slabs.partition(26, 3, 3)
    assert [(s.g0, s.g1) for s in p] == [(0, 9), (9, 18), (18, 26)]
    assert [(s.ghost_lo, s.ghost_hi) for s in p] == [(0, 1), (1, 1), (1, 0)]
    assert [(s.pml_lo, s.pml_hi) for s in p] == [(3, 0), (0, 0), (0, 3)]
    assert [s.nx_local for s in p] == [10, 11, 9]
    assert [s.l0 for s in p] == [0, 8, 17]
    assert p[1].owned == slice(1, 10) and p[1].last_owned == 9
    with pytest.raises(ValueError):
        slabs.partition(8, 3, 3)  # rank 0 would own 3 planes beside 3 CPML layers
    one = slabs.partition(26, 1, 3)[0]
    assert (one.nx_local, one.pml_lo, one.pml_hi, one.ghost_lo, one.ghost_hi) == (26, 3, 3, 0, 0)


@pytest.mark.parametrize("ranks", [2, 3])
def test_local_exchange_equals_single_domain(ranks):
    """All slabs in one process, ghosts copied directly (the path a single
    process uses when it holds several slabs)."""
    plan = slabs.partition(SHAPE[0], ranks, NPML)
    sims = [NumPyFaceCPML(SHAPE, 1e-3, npml=NPML, slab=s) for s in plan]
    for o in sims:
        o.set_epsilon(_eps())
        o.add_source(_source)
    views = lambda r: (lambda n, i: getattr(sims[r], n)[i])
    for _ in range(STEPS):
        for o in sims:
            o.step()
        slabs.local_exchange(plan, views)
    ref = _single()
    for n in FIELDS:
        got = np.concatenate([getattr(o, n)[s.owned] for o, s in zip(sims, plan)])
        assert np.abs(ref[n]).max() > 0, n
        assert np.array_equal(got, ref[n]), n


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    s = slabs.partition(SHAPE[0], world, NPML)[rank]
    o = NumPyFaceCPML(SHAPE, 1e-3, npml=NPML, slab=s)
    o.set_epsilon(_eps())
    o.add_source(_source)
    send, recv, wait = slabs.dist_transport()
    planes = lambda n, i: torch.from_numpy(getattr(o, n)[i])  # views share memory
    for _ in range(STEPS):
        o.step()
        slabs.exchange_ghosts(s, planes, send, recv)
        wait()
    np.savez(os.path.join(out_dir, f"r{rank}.npz"),
             **{n: getattr(o, n)[s.owned] for n in FIELDS})
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_equal_single_domain(tmp_path, world):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0, p.exitcode
    ref = _single()
    parts = [np.load(tmp_path / f"r{r}.npz") for r in range(world)]
    for n in FIELDS:
        got = np.concatenate([p[n] for p in parts])
        assert np.array_equal(got, ref[n]), n
