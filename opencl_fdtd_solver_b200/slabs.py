"""x-slab decomposition of one grid over several ranks (one rank per GPU).

The reference runs a grid on one device and bounds it by that device's memory
(``opencl_fdtd_solver/engine.py:320-363``).  Here a grid too large for one GPU
is split along x, the slowest axis, into contiguous slabs of planes, one per
rank.  Each rank holds its owned planes plus one ghost plane on each side that
faces another rank:

* the ghost below the owned planes holds the lower neighbour's last owned
  plane of E and H (H of the ghost is advanced locally from it, so E of the
  first owned plane sees the same H^{n+1/2} as in one domain);
* the ghost above holds the upper neighbour's first owned plane of E (the
  forward differences of H on the last owned plane read it).

A step is the unchanged single-domain step on the local grid, with the x-CPML
only on the sides that are global faces, followed by one ghost exchange: Ex,
Ey, Ez, Hy, Hz of the last owned plane go up, Ey, Ez of the first owned plane go
down (the planes the next step reads; a plane at fixed i is contiguous in the
C-order layout, so no packing is needed).  Ghost planes are recomputed with
boundary-guarded differences during the step and then overwritten, so owned
cells see exactly the values of one domain and the result is identical to the
single-domain run bit for bit.

The exchange runs over ``torch.distributed`` point-to-point operations (NCCL on
GPUs, gloo on CPU), or, for slabs held by one process, as direct copies.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

# planes a ghost needs: the lower ghost E (all) and Hy, Hz; the upper ghost Ey, Ez
UP_FIELDS = ("Ex", "Ey", "Ez", "Hy", "Hz")
DOWN_FIELDS = ("Ey", "Ez")


@dataclass(frozen=True)
class SlabLocal:
    """One rank's slab: owned global planes [g0, g1) and its local grid."""

    rank: int
    ranks: int
    nx: int        # global planes
    g0: int
    g1: int
    npml: int

    @property
    def ghost_lo(self) -> int:
        return 1 if self.rank > 0 else 0

    @property
    def ghost_hi(self) -> int:
        return 1 if self.rank < self.ranks - 1 else 0

    @property
    def l0(self) -> int:
        """Global index of local plane 0."""
        return self.g0 - self.ghost_lo

    @property
    def nx_local(self) -> int:
        return self.g1 - self.g0 + self.ghost_lo + self.ghost_hi

    @property
    def pml_lo(self) -> int:
        """x-CPML layers at the local low side (the global low face only)."""
        return self.npml if self.rank == 0 else 0

    @property
    def pml_hi(self) -> int:
        return self.npml if self.rank == self.ranks - 1 else 0

    @property
    def owned(self) -> slice:
        """Local planes this rank owns."""
        return slice(self.ghost_lo, self.ghost_lo + self.g1 - self.g0)

    @property
    def first_owned(self) -> int:
        return self.ghost_lo

    @property
    def last_owned(self) -> int:
        return self.ghost_lo + self.g1 - self.g0 - 1


def partition(nx: int, ranks: int, npml: int) -> list[SlabLocal]:
    """Balanced contiguous x-slabs (sizes differ by at most one plane).

    Each slab must own more planes than the x-CPML it carries, so that its
    ghost planes lie outside the CPML, and at least two planes.
    """
    if ranks < 1:
        raise ValueError(f"ranks must be >= 1, got {ranks}")
    base, extra = divmod(int(nx), ranks)
    out, g = [], 0
    for r in range(ranks):
        n = base + (1 if r < extra else 0)
        s = SlabLocal(rank=r, ranks=ranks, nx=int(nx), g0=g, g1=g + n, npml=int(npml))
        need = max(2, (s.pml_lo + s.pml_hi) + 1) if ranks > 1 else 1
        if n < need:
            raise ValueError(f"slab {r} owns {n} planes; it needs at least {need} "
                             f"(nx={nx}, ranks={ranks}, npml={npml})")
        out.append(s)
        g += n
    return out


def clip_sheet(s: SlabLocal, i0: int, i1: int) -> tuple[int, int]:
    """A sheet's global [i0, i1) in local plane indices (may reach outside the
    local grid; the kernels and host code apply it only to local cells, and the
    rim taper still refers to the sheet's global edges)."""
    return i0 - s.l0, i1 - s.l0


def exchange_ghosts(s: SlabLocal, planes, send, recv) -> None:
    """One ghost exchange after a step.

    planes(name, local_i) -> the plane tensor/array view of field ``name``;
    send(peer, tensors) / recv(peer, tensors) move lists of planes (recv fills
    the given views in place).  The lower neighbour gets this rank's first owned
    plane of DOWN_FIELDS into its upper ghost; the upper neighbour gets the last
    owned plane of UP_FIELDS into its lower ghost.
    """
    ops = []
    if s.rank < s.ranks - 1:
        ops.append(("send", s.rank + 1, [planes(n, s.last_owned) for n in UP_FIELDS]))
        ops.append(("recv", s.rank + 1, [planes(n, s.nx_local - 1) for n in DOWN_FIELDS]))
    if s.rank > 0:
        ops.append(("send", s.rank - 1, [planes(n, s.first_owned) for n in DOWN_FIELDS]))
        ops.append(("recv", s.rank - 1, [planes(n, 0) for n in UP_FIELDS]))
    for kind, peer, ts in ops:
        (send if kind == "send" else recv)(peer, ts)


def dist_transport(group=None):
    """send/recv over torch.distributed.  The operations of one exchange are
    collected and posted as one batch (``batch_isend_irecv``: one NCCL group on
    GPUs, so the paired sends and receives of two ranks cannot wait on each
    other), then completed by ``wait``; returns (send, recv, wait)."""
    import torch.distributed as dist

    ops = []

    def send(peer, ts):
        for t in ts:
            ops.append(dist.P2POp(dist.isend, t.contiguous(), peer, group=group))

    def recv(peer, ts):
        for t in ts:
            ops.append(dist.P2POp(dist.irecv, t, peer, group=group))

    def wait():
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
            ops.clear()

    return send, recv, wait


def local_exchange(slabs: Sequence[SlabLocal], planes_of) -> None:
    """Ghost exchange between slabs held by one process: planes_of(rank)(name,
    local_i) gives each slab's plane views; copies go straight into the ghosts."""
    for s in slabs:
        up = s.rank + 1
        if up < s.ranks:
            t = slabs[up]
            src, dst = planes_of(s.rank), planes_of(up)
            for n in UP_FIELDS:
                _copy(dst(n, 0), src(n, s.last_owned))
            for n in DOWN_FIELDS:
                _copy(src(n, s.nx_local - 1), dst(n, t.first_owned))


def _copy(dst, src):
    if hasattr(dst, "copy_"):
        dst.copy_(src)
    else:
        dst[...] = src


class SlabFDTD:
    """This rank's slab of an x-decomposed grid, one rank per GPU.

    ``torch.distributed`` must be initialised (NCCL for GPUs); rank r of the
    group holds slab r of ``partition(shape[0], world, npml)`` on its current
    CUDA device.  The API follows ``CUDAFDTD`` for what a slab supports:
    ``set_epsilon`` (the whole grid's εr; each rank takes its planes),
    ``add_source`` (callbacks get the slab engine, whose ``add_source_Jx`` /
    ``add_source_Ex`` take global indices), ``step`` / ``run`` (one local step,
    then the ghost exchange), and ``gather(name)`` (the whole field on rank 0).
    Every rank calls every method in the same order.
    """

    def __init__(self, shape, dl, npml=20, dtype=None, *, courant=None, group=None,
                 fused=True):
        import numpy as np
        import torch
        import torch.distributed as dist

        from .engine import CUDAFDTD

        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.slab = partition(int(shape[0]), self.world, int(npml))[self.rank]
        self.engine = CUDAFDTD(shape, dl, npml=npml, dtype=np.float32 if dtype is None else dtype,
                               courant=courant, device=torch.cuda.current_device(),
                               fused=fused, slab=self.slab)
        self._send, self._recv, self._wait = dist_transport(group)

    def set_epsilon(self, eps, sigma_array=None):
        self.engine.set_epsilon(eps, sigma_array=sigma_array)

    def add_source(self, cb):
        return self.engine.add_source(cb)

    def add_monitor(self, cb):
        return self.engine.add_monitor(cb)

    @property
    def t(self):
        return self.engine.t

    @property
    def dt(self):
        return self.engine.dt

    def _plane(self, name, i):
        return self.engine.field_tensor(name)[i]

    def step(self):
        self.engine.step()
        exchange_ghosts(self.slab, self._plane, self._send, self._recv)
        self._wait()

    def run(self, n_steps):
        for _ in range(int(n_steps)):
            self.step()

    def gather(self, name):
        """Field ``name`` of the whole grid as a host array on rank 0 (None on the
        others): every rank sends its owned planes."""
        import torch
        import torch.distributed as dist

        own = self.engine.field_tensor(name)[self.slab.owned].contiguous()
        sizes = [s.g1 - s.g0 for s in partition(self.slab.nx, self.world, self.slab.npml)]
        if self.rank == 0:
            parts = [own] + [torch.empty((n,) + tuple(own.shape[1:]), dtype=own.dtype,
                                         device=own.device) for n in sizes[1:]]
            for r in range(1, self.world):
                dist.recv(parts[r], r, group=self.group)
            return torch.cat(parts).cpu().numpy()
        dist.send(own, 0, group=self.group)
        return None
