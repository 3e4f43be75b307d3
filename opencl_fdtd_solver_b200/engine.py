"""``CUDAFDTD``: the reference ``OpenCLFDTD`` API on hand-written sm_100a kernels.

Reference contract (``opencl_fdtd_solver/engine.py``):

* constructor, dt, dtype attributes, memory check: ``engine.py:99-210, 320-363``
* ``set_epsilon(eps, sigma_array=None)``: ``engine.py:212-254``
* ``add_source_Jx`` / ``add_source_Ex``: ``engine.py:448-538``
* ``step`` / ``run`` (H → sources at t+dt/2 → E → t+=dt → monitors): ``engine.py:724-744``
* host field reads ``Ex…Hz`` and ``read_point``: ``engine.py:746-789``; sub-box reads
  (``read_region``, ``read_plane``, ``host_window``) move only the cells a host
  monitor needs (``fdtd_read_regions``)

Design.  Torch tensors own every device buffer; the kernels are reached only
through the C ABI of ``libfdtd_b200.so`` (``_capi.py``).  A step normally runs as
one fused kernel (``fdtd_step``): source callbacks are executed *before* the
launch, with ``t`` at the half step, and their ``add_source_*`` calls are
recorded and applied in the kernel to ``E^n`` ahead of the E update, which is
exactly the reference ordering (H^{n+½} never depends on the injection).  If a
source callback touches field state (any field property or view), the engine
first materialises ``H^{n+½}`` with the split H kernel, applies the recorded
injections, and finishes the step with the split E kernel — so arbitrary
callbacks see the same state they would see in the reference.  GPU plane DFT
monitors registered on the engine are accumulated in the E epilogue.

Only CUDA runs the path: without a device or without the built library the
constructor raises.
"""

from __future__ import annotations

import contextlib
import ctypes
import logging
import warnings
from typing import Sequence

import numpy as np

from . import _capi as capi
from .constants import C0, EPS0, MU0
from .cpml import build_cpml_profiles, inverse_kappa_dl
from .plugin import SourceMonitorMixin, register_backend

log = logging.getLogger(__name__)

FIELD_NAMES = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
REFERENCE_COURANT = 0.99 / np.sqrt(3.0)


def _torch():
    import torch

    return torch


class CUDAFDTD(SourceMonitorMixin):
    """3-D Yee FDTD with CFS-CPML on one CUDA device (drop-in for ``OpenCLFDTD``)."""

    MEMORY_HEADROOM_FRACTION = 0.12
    MEMORY_HEADROOM_BYTES = 512 * 1024 * 1024

    def __init__(self, shape, dl, npml=20, dtype=np.float32, ctx=None, queue=None,
                 accum_fp64=False, *, courant=None, device=None, fused=True, slab=None):
        """
        shape : (Nx, Ny, Nz) Yee cells
        dl    : uniform cell size in metres
        npml  : CPML thickness in cells (0 disables the PML)
        dtype : ``np.float32`` (default) or ``np.float64``
        ctx, queue : accepted for signature compatibility; ``queue`` may be a
            ``torch.cuda.Stream`` to launch on, ``ctx`` an object whose
            ``devices[0].global_mem_size`` is used for the memory budget
        accum_fp64 : kept for API compatibility; GPU DFT accumulators are always
            float64, and host downloads are returned in ``accreal_complex_dtype``
        courant : Courant number S (dt = S·dl/c); default is the reference's
            fixed 0.99/√3
        device : CUDA device (index, string or ``torch.device``); default current
        fused : run steps with the single-pass kernel when the shape allows it
        slab  : a ``slabs.SlabLocal``: run one x-slab of the grid ``shape`` (its
            planes plus ghost planes, ``Nx`` = the local plane count, the x-CPML
            only on global faces).  ``set_epsilon`` then takes the whole grid's
            εr and sheets take global i indices; field reads return the local
            planes.  ``slabs.SlabFDTD`` drives one slab per rank.
        """
        self.global_shape = tuple(int(v) for v in shape)
        self.Nx, self.Ny, self.Nz = self.global_shape
        self.slab = slab
        self.x0 = 0  # global index of local plane 0
        if slab is not None:
            if slab.nx != self.Nx or slab.npml != int(npml):
                raise ValueError(f"slab {slab} does not belong to shape {shape} / npml {npml}")
            self.Nx, self.x0 = slab.nx_local, slab.l0
        self.dl = float(dl)
        self.npml = int(npml)
        dtype = np.dtype(dtype)
        if dtype not in (np.dtype(np.float32), np.dtype(np.float64)):
            raise ValueError(f"CUDAFDTD supports float32 or float64 computation; got {dtype!r}")
        if min(self.Nx, self.Ny, self.Nz) <= 0:
            raise ValueError(f"shape must be positive, got {tuple(shape)}")
        if self.npml < 0:
            raise ValueError(f"npml must be >= 0, got {npml}")
        self.dtype = dtype
        self.real = np.float32 if dtype == np.float32 else np.float64
        self.complex_dtype = np.dtype(np.complex64 if dtype == np.float32 else np.complex128)
        self.accum_fp64 = bool(accum_fp64) or dtype == np.float64
        self.accreal = np.float64 if self.accum_fp64 else self.real
        self.accreal_complex_dtype = (np.dtype(np.complex128) if self.accum_fp64
                                      else self.complex_dtype)
        self.t = 0.0
        self.step_num = 0
        if courant is None:
            self.courant = float(REFERENCE_COURANT)
            self.dt = 0.99 * dl / (C0 * np.sqrt(3.0))  # reference engine.py:138
        else:
            self.courant = float(courant)
            if not (0.0 < self.courant <= 1.0 / np.sqrt(3.0) + 1e-12):
                raise ValueError(f"courant must be in (0, 1/sqrt(3)], got {courant}")
            self.dt = self.courant * self.dl / C0
        self.size = self.Nx * self.Ny * self.Nz
        n = self.npml
        self._pml_x = (n, n) if slab is None else (slab.pml_lo, slab.pml_hi)
        self.psi_x_size = sum(self._pml_x) * self.Ny * self.Nz if n > 0 else 0
        self.psi_y_size = self.Nx * 2 * n * self.Nz if n > 0 else 0
        self.psi_z_size = self.Nx * self.Ny * 2 * n if n > 0 else 0
        self.ctx = ctx
        self._sources = []
        self._monitors = []
        self._fused_enabled = bool(fused)
        self._read_window = None    # boxes served by Ex…Hz inside host_window()
        self._mirror = {}           # field name -> full-shape host array (windowed reads)
        self._hostio = None         # (device staging, pinned host) buffers of fdtd_read_regions

        mem_device = ctx.devices[0] if (ctx is not None and hasattr(ctx, "devices")) else None
        torch = _torch()
        if mem_device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("No CUDA device available for CUDAFDTD.")
            self.device = torch.device("cuda", torch.cuda.current_device()
                                       if device is None else torch.device(device).index or 0)
            mem_device = torch.cuda.get_device_properties(self.device)
        else:
            self.device = None
        self._check_device_memory((self.Nx, self.Ny, self.Nz), n, dtype, mem_device)
        if self.device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("No CUDA device available for CUDAFDTD.")
            self.device = torch.device("cuda", torch.cuda.current_device())
        capi.lib()  # fail loudly if the extension is missing
        self.queue = queue if isinstance(queue, torch.cuda.Stream) else \
            torch.cuda.current_stream(self.device)
        log.info("CUDA FDTD Solver initialized on device: %s (dtype=%s)",
                 torch.cuda.get_device_name(self.device), self.dtype.name)
        self._alloc()
        self._build_cpml()
        self._build_structs()

    # ------------------------------------------------------------------ memory
    @staticmethod
    def estimate_device_memory_bytes(shape, npml, dtype=np.float32):
        """Reference estimate: 6 fields + 3 ``ce`` arrays + face ψ (``engine.py:320-334``)."""
        nx, ny, nz = shape
        item = np.dtype(dtype).itemsize
        fields = 9 * nx * ny * nz * item
        if npml <= 0:
            return fields
        psi = (4 * (2 * npml * ny * nz) + 4 * (nx * 2 * npml * nz)
               + 4 * (nx * ny * 2 * npml)) * item
        return fields + psi

    @staticmethod
    def device_footprint_bytes(shape, npml, dtype=np.float32, *, lossy=False, fused=True):
        """Bytes this engine actually allocates: fields (twice when fused, the step
        reads one set and writes the other), ``ce`` (and ``ca`` when lossy), ψ stripes."""
        nx, ny, nz = shape
        item = np.dtype(dtype).itemsize
        cells = nx * ny * nz
        arrays = 6 * (2 if fused else 1) + 3 + (3 if lossy else 0)
        psi_one = 0
        if npml > 0:
            psi_one = 2 * (2 * npml * ny * nz + nx * 2 * npml * nz + nx * ny * 2 * npml)
        return (arrays * cells + psi_one * 2) * item

    @classmethod
    def device_memory_budget_bytes(cls, device):
        """Usable device bytes after the reserved headroom (``engine.py:336-344``)."""
        if hasattr(device, "global_mem_size"):
            total = int(device.global_mem_size)
        elif hasattr(device, "total_memory"):
            total = int(device.total_memory)
        else:
            total = int(_torch().cuda.get_device_properties(device).total_memory)
        reserve = max(int(total * cls.MEMORY_HEADROOM_FRACTION), int(cls.MEMORY_HEADROOM_BYTES))
        return max(0, total - reserve)

    def _check_device_memory(self, shape, npml, dtype, device):
        needed = max(self.estimate_device_memory_bytes(shape, npml, dtype),
                     self.device_footprint_bytes(shape, npml, dtype, fused=self._fused_enabled))
        budget = self.device_memory_budget_bytes(device)
        if needed > budget:
            total = int(getattr(device, "global_mem_size", getattr(device, "total_memory", 0)))
            name = getattr(device, "name", "device")
            raise MemoryError(
                f"Model needs ~{needed / 1024**3:.2f} GB device memory, but {name} only has "
                f"~{budget / 1024**3:.2f} GB usable ({total / 1024**3:.2f} GB total minus "
                f"headroom). Reduce the grid or npml.")

    # ------------------------------------------------------------- allocation
    def _alloc(self):
        torch = _torch()
        tdt = torch.float32 if self.dtype == np.float32 else torch.float64
        self._tdt = tdt
        shp = (self.Nx, self.Ny, self.Nz)
        dev = self.device
        with torch.cuda.stream(self.queue):
            z = lambda s: torch.zeros(s, dtype=tdt, device=dev)  # noqa: E731
            self._E = [z(shp) for _ in range(3)]
            self._H = [z(shp) for _ in range(3)]
            if self._fused_enabled:
                self._En = [torch.empty(shp, dtype=tdt, device=dev) for _ in range(3)]
                self._Hn = [torch.empty(shp, dtype=tdt, device=dev) for _ in range(3)]
            else:
                self._En = self._Hn = None
            vac = self.real(self.dt / EPS0)
            self._ce = [torch.full(shp, float(vac), dtype=tdt, device=dev) for _ in range(3)]
            self._ca = None
        self.lossy = False
        self._parity = 0

    def _build_cpml(self):
        torch = _torch()
        n = self.npml
        prof = build_cpml_profiles(self.global_shape, npml=n, dl=self.dl, dt=self.dt,
                                   dtype=self.dtype)
        self.cpml_profiles = prof
        up = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)  # noqa: E731
        xs = slice(self.x0, self.x0 + self.Nx)  # a slab's planes of the x profiles
        self._cp = {}
        for stag, axes in (("h", prof.h), ("e", prof.e)):
            self._cp[stag] = [(up(p.b[xs] if a == 0 else p.b), up(p.c[xs] if a == 0 else p.c),
                               up(inverse_kappa_dl(p.kappa[xs] if a == 0 else p.kappa, self.dl,
                                                   self.dtype)))
                              for a, p in enumerate(axes)]
        nx, ny, nz = self.Nx, self.Ny, self.Nz
        sx, sy, sz = (sum(self._pml_x), ny, nz), (nx, 2 * n, nz), (nx, ny, 2 * n)
        if n == 0:
            sx = sy = sz = (1,)
        if sx[0] == 0:
            sx = (1,)  # a slab without x-CPML faces: the stripe is never indexed
        mk = lambda s: torch.zeros(s, dtype=self._tdt, device=self.device)  # noqa: E731
        order = (sy, sz, sx, sz, sx, sy)  # Hx_y, Hx_z, Hy_x, Hy_z, Hz_x, Hz_y / E likewise
        with torch.cuda.stream(self.queue):
            self._psi_h = [mk(s) for s in order]
            self._psi_e = [mk(s) for s in order]

    def _build_structs(self):
        g = capi.Grid()
        g.nx, g.ny, g.nz, g.npml = self.Nx, self.Ny, self.Nz, self.npml
        g.dtype = capi.FDTD_F32 if self.dtype == np.float32 else capi.FDTD_F64
        if self.slab is not None:
            g.x_slab = 1
            g.pml_x_lo, g.pml_x_hi = self._pml_x
            g.ghost_lo, g.ghost_hi = self.slab.ghost_lo, self.slab.ghost_hi
        g.lossy = 1 if self.lossy else 0
        g.dtm = self.dt / MU0
        g.dtm_dl = self.dt / (MU0 * self.dl)
        g.inv_dl = 1.0 / self.dl
        self._grid = g
        cp = capi.Cpml()
        for a in range(3):
            for stag, (bn, cn, kn) in (("h", ("b_h", "c_h", "ik_h")), ("e", ("b_e", "c_e", "ik_e"))):
                b, c, ik = self._cp[stag][a]
                getattr(cp, bn)[a] = b.data_ptr()
                getattr(cp, cn)[a] = c.data_ptr()
                getattr(cp, kn)[a] = ik.data_ptr()
        self._cpml_base = cp
        self._refresh_structs()

    def _refresh_structs(self):
        self._fields_by_parity = {}
        self._build_fields()
        cp = capi.Cpml.from_buffer_copy(self._cpml_base)
        for q in range(6):
            cp.psi_h[q] = self._psi_h[q].data_ptr()
            cp.psi_e[q] = self._psi_e[q].data_ptr()
        self._cpml = cp
        self._grid.lossy = 1 if self.lossy else 0

    def _build_fields(self):
        cached = self._fields_by_parity.get(self._parity)
        if cached is not None:
            self._fields = cached
            return
        f = capi.Fields()
        for a in range(3):
            f.E[a] = self._E[a].data_ptr()
            f.H[a] = self._H[a].data_ptr()
            f.ce[a] = self._ce[a].data_ptr()
            if self._ca is not None:
                f.ca[a] = self._ca[a].data_ptr()
            if self._En is not None:
                f.E_next[a] = self._En[a].data_ptr()
                f.H_next[a] = self._Hn[a].data_ptr()
        self._fields = f
        self._fields_by_parity[self._parity] = f

    # -------------------------------------------------------------- materials
    def set_epsilon(self, eps_array, sigma_array=None):
        """Cell-centred εr (and optional σ in S/m) → Yee-edge ``ce`` (and ``ca``).

        The arrays are uploaded once and the edge average and coefficients are
        computed on the device in float64 (``fdtd_set_epsilon``), with the same
        operations as the reference host math (``materials.py:28-88``), so the
        rounded coefficients are identical to ``yee_edge_ce`` / ``yee_edge_ca_cb``.
        """
        torch = _torch()
        expected = self.global_shape
        if tuple(np.shape(eps_array)) != expected:
            raise ValueError(
                f"Epsilon shape mismatch: expected {expected}, got {tuple(np.shape(eps_array))}")
        if sigma_array is not None and tuple(np.shape(sigma_array)) != expected:
            raise ValueError(f"Sigma shape mismatch: expected {expected}, "
                             f"got {tuple(np.shape(sigma_array))}")
        self._materialize()
        xs = slice(self.x0, self.x0 + self.Nx)  # a slab's planes (ghosts included)
        eps = np.asarray(eps_array)[xs]
        sig = None if sigma_array is None else np.asarray(sigma_array)[xs]
        narrow = eps.dtype == np.float32 and (sig is None or sig.dtype == np.float32)
        src = np.float32 if narrow else np.float64
        with torch.cuda.stream(self.queue):
            eps_d = torch.from_numpy(np.ascontiguousarray(eps, dtype=src)).to(self.device)
            sig_d = None
            if sig is not None:
                sig_d = torch.from_numpy(np.ascontiguousarray(sig, dtype=src)).to(self.device)
                if self._ca is None:
                    self._ca = [torch.empty_like(c) for c in self._ce]
            ce = (ctypes.c_void_p * 3)(*[c.data_ptr() for c in self._ce])
            ca = (ctypes.c_void_p * 3)(*([c.data_ptr() for c in self._ca] if sig_d is not None
                                         else [None, None, None]))
            capi.run("fdtd_set_epsilon", self._grid, eps_d.data_ptr(),
                     None if sig_d is None else sig_d.data_ptr(),
                     capi.FDTD_F32 if narrow else capi.FDTD_F64, float(self.dt), float(EPS0),
                     ce, ca, self.queue.cuda_stream)
            if sig_d is None:
                self._ca = None
            self.lossy = sig_d is not None
            del eps_d, sig_d
        self._refresh_structs()

    # ---------------------------------------------------------------- sources
    def _sheet(self, i0, i1, j0, j1):
        """Sheet bounds in local indices (a slab shifts global i by its first plane;
        the kernels apply the sheet to local cells only, rim weights still at the
        sheet's own edges)."""
        i0 = 0 if i0 is None else int(i0)
        i1 = self.global_shape[0] if i1 is None else int(i1)
        return (i0 - self.x0, i1 - self.x0,
                0 if j0 is None else int(j0), self.Ny if j1 is None else int(j1))

    def add_source_Ex(self, z_src, amp, i0=None, i1=None, j0=None, j1=None):
        """Legacy soft add of ``amp`` onto an Ex sheet (``engine.py:448-480``)."""
        warnings.warn(
            "add_source_Ex is a legacy Ex soft-add; prefer add_source_Jx for SI current density",
            DeprecationWarning, stacklevel=2)
        i0, i1, j0, j1 = self._sheet(i0, i1, j0, j1)
        s = capi.Source(kind=capi.FDTD_SRC_EX, z=int(z_src), i0=i0, i1=i1, j0=j0, j1=j1,
                        rim_taper=0, amp=float(amp), rim_edge=0.0)
        self._inject(s)

    def add_source_Jx(self, z_src, Jx, i0=None, i1=None, j0=None, j1=None, *,
                      rim_taper=False, rim_edge=0.8, rim_renorm=True):
        """SI current density ``Jx`` on a constant-z sheet: ``Ex += −dt/(ε0 εr)·Jx·w``
        (``engine.py:482-538``).  ``rim_taper`` weights edges by ``rim_edge`` and corners
        by its square; ``rim_renorm`` rescales ``Jx`` so the weights sum to the cell count."""
        i0, i1, j0, j1 = self._sheet(i0, i1, j0, j1)
        jx = float(Jx)
        re = float(rim_edge)
        if rim_taper and rim_renorm:
            nxs, nys = max(0, i1 - i0), max(0, j1 - j0)
            if nxs >= 2 and nys >= 2:
                ni, nj = nxs - 2, nys - 2
                wsum = ni * nj + re * (2 * ni + 2 * nj) + (re * re) * 4
                jx *= (nxs * nys) / wsum
        s = capi.Source(kind=capi.FDTD_SRC_JX, z=int(z_src), i0=i0, i1=i1, j0=j0, j1=j1,
                        rim_taper=1 if rim_taper else 0, amp=jx, rim_edge=re)
        self._inject(s)

    def _inject(self, s):
        if not (0 <= s.z < self.Nz):
            raise ValueError(f"source plane z={s.z} outside [0, {self.Nz})")
        if getattr(self, "_in_source_phase", False) and not self._h_done:
            if len(self._pending) < capi.FDTD_MAX_SOURCES:
                self._pending.append(s)
                return
            self._materialize()
        self._launch_source(s)

    def _launch_source(self, s):
        capi.run("fdtd_add_source", self._grid, self._E[0].data_ptr(), self._ce[0].data_ptr(), s,
                 self.queue.cuda_stream)

    def _materialize(self):
        """Inside a source callback: run the H half step now and flush recorded
        injections, so that field state is what the reference would show."""
        if getattr(self, "_in_source_phase", False) and not self._h_done:
            capi.run("fdtd_update_H", self._grid, self._fields, self._cpml, self.queue.cuda_stream)
            self._h_done = True
            pend, self._pending = self._pending, []
            for s in pend:
                self._launch_source(s)

    # ------------------------------------------------------------------- step
    def _plane_monitors(self):
        from .monitors import CUDAPlaneDFTMonitor

        return [m for m in self._monitors if isinstance(m, CUDAPlaneDFTMonitor) and m.fdtd is self]

    def step(self):
        """One Yee step: H, sources at t+dt/2, E (+ fused plane DFTs), t += dt, monitors."""
        t_int = self.t
        self.t = t_int + 0.5 * self.dt
        self._in_source_phase = True
        self._h_done = False
        self._pending = []
        try:
            for src in self._sources:
                src(self)
        finally:
            self._in_source_phase = False
            self.t = t_int
        pend, self._pending = self._pending, []
        t_next = t_int + self.dt
        planes = self._plane_monitors()
        if len(planes) > capi.FDTD_MAX_PLANES:
            raise ValueError(f"at most {capi.FDTD_MAX_PLANES} plane DFT monitors per engine")
        pd = (capi.PlaneDft * max(1, len(planes)))()
        for q, m in enumerate(planes):
            pd[q] = m._descriptor(t_next)
        sa = (capi.Source * max(1, len(pend)))(*pend)
        st = self.queue.cuda_stream
        if self._h_done:
            capi.run("fdtd_update_E", self._grid, self._fields, self._cpml, sa, len(pend), pd,
                     len(planes), st)
        else:
            done = False
            if self._fused_enabled:
                rc = capi.call("fdtd_step", self._grid, self._fields, self._cpml, sa, len(pend),
                               pd, len(planes), st)
                if rc == capi.FDTD_OK:
                    self._swap()
                    done = True
                elif rc == capi.FDTD_ERR_UNSUPPORTED:
                    self._fused_enabled = False
                else:
                    capi.check(rc, "fdtd_step")
            if not done:
                capi.run("fdtd_update_H", self._grid, self._fields, self._cpml, st)
                capi.run("fdtd_update_E", self._grid, self._fields, self._cpml, sa, len(pend), pd,
                         len(planes), st)
        self.t += self.dt
        self.step_num += 1
        for mon in self._monitors:
            regs = getattr(mon, "host_regions", None)
            if regs is None:
                mon(self)
            else:
                with self.host_window(regs() if callable(regs) else regs):
                    mon(self)

    def _swap(self):
        self._E, self._En = self._En, self._E
        self._H, self._Hn = self._Hn, self._H
        self._parity ^= 1
        self._build_fields()

    def run(self, n_steps, progress_every=0):
        """Run ``n_steps`` steps; log progress at INFO every ``progress_every`` steps."""
        for i in range(int(n_steps)):
            self.step()
            if progress_every and i % progress_every == 0:
                log.info("  step %d/%d  t=%.3e s", i, n_steps, self.t)

    def synchronize(self):
        self.queue.synchronize()

    # ------------------------------------------------------ state snapshots
    def _state_tensors(self):
        """The tensors that carry the time-stepping state: E, H, ψ_H, ψ_E."""
        return list(self._E) + list(self._H) + list(self._psi_h) + list(self._psi_e)

    def save_state(self):
        """Device copy of the full time-stepping state (fields, ψ stripes, t, step_num)."""
        torch = _torch()
        self._materialize()
        with torch.cuda.stream(self.queue):
            tensors = [t.clone() for t in self._state_tensors()]
        return {"tensors": tensors, "t": self.t, "step_num": self.step_num}

    def load_state(self, state):
        """Restore a state taken by :meth:`save_state` on this engine."""
        torch = _torch()
        cur = self._state_tensors()
        if len(cur) != len(state["tensors"]):
            raise ValueError("state was saved from a different engine layout")
        with torch.cuda.stream(self.queue):
            for dst, src in zip(cur, state["tensors"]):
                dst.copy_(src)
        self.t = float(state["t"])
        self.step_num = int(state["step_num"])

    def reset_state(self):
        """Zero the fields and ψ stripes and rewind to t = 0 (coefficients kept)."""
        torch = _torch()
        with torch.cuda.stream(self.queue):
            for t in self._state_tensors():
                t.zero_()
        self.t = 0.0
        self.step_num = 0

    # ----------------------------------------------------------- field access
    def field_tensor(self, name):
        """Current device tensor of field ``name`` (``'Ex'`` … ``'Hz'``), shape (Nx, Ny, Nz)."""
        self._materialize()
        k = FIELD_NAMES.index(name)
        return self._E[k] if k < 3 else self._H[k - 3]

    def _read_field(self, name):
        if self._read_window is not None:
            return self._window_read(name, self._read_window)
        t = self.field_tensor(name)
        self.queue.synchronize()
        return t.cpu().numpy()

    # ---------------------------------------------------- sub-box host reads
    def _norm_regions(self, regions):
        """Validated half-open boxes ``((i0, i1), (j0, j1), (k0, k1))``."""
        dims = (self.Nx, self.Ny, self.Nz)
        out = []
        for r in regions:
            box = tuple((int(a), int(b)) for a, b in r)
            if len(box) != 3 or any(not 0 <= a <= b <= n for (a, b), n in zip(box, dims)):
                raise ValueError(f"region {r!r} is not a half-open box inside {dims}")
            out.append(box)
        return out

    def _gather(self, name, boxes):
        """Host views of ``boxes`` of field ``name``, valid until the next gather.

        One ``fdtd_read_regions`` call (one gather launch plus one device-to-host
        copy into a pinned buffer) per ``FDTD_MAX_REGIONS`` boxes, then one stream
        synchronisation.
        """
        torch = _torch()
        t = self.field_tensor(name)
        sizes = [(i1 - i0) * (j1 - j0) * (k1 - k0) for (i0, i1), (j0, j1), (k0, k1) in boxes]
        total = int(sum(sizes))
        if self._hostio is None or self._hostio[0].numel() < total:
            n = 1 << max(16, (max(total, 1) - 1).bit_length())
            with torch.cuda.stream(self.queue):
                dev = torch.empty(n, dtype=t.dtype, device=self.device)
            self._hostio = (dev, torch.empty(n, dtype=t.dtype, pin_memory=True))
        dev, pin = self._hostio
        item = t.element_size()
        dt = capi.FDTD_F64 if self.dtype == np.float64 else capi.FDTD_F32
        off = 0
        for c in range(0, len(boxes), capi.FDTD_MAX_REGIONS):
            chunk = boxes[c:c + capi.FDTD_MAX_REGIONS]
            regs = (capi.Region * len(chunk))()
            for q, box in enumerate(chunk):
                regs[q].lo[:] = [a for a, _ in box]
                regs[q].hi[:] = [b for _, b in box]
            capi.run("fdtd_read_regions", t.data_ptr(), dt, self.Nx, self.Ny, self.Nz, regs,
                     len(chunk), dev.data_ptr() + off * item, pin.data_ptr() + off * item,
                     self.queue.cuda_stream)
            off += sum(sizes[c:c + capi.FDTD_MAX_REGIONS])
        self.queue.synchronize()
        flat = pin.numpy()
        out, off = [], 0
        for box, n in zip(boxes, sizes):
            out.append(flat[off:off + n].reshape([b - a for a, b in box]))
            off += n
        return out

    def read_region(self, name, lo, hi):
        """Host copy of field ``name`` over the half-open box ``[lo, hi)``.

        Only the box crosses to the host (gathered on the device, then one copy
        through pinned memory), instead of the whole volume that the ``Ex…Hz``
        properties move (``engine.py:747-751``).
        """
        FIELD_NAMES.index(name)
        box = self._norm_regions([tuple(zip(lo, hi))])
        return self._gather(name, box)[0].copy()

    def read_plane(self, name, axis, index):
        """Host copy of one plane of field ``name``: ``axis`` in ``'x'``/``'y'``/``'z'`` or 0-2."""
        a = {"x": 0, "y": 1, "z": 2}.get(axis, axis)
        if a not in (0, 1, 2):
            raise ValueError(f"axis must be x, y, z or 0-2, got {axis!r}")
        dims = (self.Nx, self.Ny, self.Nz)
        index = int(index)
        if not 0 <= index < dims[a]:
            raise ValueError(f"plane index {index} outside [0, {dims[a]})")
        lo = [0, 0, 0]
        hi = list(dims)
        lo[a], hi[a] = index, index + 1
        return self.read_region(name, lo, hi).reshape([d for q, d in enumerate(dims) if q != a])

    def _window_read(self, name, boxes):
        mirror = self._mirror.get(name)
        if mirror is None:
            mirror = self._mirror[name] = np.zeros((self.Nx, self.Ny, self.Nz), self.dtype)
        for box, part in zip(boxes, self._gather(name, boxes)):
            mirror[tuple(slice(a, b) for a, b in box)] = part
        view = mirror.view()
        view.flags.writeable = False
        return view

    @contextlib.contextmanager
    def host_window(self, regions):
        """Serve ``Ex…Hz`` reads inside the block from the listed boxes only.

        ``regions`` is a list of half-open boxes ``((i0, i1), (j0, j1), (k0, k1))``.
        Within the block a field property returns a read-only ``(Nx, Ny, Nz)``
        array that holds the current values inside the boxes (values elsewhere
        are unspecified), and only the boxes cross to the host.  ``step()`` opens
        this window around each monitor that declares ``host_regions`` (a list of
        boxes, or a callable returning one), so a host monitor that reads a few
        planes per step moves those planes rather than six volumes.  Reads
        outside the block are full reads again.
        """
        boxes = self._norm_regions(regions)
        prev, self._read_window = self._read_window, boxes
        try:
            yield self
        finally:
            self._read_window = prev

    def _write_field(self, name, value):
        torch = _torch()
        arr = np.asarray(value, dtype=self.dtype)
        if arr.shape != (self.Nx, self.Ny, self.Nz):
            raise ValueError(f"{name} shape mismatch: expected {(self.Nx, self.Ny, self.Nz)}, "
                             f"got {arr.shape}")
        t = self.field_tensor(name)
        with torch.cuda.stream(self.queue):
            t.copy_(torch.from_numpy(np.ascontiguousarray(arr)))
        self.queue.synchronize()

    def read_point(self, field_name, i, j, k):
        """Single cell value (``engine.py:753-765``)."""
        t = self.field_tensor(field_name)
        self.queue.synchronize()
        return float(t[int(i), int(j), int(k)].item())

    def coefficient_tensors(self):
        """``{'ce': [x, y, z], 'ca': [x, y, z] or None}`` device tensors."""
        return {"ce": list(self._ce), "ca": None if self._ca is None else list(self._ca)}


def _field_property(name):
    def getter(self):
        return self._read_field(name)

    def setter(self, value):
        self._write_field(name, value)

    return property(getter, setter, doc=f"Host copy of {name} (Nx, Ny, Nz); assignment uploads.")


def _tensor_property(name):
    return property(lambda self: self.field_tensor(name),
                    doc=f"Device tensor of {name} (zero-copy; valid until the next step).")


for _n in FIELD_NAMES:
    setattr(CUDAFDTD, _n, _field_property(_n))
    setattr(CUDAFDTD, _n + "_t", _tensor_property(_n))

register_backend("cuda", CUDAFDTD)
