"""GPU DFT monitors for ``CUDAFDTD``.

``CUDANear2FarMonitor`` keeps the surface of the reference ``OpenCLNear2FarMonitor``
(``opencl_fdtd_solver/monitors.py:383-804``): box snapping (``:37-45``), packed faces
x0,x1,y0,y1,z0,z1 (``:396-412``), per-step phase recurrence (``:456-459, 571-584``),
``get_farfield(s)`` (``:644-735``), ``farfield_polar_xz`` (``:737-755``),
``snapshot_dft`` / ``dft_relative_change`` (``:487-569``) and ``fetch_dft_fields``
(``:757-804``).  It additionally accepts a list of frequencies (one accumulator
slice per frequency); a scalar ``freq`` keeps the reference form.  Far fields use
the reference kernel's sign ``η·N⊥ − r̂×L`` (``dft_farfield.cl:617``).

``NumPyNear2FarMonitor`` is the reference's host monitor (``monitors.py:186-380``):
it accumulates from the engine's host field reads, which ``CUDAFDTD`` restricts
to the face slabs the monitor declares.

``CUDAPlaneDFTMonitor`` has no reference class: a running DFT of chosen field
components on one grid plane, accumulated inside the E-update kernel (no extra
pass over the fields), with the same phase convention (E at the step time, H half
a step earlier).

Accumulators are complex128 on the device; the phase recurrence is evaluated on
the host in complex128 exactly as the reference does and uploaded in chunks.
"""

from __future__ import annotations

import numpy as np

from . import _capi as capi
from .constants import C0, ETA0

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
_PHASE_CHUNK = 512


def _torch():
    import torch

    return torch


def _box_struct(box, offsets, n_face, nfreq):
    b = capi.Box()
    b.ix0, b.ix1, b.iy0, b.iy1, b.iz0, b.iz1 = box
    for q in range(6):
        b.off[q] = offsets[q]
    b.n_face = n_face
    b.nfreq = nfreq
    return b


def _device_farfields(fdtd, cbox, acc, fi, freq, pts):
    """Far E, H ``(n_obs, 6)`` complex128 from face accumulators ``acc`` (device,
    ``(6, nfreq, n_face, 2)`` float64) with the float64 surface-sum kernel."""
    torch = _torch()
    n_obs = int(pts.shape[0])
    q = fdtd.queue
    with torch.cuda.stream(q):
        obs = torch.from_numpy(pts.astype(np.float64)).to(fdtd.device)
        nl = torch.empty((n_obs, 6, 2), dtype=torch.float64, device=fdtd.device)
        eh = torch.empty((n_obs, 6, 2), dtype=torch.float64, device=fdtd.device)
    k_wave = 2.0 * np.pi * freq / C0
    capi.run("fdtd_farfield", cbox, acc.data_ptr(), int(fi), float(fdtd.dl), k_wave, float(ETA0),
             obs.data_ptr(), n_obs, nl.data_ptr(), eh.data_ptr(), q.cuda_stream)
    q.synchronize()
    h = eh.cpu().numpy()
    return (h[..., 0] + 1j * h[..., 1]).astype(np.complex128)


def _obs_array(obs_points, dtype):
    pts = np.asarray(obs_points, dtype=dtype)
    if pts.ndim == 1:
        pts = pts.reshape(1, 3)
    if pts.ndim != 2 or pts.shape[1] != 3:
        raise ValueError("obs_points must be (n,3) or (3,)")
    return pts


class _PhaseTable:
    """Device table of the per-step phases ``[chunk][nfreq][4]`` (E re, E im, H re, H im).

    The first call uses ``e^{jωt}·dt``; later calls multiply by ``e^{jωdt}``
    (reference ``monitors.py:571-577``), computed ahead a chunk at a time.  Each
    chunk goes up through one of two pinned host buffers with an asynchronous
    copy on the engine's stream into one of two device tables, so refilling
    never waits for the device to catch up with the host; a pinned buffer is
    refilled only after its previous copy completed (an event), and a device
    table is overwritten in stream order after the steps that read it.  Without
    a stream the table stays on the host (the phase sequence alone).
    """

    def __init__(self, freqs, dt, device, stream=None):
        self.omega = 2.0 * np.pi * np.asarray(freqs, dtype=np.float64)
        self.dt = float(dt)
        self.dphase = np.exp(1j * self.omega * self.dt)
        self.half = np.exp(-0.5j * self.omega * self.dt)
        self.device = device
        self.stream = stream
        self.phase = None  # host value of the most recent step (complex128 [nfreq])
        self._pin = self._dev_tabs = self._done = None
        self._dev = None
        self._slot = 1
        self._cursor = 0

    def _fill(self, first):
        torch = _torch()
        nf = self.omega.size
        if self.stream is None:  # host-only table (no device upload)
            self._seq = self._sequence(first)
            self._dev = torch.zeros(1)
            self._cursor = 0
            return
        if self._pin is None:
            shape = (_PHASE_CHUNK, nf, 4)
            self._pin = [torch.empty(shape, dtype=torch.float64, pin_memory=True)
                         for _ in range(2)]
            with torch.cuda.stream(self.stream):
                self._dev_tabs = [torch.empty(shape, dtype=torch.float64, device=self.device)
                                  for _ in range(2)]
            self._done = [None, None]
        seq = self._sequence(first)
        ph = seq * self.half
        self._slot ^= 1
        b = self._slot
        if self._done[b] is not None:
            self._done[b].synchronize()  # the copy from this pinned buffer has landed
        host = self._pin[b].numpy()
        host[:, :, 0], host[:, :, 1] = seq.real, seq.imag
        host[:, :, 2], host[:, :, 3] = ph.real, ph.imag
        self._seq = seq
        with torch.cuda.stream(self.stream):
            self._dev_tabs[b].copy_(self._pin[b], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
        self._done[b] = ev
        self._dev = self._dev_tabs[b]
        self._cursor = 0

    def _sequence(self, first):
        p = first
        seq = np.empty((_PHASE_CHUNK, self.omega.size), np.complex128)
        for s in range(_PHASE_CHUNK):
            if s > 0:
                p = p * self.dphase
            seq[s] = p
        return seq

    def next_ptr(self, t):
        """Advance one step (monitor time ``t``) and return the device pointer of its phases."""
        if self._dev is None:
            self._fill(np.exp(1j * self.omega * t) * self.dt)
        elif self._cursor >= _PHASE_CHUNK:
            self._fill(self._seq[-1] * self.dphase)
        s = self._cursor
        self.phase = self._seq[s]
        self._cursor += 1
        return self._dev.data_ptr() + s * self.omega.size * 4 * 8


class CUDAPlaneDFTMonitor:
    """Running DFT of ``components`` on the plane ``axis = index`` at ``freqs``.

    ``axis`` is 0/1/2 or ``'x'/'y'/'z'``.  Accumulated in the E-update kernel; the
    result ``dft(c)`` has shape ``(n_freq, n1, n2)`` over the two other axes in
    C order.  Registers itself on ``fdtd`` (at most four per engine).
    """

    def __init__(self, fdtd, axis, index, freqs, components=("Ex",)):
        torch = _torch()
        self.fdtd = fdtd
        self.axis = {"x": 0, "y": 1, "z": 2}.get(axis, axis)
        if self.axis not in (0, 1, 2):
            raise ValueError(f"axis must be 0, 1, 2 or 'x', 'y', 'z'; got {axis!r}")
        dims = [fdtd.Nx, fdtd.Ny, fdtd.Nz]
        self.index = int(index)
        if not 0 <= self.index < dims[self.axis]:
            raise ValueError(f"plane index {index} outside [0, {dims[self.axis]})")
        self.freqs = np.atleast_1d(np.asarray(freqs, dtype=np.float64))
        if not 0 < self.freqs.size <= capi.FDTD_MAX_FREQS:
            raise ValueError(f"1 to {capi.FDTD_MAX_FREQS} frequencies, got {self.freqs.size}")
        comps = (components,) if isinstance(components, str) else tuple(components)
        for c in comps:
            if c not in FIELDS:
                raise ValueError(f"unknown component {c!r}")
        # stored in Ex..Hz order (the kernel's slot order)
        self.components = tuple(c for c in FIELDS if c in comps)
        self.comp_mask = sum(1 << FIELDS.index(c) for c in self.components)
        del dims[self.axis]
        self.plane_shape = tuple(dims)
        with torch.cuda.stream(fdtd.queue):
            self.acc = torch.zeros((len(self.components), self.freqs.size, *dims, 2),
                                   dtype=torch.float64, device=fdtd.device)
        self._phases = _PhaseTable(self.freqs, fdtd.dt, fdtd.device, fdtd.queue)
        n_planes = sum(1 for m in fdtd._monitors if isinstance(m, CUDAPlaneDFTMonitor))
        if n_planes >= capi.FDTD_MAX_PLANES:
            raise ValueError(f"at most {capi.FDTD_MAX_PLANES} plane DFT monitors per engine")
        fdtd.add_monitor(self)

    @property
    def _phase(self):
        return self._phases.phase

    def _descriptor(self, t_next):
        d = capi.PlaneDft()
        d.axis, d.index, d.comp_mask, d.nfreq = self.axis, self.index, self.comp_mask, \
            self.freqs.size
        d.acc = self.acc.data_ptr()
        d.phase = self._phases.next_ptr(t_next)
        return d

    def __call__(self, fdtd):
        # accumulation happened inside the E update of this step
        return None

    def dft_tensor(self):
        """Device view ``complex128 [n_comp, n_freq, n1, n2]``."""
        return _torch().view_as_complex(self.acc)

    def dft(self, component=None):
        """Host ``complex128`` array ``(n_freq, n1, n2)`` for one component (default: first)."""
        c = self.components[0] if component is None else component
        q = self.components.index(c)
        self.fdtd.queue.synchronize()
        a = self.acc[q].cpu().numpy()
        return a[..., 0] + 1j * a[..., 1]


class CUDANear2FarMonitor:
    """Huygens-box DFT + near-to-far transform on the GPU (``OpenCLNear2FarMonitor`` API)."""

    def __init__(self, fdtd, center, size, freq):
        torch = _torch()
        if getattr(fdtd, "slab", None) is not None:
            raise NotImplementedError("the Huygens-box monitor runs on a whole grid, not on one "
                                      "x-slab of a decomposed grid")
        self.fdtd = fdtd
        self.freqs = np.atleast_1d(np.asarray(freq, dtype=np.float64))
        if not 0 < self.freqs.size <= capi.FDTD_MAX_FREQS:
            raise ValueError(f"1 to {capi.FDTD_MAX_FREQS} frequencies, got {self.freqs.size}")
        self.freq = float(self.freqs[0]) if np.ndim(freq) == 0 else self.freqs
        self.omega = 2.0 * np.pi * self.freq if np.ndim(freq) == 0 else 2.0 * np.pi * self.freqs
        self.dl = fdtd.dl
        cx, cy, cz = center
        sx, sy, sz = size

        def _idx(phys):
            return int(round(phys / fdtd.dl))

        self.ix0 = max(0, _idx(cx - sx / 2))
        self.ix1 = min(fdtd.Nx - 1, _idx(cx + sx / 2))
        self.iy0 = max(0, _idx(cy - sy / 2))
        self.iy1 = min(fdtd.Ny - 1, _idx(cy + sy / 2))
        self.iz0 = max(0, _idx(cz - sz / 2))
        self.iz1 = min(fdtd.Nz - 1, _idx(cz + sz / 2))
        if self.ix0 > self.ix1 or self.iy0 > self.iy1 or self.iz0 > self.iz1:
            raise ValueError("Huygens box is empty after snapping to the grid")
        self._box = (self.ix0, self.ix1, self.iy0, self.iy1, self.iz0, self.iz1)
        self.nxf = self.ix1 - self.ix0 + 1
        self.nyf = self.iy1 - self.iy0 + 1
        self.nzf = self.iz1 - self.iz0 + 1
        self._face_counts = (self.nyf * self.nzf, self.nyf * self.nzf, self.nxf * self.nzf,
                             self.nxf * self.nzf, self.nxf * self.nyf, self.nxf * self.nyf)
        offs = [0]
        for c in self._face_counts[:-1]:
            offs.append(offs[-1] + c)
        self._face_offsets = tuple(offs)
        self.n_face_samples = int(sum(self._face_counts))
        self._dtype = fdtd.dtype
        self._acc_complex_dtype = fdtd.accreal_complex_dtype
        self._cbox = _box_struct(self._box, self._face_offsets, self.n_face_samples,
                                 self.freqs.size)
        with torch.cuda.stream(fdtd.queue):
            self.acc = torch.zeros((6, self.freqs.size, self.n_face_samples, 2),
                                   dtype=torch.float64, device=fdtd.device)
        self._phases = _PhaseTable(self.freqs, fdtd.dt, fdtd.device, fdtd.queue)
        self._dft_snap = None
        self.Ex_dft = self.Ey_dft = self.Ez_dft = None
        self.Hx_dft = self.Hy_dft = self.Hz_dft = None
        fdtd.add_monitor(self)

    @property
    def _phase(self):
        p = self._phases.phase
        if p is None:
            return None
        return complex(p[0]) if np.ndim(self.freq) == 0 else p

    def __call__(self, fdtd):
        ptr = self._phases.next_ptr(fdtd.t)
        E = (capi.c_void_p * 3)(*[t.data_ptr() for t in fdtd._E])
        H = (capi.c_void_p * 3)(*[t.data_ptr() for t in fdtd._H])
        capi.run("fdtd_dft_faces", fdtd._grid, E, H, self._cbox, self.acc.data_ptr(), ptr,
                 fdtd.queue.cuda_stream)

    # ------------------------------------------------------------ far field
    def _fi(self, freq_index):
        fi = int(freq_index)
        if not 0 <= fi < self.freqs.size:
            raise IndexError(f"frequency index {fi} outside [0, {self.freqs.size})")
        return fi

    def get_farfields(self, obs_points, freq_index=0, *, method="direct") -> np.ndarray:
        """Far E, H at many points (metres): ``(n_obs, 6)`` complex128 (Ex, Ey, Ez, Hx, Hy, Hz).

        ``method="direct"`` (default) is the float64 surface sum per point, as the
        reference kernel does; ``"bf16x3"`` or ``"tf32"`` evaluates the surface sums
        with the tensor-core contraction (``near2far_contract``, FP32 accumulation)
        and then the same second stage.

        Accuracy classes, as the maximum error over the peak of the float64 sums:
        ``"bf16x3"`` stays within 1e-5 (about 5e-6 measured), the FP32-mode
        tolerance of the far-field parity gate; ``"tf32"`` is about 3e-4 and is
        *outside* that class (10 mantissa bits per operand): use it for previews
        and sweeps, not for results held to 1e-5.
        """
        if method != "direct":
            return self._farfields_contract(obs_points, freq_index, method)
        pts = _obs_array(obs_points, self._dtype)
        fi = self._fi(freq_index)
        return _device_farfields(self.fdtd, self._cbox, self.acc, fi, float(self.freqs[fi]), pts)

    def _farfields_contract(self, obs_points, freq_index, method):
        from .n2f import box_faces, near2far_contract

        torch = _torch()
        # points in the engine dtype, as the direct path and the reference do
        pts = _obs_array(obs_points, self._dtype).astype(np.float64)
        fi = self._fi(freq_index)
        q = self.fdtd.queue
        faces = box_faces(self)
        for f in faces:
            f.cur = f.cur[fi:fi + 1].contiguous()
        nl = near2far_contract(faces, [self.freqs[fi]], pts, mode=method, stream=q)
        n_obs = int(pts.shape[0])
        with torch.cuda.stream(q):
            obs = torch.from_numpy(pts).to(self.fdtd.device)
            eh = torch.empty((n_obs, 6, 2), dtype=torch.float64, device=self.fdtd.device)
        k_wave = 2.0 * np.pi * float(self.freqs[fi]) / C0
        capi.run("fdtd_farfield_eh", nl.data_ptr(), capi.FDTD_F32, obs.data_ptr(), n_obs, k_wave,
                 float(ETA0), eh.data_ptr(), q.cuda_stream)
        q.synchronize()
        h = eh.cpu().numpy()
        return (h[..., 0] + 1j * h[..., 1]).astype(np.complex128)

    def get_farfield(self, obs_point, freq_index=0):
        """Far E, H at one point (metres)."""
        return self.get_farfields([obs_point], freq_index)[0]

    def farfield_polar_xz(self, *, distance_m: float = 1000.0, n_angles: int = 73,
                          freq_index: int = 0):
        """XZ-plane cut: ``(angles_deg, |S| dB)`` at ``distance_m``."""
        R = float(distance_m)
        if R <= 0.0:
            raise ValueError("distance_m must be positive")
        n = max(3, int(n_angles))
        angles = np.linspace(-180.0, 180.0, n, dtype=np.float64)
        rad = np.deg2rad(angles)
        pts = np.column_stack([R * np.sin(rad), np.zeros(n), R * np.cos(rad)]).astype(self._dtype)
        eh = self.get_farfields(pts, freq_index)
        db = np.empty(n, dtype=np.float64)
        for i in range(n):
            db[i], _ = _poynting_db(eh[i])
        return angles, db

    # ----------------------------------------------------- DFT convergence
    def snapshot_dft(self) -> None:
        """Copy the face DFTs to a device snapshot (no host round trip)."""
        torch = _torch()
        with torch.cuda.stream(self.fdtd.queue):
            if self._dft_snap is None:
                self._dft_snap = torch.empty_like(self.acc)
            self._dft_snap.copy_(self.acc)

    def dft_relative_change(self, freq_index=0) -> float:
        """``‖cur − prev‖₂ / ‖cur‖₂`` over the six face DFTs (1.0 without a snapshot)."""
        if self._dft_snap is None:
            return 1.0
        torch = _torch()
        fi = self._fi(freq_index)
        q = self.fdtd.queue
        nblk = int(capi.lib().fdtd_rel_change_blocks(self.n_face_samples))
        with torch.cuda.stream(q):
            scratch = torch.empty(2 * nblk, dtype=torch.float64, device=self.fdtd.device)
            out = torch.empty(2, dtype=torch.float64, device=self.fdtd.device)
        capi.run("fdtd_dft_rel_change", self.acc.data_ptr(), self._dft_snap.data_ptr(),
                 self.n_face_samples, self.freqs.size, fi, scratch.data_ptr(), out.data_ptr(),
                 q.cuda_stream)
        q.synchronize()
        num, den = (float(v) for v in out.cpu().numpy())
        if den <= 0.0 or not np.isfinite(den) or not np.isfinite(num):
            return 1.0
        return float(np.sqrt(max(num, 0.0) / den))

    # ----------------------------------------------------------- download
    def face_dft(self, freq_index=0):
        """Face-packed complex128 DFTs ``{name: (n_face,)}`` for one frequency."""
        fi = self._fi(freq_index)
        self.fdtd.queue.synchronize()
        a = self.acc[:, fi].cpu().numpy()
        return {n: a[q, :, 0] + 1j * a[q, :, 1] for q, n in enumerate(FIELDS)}

    def fetch_dft_fields(self, freq_index=0):
        """Download face DFTs and scatter them into sparse host volumes ``Ex_dft``…``Hz_dft``."""
        faces = {k: v.astype(self._acc_complex_dtype) for k, v in
                 self.face_dft(freq_index).items()}
        shape = (self.fdtd.Nx, self.fdtd.Ny, self.fdtd.Nz)

        def scatter(face_arr):
            vol = np.zeros(shape, dtype=self._acc_complex_dtype)
            for fid, ii in ((0, self.ix0), (1, self.ix1)):
                b = self._face_offsets[fid]
                vol[ii, self.iy0:self.iy1 + 1, self.iz0:self.iz1 + 1] = \
                    face_arr[b:b + self.nyf * self.nzf].reshape(self.nyf, self.nzf)
            for fid, jj in ((2, self.iy0), (3, self.iy1)):
                b = self._face_offsets[fid]
                vol[self.ix0:self.ix1 + 1, jj, self.iz0:self.iz1 + 1] = \
                    face_arr[b:b + self.nxf * self.nzf].reshape(self.nxf, self.nzf)
            for fid, kk in ((4, self.iz0), (5, self.iz1)):
                b = self._face_offsets[fid]
                vol[self.ix0:self.ix1 + 1, self.iy0:self.iy1 + 1, kk] = \
                    face_arr[b:b + self.nxf * self.nyf].reshape(self.nxf, self.nyf)
            return vol

        for n in FIELDS:
            setattr(self, f"{n}_dft", scatter(faces[n]))
        return faces


class NumPyNear2FarMonitor:
    """Host Huygens-box monitor: the reference ``NumPyNear2FarMonitor`` surface
    (``opencl_fdtd_solver/monitors.py:186-380``) on any engine with ``Ex…Hz``.

    Per step it accumulates the face-packed DFT on the host from the engine's
    field reads with the reference arithmetic (``monitors.py:229-295``):
    tangential samples co-located at face centres (2-point means of E, 4-point
    means of H, clamped at the grid edge), E phase ``e^{jωt}·dt``, H phase
    ``e^{jωt}·dt·e^{−jωdt/2}``, complex64 accumulators ``Ex_dft_f … Hz_dft_f`` in
    the x0, x1, y0, y1, z0, z1 packing.  Each face is evaluated as array
    operations instead of the per-sample loop, with the same operands in the
    same order, so every accumulator rounds the same way.

    The monitor declares ``host_regions`` (each face plane with the neighbouring
    planes its means read), so on ``CUDAFDTD`` a step moves those slabs to the
    host instead of six full volumes (``CUDAFDTD.host_window``).  On an engine
    without windowed reads it reads full arrays, as the reference does.

    ``get_farfield(s)`` runs the float64 surface sums on the device with the
    OpenCL kernel's convention ``η·N⊥ − r̂×L`` (``dft_farfield.cl:617``).  The
    reference's host ``get_farfield`` adds ``+ r̂×L`` (``monitors.py:378``), which
    disagrees with its own kernel; the kernel convention is kept here.
    """

    def __init__(self, fdtd, center, size, freq):
        self.fdtd = fdtd
        self.freq = freq
        self.omega = 2.0 * np.pi * freq
        self.dl = fdtd.dl
        cx, cy, cz = center
        sx, sy, sz = size

        def _idx(phys):
            return int(round(phys / fdtd.dl))

        self.ix0 = max(0, _idx(cx - sx / 2))
        self.ix1 = min(fdtd.Nx - 1, _idx(cx + sx / 2))
        self.iy0 = max(0, _idx(cy - sy / 2))
        self.iy1 = min(fdtd.Ny - 1, _idx(cy + sy / 2))
        self.iz0 = max(0, _idx(cz - sz / 2))
        self.iz1 = min(fdtd.Nz - 1, _idx(cz + sz / 2))
        if self.ix0 > self.ix1 or self.iy0 > self.iy1 or self.iz0 > self.iz1:
            raise ValueError("Huygens box is empty after snapping to the grid")
        self._faces = [("x", self.ix0, -1), ("x", self.ix1, +1), ("y", self.iy0, -1),
                       ("y", self.iy1, +1), ("z", self.iz0, -1), ("z", self.iz1, +1)]
        self._box = (self.ix0, self.ix1, self.iy0, self.iy1, self.iz0, self.iz1)
        self.nxf = self.ix1 - self.ix0 + 1
        self.nyf = self.iy1 - self.iy0 + 1
        self.nzf = self.iz1 - self.iz0 + 1
        self._face_counts = (self.nyf * self.nzf, self.nyf * self.nzf, self.nxf * self.nzf,
                             self.nxf * self.nzf, self.nxf * self.nyf, self.nxf * self.nyf)
        offs = [0]
        for c in self._face_counts[:-1]:
            offs.append(offs[-1] + c)
        self._face_offsets = tuple(offs)
        self.n_face_samples = int(sum(self._face_counts))
        for n in FIELDS:
            setattr(self, f"{n}_dft_f", np.zeros(self.n_face_samples, dtype=np.complex64))
        # Volume placeholders of the reference (monitors.py:219-226); np.zeros
        # reserves the pages lazily, so untouched volumes cost no memory.
        shape = (fdtd.Nx, fdtd.Ny, fdtd.Nz)
        for n in FIELDS:
            setattr(self, f"{n}_dft", np.zeros(shape, dtype=np.complex64))
        self._build_indices()
        fdtd.add_monitor(self)

    def _build_indices(self):
        """Per axis: the face samples as a slice, their clamped ``+1`` neighbours
        as a slice (an index array when the box touches the high edge, where the
        reference clamps ``i+1`` to ``i``), and the mask of samples whose
        neighbour differs from themselves."""
        dims = (self.fdtd.Nx, self.fdtd.Ny, self.fdtd.Nz)
        self._sel = []
        for (lo, hi), n in zip(((self.ix0, self.ix1), (self.iy0, self.iy1),
                                (self.iz0, self.iz1)), dims):
            v = np.arange(lo, hi + 1)
            v1 = np.where(v + 1 < n, v + 1, v)
            nxt = slice(lo + 1, hi + 2) if hi + 1 < n else v1
            self._sel.append((slice(lo, hi + 1), nxt, v1 != v))
        # the same selections relative to the box corner, for the z-face slabs
        # that __call__ copies out of the volume (k is the strided axis there)
        self._rel = []
        for (lo, hi), n in zip(((self.ix0, self.ix1), (self.iy0, self.iy1)), dims[:2]):
            v = np.arange(lo, hi + 1)
            v1 = np.where(v + 1 < n, v + 1, v)
            nxt = slice(1, hi - lo + 2) if hi + 1 < n else v1 - lo
            self._rel.append((slice(0, hi - lo + 1), nxt, min(hi + 2, n)))

    def host_regions(self):
        """Half-open boxes of every cell ``__call__`` reads: each face plane, the
        plane below it (H means) and one extra row/column above the face (means)."""
        nx, ny, nz = self.fdtd.Nx, self.fdtd.Ny, self.fdtd.Nz
        ix0, ix1, iy0, iy1, iz0, iz1 = self._box
        ih, jh, kh = min(ix1 + 2, nx), min(iy1 + 2, ny), min(iz1 + 2, nz)
        regs = [((max(i - 1, 0), i + 1), (iy0, jh), (iz0, kh)) for i in (ix0, ix1)]
        regs += [((ix0, ih), (max(j - 1, 0), j + 1), (iz0, kh)) for j in (iy0, iy1)]
        regs += [((ix0, ih), (iy0, jh), (max(k - 1, 0), k + 1)) for k in (iz0, iz1)]
        return regs

    def __call__(self, fdtd):
        phase_e = np.exp(1j * self.omega * fdtd.t) * fdtd.dt
        phase_h = phase_e * np.exp(-0.5j * self.omega * fdtd.dt)
        ph4 = phase_h * 0.25
        Ex, Ey, Ez = np.asarray(fdtd.Ex), np.asarray(fdtd.Ey), np.asarray(fdtd.Ez)
        Hx, Hy, Hz = np.asarray(fdtd.Hx), np.asarray(fdtd.Hy), np.asarray(fdtd.Hz)
        (I, I1, okI), (J, J1, okJ), (K, K1, okK) = self._sel  # noqa: F841
        o = self._face_offsets
        c = self._face_counts

        def at(plane, r, q):
            # rows r and columns q of a 2-D plane view; slices stay views
            if isinstance(r, slice) or isinstance(q, slice):
                return plane[r, q]
            return plane[np.ix_(r, q)]

        def acc(arr, f, vals, ph):
            arr[o[f]:o[f] + c[f]] += ph * vals.ravel()

        rowJ, rowI, colK, colJ = okJ[:, None], okI[:, None], okK[None, :], okJ[None, :]
        # x faces: samples (j, k), j outer.  Means: Ey over k, Ez over j, Hy over
        # (i-1, j+1), Hz over (i-1, k+1), in the reference operand order.
        for f, i in ((0, self.ix0), (1, self.ix1)):
            il = i - 1 if i > 0 else i
            a = at(Ey[i], J, K)
            acc(self.Ey_dft_f, f, np.where(colK, 0.5 * (a + at(Ey[i], J, K1)), a), phase_e)
            a = at(Ez[i], J, K)
            acc(self.Ez_dft_f, f, np.where(rowJ, 0.5 * (a + at(Ez[i], J1, K)), a), phase_e)
            acc(self.Hy_dft_f, f, at(Hy[i], J, K) + at(Hy[il], J, K) + at(Hy[i], J1, K)
                + at(Hy[il], J1, K), ph4)
            acc(self.Hz_dft_f, f, at(Hz[i], J, K) + at(Hz[il], J, K) + at(Hz[i], J, K1)
                + at(Hz[il], J, K1), ph4)
        # y faces: samples (i, k), i outer
        for f, j in ((2, self.iy0), (3, self.iy1)):
            jl = j - 1 if j > 0 else j
            a = at(Ex[:, j], I, K)
            acc(self.Ex_dft_f, f, np.where(colK, 0.5 * (a + at(Ex[:, j], I, K1)), a), phase_e)
            a = at(Ez[:, j], I, K)
            acc(self.Ez_dft_f, f, np.where(rowI, 0.5 * (a + at(Ez[:, j], I1, K)), a), phase_e)
            acc(self.Hx_dft_f, f, at(Hx[:, j], I, K) + at(Hx[:, jl], I, K) + at(Hx[:, j], I1, K)
                + at(Hx[:, jl], I1, K), ph4)
            acc(self.Hz_dft_f, f, at(Hz[:, j], I, K) + at(Hz[:, jl], I, K) + at(Hz[:, j], I, K1)
                + at(Hz[:, jl], I, K1), ph4)
        # z faces: samples (i, j), i outer.  The planes are strided in memory, so
        # each field's (i, j, kl..k) slab is copied once and indexed from the box corner.
        (Ir, I1r, ie), (Jr, J1r, je) = self._rel
        i0, j0 = self.ix0, self.iy0
        for f, k in ((4, self.iz0), (5, self.iz1)):
            kl = k - 1 if k > 0 else k

            def slab(F):
                s_ = np.ascontiguousarray(F[i0:ie, j0:je, kl:k + 1])
                return s_[:, :, k - kl], s_[:, :, 0]

            P, _ = slab(Ex)
            a = at(P, Ir, Jr)
            acc(self.Ex_dft_f, f, np.where(colJ, 0.5 * (a + at(P, Ir, J1r)), a), phase_e)
            P, _ = slab(Ey)
            a = at(P, Ir, Jr)
            acc(self.Ey_dft_f, f, np.where(rowI, 0.5 * (a + at(P, I1r, Jr)), a), phase_e)
            P, Q = slab(Hx)
            acc(self.Hx_dft_f, f, at(P, Ir, Jr) + at(Q, Ir, Jr) + at(P, Ir, J1r)
                + at(Q, Ir, J1r), ph4)
            P, Q = slab(Hy)
            acc(self.Hy_dft_f, f, at(P, Ir, Jr) + at(Q, Ir, Jr) + at(P, I1r, Jr)
                + at(Q, I1r, Jr), ph4)

    def get_farfields(self, obs_points) -> np.ndarray:
        """Far E, H at many points (metres): ``(n_obs, 6)`` complex128."""
        torch = _torch()
        pts = _obs_array(obs_points, self.fdtd.dtype)
        packed = np.stack([getattr(self, f"{n}_dft_f") for n in FIELDS])  # (6, n_face)
        ri = np.stack([packed.real, packed.imag], axis=-1).astype(np.float64)[:, None]
        with torch.cuda.stream(self.fdtd.queue):
            acc = torch.from_numpy(np.ascontiguousarray(ri)).to(self.fdtd.device)
        cbox = _box_struct(self._box, self._face_offsets, self.n_face_samples, 1)
        return _device_farfields(self.fdtd, cbox, acc, 0, float(self.freq), pts)

    def get_farfield(self, obs_point):
        """Far E, H at one point (metres): ``(6,)`` complex128."""
        return self.get_farfields([obs_point])[0]


def _poynting_mag(ff) -> float:
    """``|½ E × H*|`` of a 6-vector (reference ``monitors.py:807-813``)."""
    E = ff[0:3]
    H = ff[3:6]
    Sx = 0.5 * (E[1] * np.conj(H[2]) - E[2] * np.conj(H[1]))
    Sy = 0.5 * (E[2] * np.conj(H[0]) - E[0] * np.conj(H[2]))
    Sz = 0.5 * (E[0] * np.conj(H[1]) - E[1] * np.conj(H[0]))
    return float(np.sqrt(np.abs(Sx) ** 2 + np.abs(Sy) ** 2 + np.abs(Sz) ** 2))


def _poynting_db(ff) -> tuple[float, float]:
    """``(20·log10|S|, |S|)``, ``-inf`` for zero or non-finite (``monitors.py:816-827``)."""
    mag = _poynting_mag(ff)
    if not np.isfinite(mag) or mag <= 0.0:
        return float("-inf"), 0.0
    return float(20.0 * np.log10(mag)), mag
