"""NumPy restatement of the reference DFT monitors and near-to-far transform (TEST INFRASTRUCTURE).

* Huygens box snapping: ``opencl_fdtd_solver/monitors.py:37-45``
* face packing x0,x1,y0,y1,z0,z1: ``monitors.py:396-412``
* per-step phase recurrence: ``monitors.py:456-459, 571-584``
* co-located tangential face DFT: ``opencl_fdtd_solver/kernels/dft_farfield.cl:116-230``
* relative-change reduction: ``dft_farfield.cl:237-290``, ``monitors.py:505-569``
* N/L surface integral with trapezoid weights: ``dft_farfield.cl:372-474``
* far E/H from N, L (``η·N⊥ − r̂×L``): ``dft_farfield.cl:559-635``
* XZ polar cut and Poynting dB: ``monitors.py:737-755, 807-827``

The plane DFT monitor has no reference class; its semantics are those of the face
kernel without co-location (``dft_farfield.cl:50-96``) with the same phase
convention (E at the step time, H half a step earlier).

Everything here is evaluated in float64/complex128 (the reference's ``accum_fp64``
precision); far-field phases are computed in float64 rather than the reference's
field dtype, which is the more accurate of the two.
"""

from __future__ import annotations

import numpy as np

from .host_math import C0, ETA0

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def snap_box(shape, dl, center, size):
    """Half-open-free inclusive index box ``(ix0, ix1, iy0, iy1, iz0, iz1)``."""
    nx, ny, nz = shape
    out = []
    for c, s, n in zip(center, size, (nx, ny, nz)):
        lo = max(0, int(round((c - s / 2) / dl)))
        hi = min(n - 1, int(round((c + s / 2) / dl)))
        out += [lo, hi]
    return tuple(out)


def face_layout(box):
    ix0, ix1, iy0, iy1, iz0, iz1 = box
    nxf, nyf, nzf = ix1 - ix0 + 1, iy1 - iy0 + 1, iz1 - iz0 + 1
    counts = (nyf * nzf, nyf * nzf, nxf * nzf, nxf * nzf, nxf * nyf, nxf * nyf)
    offs = tuple(int(v) for v in np.concatenate([[0], np.cumsum(counts)[:-1]]))
    return (nxf, nyf, nzf), counts, offs, int(sum(counts))


def face_samples(box):
    """Per packed sample: ``face, i, j, k`` (int arrays) in the reference packing order."""
    ix0, ix1, iy0, iy1, iz0, iz1 = box
    (nxf, nyf, nzf), counts, offs, n = face_layout(box)
    face = np.empty(n, np.int64)
    I = np.empty(n, np.int64)
    J = np.empty(n, np.int64)
    K = np.empty(n, np.int64)
    for f in range(6):
        sl = slice(offs[f], offs[f] + counts[f])
        loc = np.arange(counts[f])
        face[sl] = f
        if f < 2:
            I[sl] = ix0 if f == 0 else ix1
            J[sl] = iy0 + loc // nzf
            K[sl] = iz0 + loc % nzf
        elif f < 4:
            I[sl] = ix0 + loc // nzf
            J[sl] = iy0 if f == 2 else iy1
            K[sl] = iz0 + loc % nzf
        else:
            I[sl] = ix0 + loc // nyf
            J[sl] = iy0 + loc % nyf
            K[sl] = iz0 if f == 4 else iz1
    return face, I, J, K


def colocated_face_values(fields, box, real=np.float32):
    """Tangential E/H co-located at face centres, ``{name: (n,) array or None}``.

    Averages are evaluated in the field dtype in the reference operand order.
    """
    face, I, J, K = face_samples(box)
    Ex, Ey, Ez, Hx, Hy, Hz = (np.asarray(fields[n]) for n in FIELDS)
    nx, ny, nz = Ex.shape
    r = np.dtype(real).type
    half, quarter = r(0.5), r(0.25)
    n = face.size
    out = {name: np.zeros(n, dtype=real) for name in FIELDS}
    i1 = np.where(I + 1 < nx, I + 1, I)
    j1 = np.where(J + 1 < ny, J + 1, J)
    k1 = np.where(K + 1 < nz, K + 1, K)
    ilo = np.where(I > 0, I - 1, I)
    jlo = np.where(J > 0, J - 1, J)
    klo = np.where(K > 0, K - 1, K)

    def avg2(a, b, ok):
        return np.where(ok, half * (a + b), a)

    def avg4(a, b, c, d):
        return quarter * (((a + b) + c) + d)

    m = face < 2
    i, j, k = I[m], J[m], K[m]
    out["Ey"][m] = avg2(Ey[i, j, k], Ey[i, j, k1[m]], k1[m] != k)
    out["Ez"][m] = avg2(Ez[i, j, k], Ez[i, j1[m], k], j1[m] != j)
    out["Hy"][m] = avg4(Hy[i, j, k], Hy[ilo[m], j, k], Hy[i, j1[m], k], Hy[ilo[m], j1[m], k])
    out["Hz"][m] = avg4(Hz[i, j, k], Hz[ilo[m], j, k], Hz[i, j, k1[m]], Hz[ilo[m], j, k1[m]])
    m = (face >= 2) & (face < 4)
    i, j, k = I[m], J[m], K[m]
    out["Ex"][m] = avg2(Ex[i, j, k], Ex[i, j, k1[m]], k1[m] != k)
    out["Ez"][m] = avg2(Ez[i, j, k], Ez[i1[m], j, k], i1[m] != i)
    out["Hx"][m] = avg4(Hx[i, j, k], Hx[i, jlo[m], k], Hx[i1[m], j, k], Hx[i1[m], jlo[m], k])
    out["Hz"][m] = avg4(Hz[i, j, k], Hz[i, jlo[m], k], Hz[i, j, k1[m]], Hz[i, jlo[m], k1[m]])
    m = face >= 4
    i, j, k = I[m], J[m], K[m]
    out["Ex"][m] = avg2(Ex[i, j, k], Ex[i, j1[m], k], j1[m] != j)
    out["Ey"][m] = avg2(Ey[i, j, k], Ey[i1[m], j, k], i1[m] != i)
    out["Hx"][m] = avg4(Hx[i, j, k], Hx[i, j, klo[m]], Hx[i, j1[m], k], Hx[i, j1[m], klo[m]])
    out["Hy"][m] = avg4(Hy[i, j, k], Hy[i, j, klo[m]], Hy[i1[m], j, k], Hy[i1[m], j, klo[m]])
    return out


class PhaseRecurrence:
    """``p₁ = e^{jωt₁}·dt``, ``pₙ₊₁ = pₙ·e^{jωdt}``; H phase ``pₙ·e^{−jωdt/2}`` (complex128)."""

    def __init__(self, freqs, dt):
        self.omega = 2.0 * np.pi * np.atleast_1d(np.asarray(freqs, dtype=np.float64))
        self.dt = float(dt)
        self.dphase = np.exp(1j * self.omega * self.dt)
        self.half = np.exp(-0.5j * self.omega * self.dt)
        self.phase = None

    def next(self, t):
        if self.phase is None:
            self.phase = np.exp(1j * self.omega * t) * self.dt
        else:
            self.phase = self.phase * self.dphase
        return self.phase, self.phase * self.half


class OracleNear2FarMonitor:
    """Face-packed DFT box at one or more frequencies, with reference far-field math."""

    def __init__(self, fdtd, center, size, freq):
        self.fdtd = fdtd
        self.freqs = np.atleast_1d(np.asarray(freq, dtype=np.float64))
        self.freq = float(self.freqs[0])
        self.dl = fdtd.dl
        self.box = snap_box((fdtd.Nx, fdtd.Ny, fdtd.Nz), fdtd.dl, center, size)
        (self.nxf, self.nyf, self.nzf), self.counts, self.offsets, self.n_face_samples = \
            face_layout(self.box)
        nf = self.freqs.size
        self.dft = {n: np.zeros((nf, self.n_face_samples), np.complex128) for n in FIELDS}
        self._rec = PhaseRecurrence(self.freqs, fdtd.dt)
        self._snap = None
        fdtd.add_monitor(self)

    def __call__(self, fdtd):
        pe, ph = self._rec.next(fdtd.t)
        vals = colocated_face_values(fdtd.fields(), self.box, real=fdtd.dtype)
        for name in FIELDS:
            p = pe if name[0] == "E" else ph
            self.dft[name] += p[:, None] * vals[name].astype(np.float64)[None, :]

    def snapshot_dft(self):
        self._snap = {n: v.copy() for n, v in self.dft.items()}

    def dft_relative_change(self, fi=0):
        if self._snap is None:
            return 1.0
        num = sum(float(np.sum(np.abs(self.dft[n][fi] - self._snap[n][fi]) ** 2)) for n in FIELDS)
        den = sum(float(np.sum(np.abs(self.dft[n][fi]) ** 2)) for n in FIELDS)
        if den <= 0 or not np.isfinite(den) or not np.isfinite(num):
            return 1.0
        return float(np.sqrt(max(num, 0.0) / den))

    def get_farfields(self, points, fi=0, reference_fp32_k=False):
        return farfield_eh(self.dft, self.box, self.dl, self.freqs[fi], points, fi=fi,
                           reference_fp32_k=reference_fp32_k)

    def get_farfield(self, point, fi=0, reference_fp32_k=False):
        pts = np.asarray(point, dtype=np.float64).reshape(1, 3)
        return self.get_farfields(pts, fi, reference_fp32_k)[0]

    def farfield_polar_xz(self, *, distance_m=1000.0, n_angles=73, fi=0):
        return polar_xz(lambda pts: self.get_farfields(pts, fi), distance_m, n_angles)


def surface_currents(dft, box, dl, fi=0):
    """Per-sample ``(positions (n,3), weight·dA (n,), cur (n,6) complex)`` for N/L."""
    face, I, J, K = face_samples(box)
    ix0, ix1, iy0, iy1, iz0, iz1 = box
    n = face.size
    pos = np.zeros((n, 3))
    w = np.ones(n)
    cur = np.zeros((n, 6), np.complex128)
    nf = np.where(face % 2 == 0, -1.0, 1.0)
    g = {k: v[fi] for k, v in dft.items()}
    edge = lambda a, lo, hi: np.where((a == lo) | (a == hi), 0.5, 1.0)  # noqa: E731
    m = face < 2
    pos[m] = np.stack([I[m] * dl, (J[m] + 0.5) * dl, (K[m] + 0.5) * dl], 1)
    w[m] = edge(J[m], iy0, iy1) * edge(K[m], iz0, iz1)
    cur[m, 1] = nf[m] * g["Hz"][m]
    cur[m, 2] = -nf[m] * g["Hy"][m]
    cur[m, 4] = -nf[m] * g["Ez"][m]
    cur[m, 5] = nf[m] * g["Ey"][m]
    m = (face >= 2) & (face < 4)
    pos[m] = np.stack([(I[m] + 0.5) * dl, J[m] * dl, (K[m] + 0.5) * dl], 1)
    w[m] = edge(I[m], ix0, ix1) * edge(K[m], iz0, iz1)
    cur[m, 0] = -nf[m] * g["Hz"][m]
    cur[m, 2] = nf[m] * g["Hx"][m]
    cur[m, 3] = nf[m] * g["Ez"][m]
    cur[m, 5] = -nf[m] * g["Ex"][m]
    m = face >= 4
    pos[m] = np.stack([(I[m] + 0.5) * dl, (J[m] + 0.5) * dl, K[m] * dl], 1)
    w[m] = edge(I[m], ix0, ix1) * edge(J[m], iy0, iy1)
    cur[m, 0] = nf[m] * g["Hy"][m]
    cur[m, 1] = -nf[m] * g["Hx"][m]
    cur[m, 3] = -nf[m] * g["Ey"][m]
    cur[m, 4] = nf[m] * g["Ex"][m]
    return pos, w * dl * dl, cur


def nl_integrals(pos, wda, cur, k, points, chunk=256):
    """``NL[o, c] = Σ_s wda_s·e^{+jk r̂_o·r_s}·cur[s, c]`` in complex128."""
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    r = np.sqrt(np.sum(pts**2, axis=1))
    r = np.maximum(r, 1e-30)
    rhat = pts / r[:, None]
    out = np.zeros((pts.shape[0], 6), np.complex128)
    wc = cur * wda[:, None]
    for a in range(0, pts.shape[0], chunk):
        ph = np.exp(1j * k * (rhat[a:a + chunk] @ pos.T))
        out[a:a + chunk] = ph @ wc
    return out


def nl_to_eh(nl, points, k, kr_dtype=np.float64):
    """Far E, H from N/L: ``E = −jk e^{−jkr}/(4πr)·(η0 N⊥ − r̂×L)``, ``H = −r̂×E/η0``.

    ``kr_dtype=np.float32`` evaluates the prefactor angle ``k·r`` in single
    precision the way the reference does with ``accum_fp64=False``
    (``dft_farfield.cl:581-584``); at ``r = 10 m`` that single rounding is a
    global phase of ~3e-5 rad and is the whole of the difference between this
    float64 restatement and the reference's committed far-field arrays.
    """
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    r = np.maximum(np.sqrt(np.sum(pts**2, axis=1)), 1e-30)
    rhat = pts / r[:, None]
    N, L = nl[:, :3], nl[:, 3:]
    kr = (np.asarray(k, kr_dtype) * r.astype(kr_dtype)).astype(np.float64)
    pref = (-1j * k / (4.0 * np.pi * r)) * np.exp(-1j * kr)
    Nt = N - np.sum(rhat * N, axis=1)[:, None] * rhat
    rxL = np.cross(rhat, L)
    E = pref[:, None] * (ETA0 * Nt - rxL)
    H = -np.cross(rhat, E) / ETA0
    return np.concatenate([E, H], axis=1)


def farfield_eh(dft, box, dl, freq, points, fi=0, reference_fp32_k=False):
    """``(n_obs, 6)`` complex far E, H.  ``reference_fp32_k`` rounds ``k`` and the
    prefactor angle to float32 as the reference's default (single-precision
    accumulator) build does; it exists to pin this restatement to the
    reference's committed far-field arrays."""
    k = 2.0 * np.pi * float(freq) / C0
    kr_dtype = np.float64
    if reference_fp32_k:
        k = float(np.float32(k))
        kr_dtype = np.float32
    pos, wda, cur = surface_currents(dft, box, dl, fi)
    nl = nl_integrals(pos, wda, cur, k, points)
    return nl_to_eh(nl, points, k, kr_dtype=kr_dtype)


def poynting_mag(ff):
    E, H = ff[0:3], ff[3:6]
    sx = 0.5 * (E[1] * np.conj(H[2]) - E[2] * np.conj(H[1]))
    sy = 0.5 * (E[2] * np.conj(H[0]) - E[0] * np.conj(H[2]))
    sz = 0.5 * (E[0] * np.conj(H[1]) - E[1] * np.conj(H[0]))
    return float(np.sqrt(abs(sx) ** 2 + abs(sy) ** 2 + abs(sz) ** 2))


def poynting_db(ff):
    mag = poynting_mag(ff)
    if not np.isfinite(mag) or mag <= 0.0:
        return float("-inf"), 0.0
    return float(20.0 * np.log10(mag)), mag


def polar_xz(get_farfields, distance_m, n_angles):
    R = float(distance_m)
    if R <= 0.0:
        raise ValueError("distance_m must be positive")
    n = max(3, int(n_angles))
    ang = np.linspace(-180.0, 180.0, n)
    rad = np.deg2rad(ang)
    pts = np.column_stack([R * np.sin(rad), np.zeros(n), R * np.cos(rad)])
    eh = get_farfields(pts)
    return ang, np.array([poynting_db(eh[i])[0] for i in range(n)])


class OraclePlaneDFTMonitor:
    """Single-plane DFT of chosen components at several frequencies (complex128 sums)."""

    def __init__(self, fdtd, axis, index, freqs, components=("Ex",)):
        self.fdtd = fdtd
        self.axis = {"x": 0, "y": 1, "z": 2}.get(axis, axis)
        self.index = int(index)
        self.freqs = np.atleast_1d(np.asarray(freqs, dtype=np.float64))
        self.components = tuple(components)
        shp = [fdtd.Nx, fdtd.Ny, fdtd.Nz]
        del shp[self.axis]
        self.dft = {c: np.zeros((self.freqs.size, *shp), np.complex128) for c in self.components}
        self._rec = PhaseRecurrence(self.freqs, fdtd.dt)
        fdtd.add_monitor(self)

    def __call__(self, fdtd):
        pe, ph = self._rec.next(fdtd.t)
        sl = [slice(None)] * 3
        sl[self.axis] = self.index
        for c in self.components:
            p = pe if c[0] == "E" else ph
            plane = getattr(fdtd, c)[tuple(sl)].astype(np.float64)
            self.dft[c] += p[:, None, None] * plane[None]
