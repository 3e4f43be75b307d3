"""CPU oracle engine with the reference ``OpenCLFDTD`` control flow (TEST INFRASTRUCTURE).

``OracleFDTD`` drives the C restatement in ``oracle/fdtd_oracle.c`` (or, with
``backend="ref"``, the reference's own kernels compiled as C into
``oracle/_ref/libfdtd_ref.so``) through the same sequence as the reference engine:

* constructor, dt and default coefficients: ``opencl_fdtd_solver/engine.py:99-210``
* ``set_epsilon``: ``engine.py:212-254``
* CPML profiles and ψ stripe sizes: ``engine.py:256-318``
* ``add_source_Ex`` / ``add_source_Jx`` (host rim renormalisation): ``engine.py:448-538``
* ``_update_H`` / ``_update_E`` scalar folding: ``engine.py:540-544, 631-634``
* ``step`` / ``run`` timing contract: ``engine.py:724-744``

``courant=`` overrides the reference's fixed ``0.99/√3`` (``engine.py:138``) for the
configurations quoted at Courant 0.5; CPML ``b, c`` are rebuilt from that dt.
Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use
this module, as the checker.
"""

from __future__ import annotations

import ctypes
import os
import warnings
from pathlib import Path

import numpy as np

from . import host_math as hm

_HERE = Path(__file__).resolve().parent
_LIBS: dict[str, ctypes.CDLL] = {}


def _lib(backend: str) -> ctypes.CDLL:
    if backend not in _LIBS:
        path = _HERE / ("libfdtd_oracle.so" if backend == "oracle" else "_ref/libfdtd_ref.so")
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built; run `python -m oracle.build`")
        _LIBS[backend] = ctypes.CDLL(str(path))
    return _LIBS[backend]


def ref_available() -> bool:
    """True when the reference kernels compiled as C are present."""
    return (_HERE / "_ref/libfdtd_ref.so").exists()


def num_threads() -> int:
    return int(_lib("oracle").og_num_threads())


def set_num_threads(n: int) -> None:
    _lib("oracle").og_set_num_threads(int(n))


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleFDTD:
    """Reference-semantics FDTD on the CPU (fields are plain NumPy arrays)."""

    def __init__(self, shape, dl, npml=20, dtype=np.float32, accum_fp64=False,
                 courant=None, backend="oracle"):
        self.Nx, self.Ny, self.Nz = (int(v) for v in shape)
        self.dl = float(dl)
        self.npml = int(npml)
        dtype = np.dtype(dtype)
        if dtype not in (np.dtype(np.float32), np.dtype(np.float64)):
            raise ValueError("oracle supports float32 or float64")
        self.dtype = dtype
        self.real = dtype.type
        self.accum_fp64 = bool(accum_fp64) or dtype == np.float64
        self.accreal = np.float64 if self.accum_fp64 else self.real
        self.backend = backend
        self._suf = "f32" if dtype == np.float32 else "f64"
        self._ctype = ctypes.c_float if dtype == np.float32 else ctypes.c_double
        lib = _lib(backend)
        pre = "og" if backend == "oracle" else "ref"
        self._fH = getattr(lib, f"{pre}_update_H_{self._suf}")
        self._fE = getattr(lib, f"{pre}_update_E_{self._suf}")
        self._fJ = getattr(lib, f"{pre}_source_Jx_{self._suf}")
        self._fX = getattr(lib, f"{pre}_source_Ex_{self._suf}")
        for f in (self._fH, self._fE, self._fJ, self._fX):
            f.restype = None
        self.t = 0.0
        self.step_num = 0
        if courant is None:
            self.dt = 0.99 * dl / (hm.C0 * np.sqrt(3.0))
        else:
            self.dt = float(courant) * self.dl / hm.C0
        shp = (self.Nx, self.Ny, self.Nz)
        self.Ex, self.Ey, self.Ez = (np.zeros(shp, dtype) for _ in range(3))
        self.Hx, self.Hy, self.Hz = (np.zeros(shp, dtype) for _ in range(3))
        vac = dtype.type(self.dt / hm.EPS0)
        self.ce = [np.full(shp, vac, dtype) for _ in range(3)]
        self.ca = [np.ones(shp, dtype) for _ in range(3)]
        self._sources = []
        self._monitors = []
        self._build_cpml()

    # -- registration (reference plugin.py:23-53)
    def add_source(self, cb):
        if not callable(cb):
            raise TypeError(f"source must be callable, got {type(cb)!r}")
        self._sources.append(cb)
        return cb

    def add_monitor(self, cb):
        if not callable(cb):
            raise TypeError(f"monitor must be callable, got {type(cb)!r}")
        self._monitors.append(cb)
        return cb

    def _build_cpml(self):
        n = self.npml
        prof = hm.cpml_all((self.Nx, self.Ny, self.Nz), n, self.dl, self.dt, self.dtype)
        self.cpml = prof
        nx, ny, nz = self.Nx, self.Ny, self.Nz
        one = np.zeros(1, self.dtype)
        sx = (2 * n, ny, nz) if n > 0 else None
        sy = (nx, 2 * n, nz) if n > 0 else None
        sz = (nx, ny, 2 * n) if n > 0 else None
        mk = (lambda s: np.zeros(s, self.dtype) if s is not None else one.copy())
        # H: Hx_y, Hx_z, Hy_x, Hy_z, Hz_x, Hz_y  (argument order of update_H_pml)
        self.psi_H = [mk(sy), mk(sz), mk(sx), mk(sz), mk(sx), mk(sy)]
        # E: Ex_y, Ex_z, Ey_x, Ey_z, Ez_x, Ez_y  (argument order of update_E_pml)
        self.psi_E = [mk(sy), mk(sz), mk(sx), mk(sz), mk(sx), mk(sy)]

    def set_epsilon(self, eps, sigma_array=None):
        exp = (self.Nx, self.Ny, self.Nz)
        if eps.shape != exp:
            raise ValueError(f"Epsilon shape mismatch: expected {exp}, got {tuple(eps.shape)}")
        if sigma_array is None:
            self.ce = list(hm.edge_ce(eps, self.dt, self.dtype))
            self.ca = [np.ones(exp, self.dtype) for _ in range(3)]
        else:
            ca, cb = hm.edge_ca_cb(eps, sigma_array, self.dt, self.dtype)
            self.ce, self.ca = list(cb), list(ca)

    def add_source_Ex(self, z_src, amp, i0=None, i1=None, j0=None, j1=None):
        warnings.warn("add_source_Ex is a legacy Ex soft-add", DeprecationWarning, stacklevel=2)
        i0 = 0 if i0 is None else int(i0)
        i1 = self.Nx if i1 is None else int(i1)
        j0 = 0 if j0 is None else int(j0)
        j1 = self.Ny if j1 is None else int(j1)
        self._fX(self.Nx, self.Ny, self.Nz, int(z_src), self._ctype(self.real(amp)),
                 i0, i1, j0, j1, _p(self.Ex))

    def add_source_Jx(self, z_src, Jx, i0=None, i1=None, j0=None, j1=None, *,
                      rim_taper=False, rim_edge=0.8, rim_renorm=True):
        i0 = 0 if i0 is None else int(i0)
        i1 = self.Nx if i1 is None else int(i1)
        j0 = 0 if j0 is None else int(j0)
        j1 = self.Ny if j1 is None else int(j1)
        jx = float(Jx)
        re = float(rim_edge)
        if rim_taper and rim_renorm:
            nxs, nys = max(0, i1 - i0), max(0, j1 - j0)
            if nxs >= 2 and nys >= 2:
                ni, nj = nxs - 2, nys - 2
                jx *= (nxs * nys) / (ni * nj + re * (2 * ni + 2 * nj) + re * re * 4)
        self._fJ(self.Nx, self.Ny, self.Nz, int(z_src), self._ctype(self.real(jx)),
                 i0, i1, j0, j1, 1 if rim_taper else 0, self._ctype(self.real(re)),
                 _p(self.ce[0]), _p(self.Ex))

    def _cp(self, stag):
        out = []
        for b, c, ik, _ in self.cpml[stag]:
            out += [_p(b), _p(c), _p(ik)]
        return out

    def update_H(self):
        r = self.real
        dtm = r(self.dt / hm.MU0)
        dtm_dl = r(self.dt / (hm.MU0 * self.dl))
        self._fH(self.Nx, self.Ny, self.Nz, self.npml, self._ctype(dtm), self._ctype(dtm_dl),
                 _p(self.Ex), _p(self.Ey), _p(self.Ez), _p(self.Hx), _p(self.Hy), _p(self.Hz),
                 *self._cp("h"), *[_p(a) for a in self.psi_H])

    def update_E(self):
        inv_dl = self.real(1.0 / self.dl)
        self._fE(self.Nx, self.Ny, self.Nz, self.npml, self._ctype(inv_dl),
                 *[_p(a) for a in self.ca], *[_p(a) for a in self.ce],
                 _p(self.Hx), _p(self.Hy), _p(self.Hz), _p(self.Ex), _p(self.Ey), _p(self.Ez),
                 *self._cp("e"), *[_p(a) for a in self.psi_E])

    def step(self):
        self.update_H()
        t_int = self.t
        self.t = t_int + 0.5 * self.dt
        for src in self._sources:
            src(self)
        self.t = t_int
        self.update_E()
        self.t += self.dt
        self.step_num += 1
        for mon in self._monitors:
            mon(self)

    def run(self, n_steps):
        for _ in range(int(n_steps)):
            self.step()

    def read_point(self, name, i, j, k):
        return float(getattr(self, name)[i, j, k])

    def fields(self):
        return {n: getattr(self, n) for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")}


def threads_hint() -> int:
    """Host threads the OpenMP runtime will use (``OMP_NUM_THREADS`` or all cores)."""
    env = os.environ.get("OMP_NUM_THREADS")
    return int(env) if env else (os.cpu_count() or 1)
