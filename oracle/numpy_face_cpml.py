"""NumPy face-striped CPML engine (TEST INFRASTRUCTURE and the NumPy CPU baseline).

A restatement of the reference's pure-NumPy engine with face-local ψ stripes,
``NumPyFDTD_FaceCPML`` (``opencl_fdtd_solver/numpy_face_cpml.py:29-218``, on the
base ``NumPyFDTD`` of ``opencl_fdtd_solver/numpy_engine.py:29-304``):

* κ-scaled curls over the whole volume, then the CPML ψ recursion and the ψ
  terms on each face stripe, low face before high face, axes x, y, z
  (``numpy_face_cpml.py:125-218``);
* one-sided differences that are zero at the last (forward) or first
  (backward) index (``numpy_engine.py:193-211``);
* sources at the half step between the two half updates
  (``numpy_engine.py:283-297``): ``add_source_Jx`` with the rim taper and the
  host renormalisation (``numpy_engine.py:96-153``), ``add_source_Ex``
  (``:70-94``);
* coefficients from the oracle's own restatement of ``cpml.py`` and
  ``materials.py`` (``host_math.py``).

Every array operation keeps the reference's operands and their order, so the
fields equal the reference engine's bit for bit (pinned by
``tests/test_numpy_port.py`` against ``tests/golden/numpy_ref.npz``, which was
made by importing the reference).  ``courant=`` reproduces the reference
override used for the configurations quoted at Courant 0.5 (set ``dt``, rebuild
``ce`` and the CPML profiles).  ``slab=`` (an ``opencl_fdtd_solver_b200.slabs.SlabLocal``)
runs one x-slab of a larger grid: the local planes with their ghosts, the x-CPML
only on global faces, the global profiles' slice, and sheets given in global
indices; the multi-rank CPU tests hold such slabs to the single-domain run.

Only tests and ``bench.py``'s CPU-baseline legs use this module, as the checker
and as the timed NumPy baseline; the product never imports it.
"""

from __future__ import annotations

import numpy as np

from . import host_math as hm

# (field updated, derivative axis of the curl term, ψ sign) per stripe axis; the
# ψ of field F on axis a is recursed from dF'/da and enters F with that sign.
_H_TERMS = {0: (("Hy", "dEz_dx", -1), ("Hz", "dEy_dx", +1)),
            1: (("Hx", "dEz_dy", +1), ("Hz", "dEx_dy", -1)),
            2: (("Hx", "dEy_dz", -1), ("Hy", "dEx_dz", +1))}
_E_TERMS = {0: (("Ey", "dHz_dx", -1), ("Ez", "dHy_dx", +1)),
            1: (("Ex", "dHz_dy", +1), ("Ez", "dHx_dy", -1)),
            2: (("Ex", "dHy_dz", -1), ("Ey", "dHx_dz", +1))}


def _fwd(f, axis):
    """Forward difference along ``axis``; zero on the last plane."""
    d = np.zeros_like(f)
    hi = [slice(None)] * 3
    lo = [slice(None)] * 3
    hi[axis] = slice(1, None)
    lo[axis] = slice(None, -1)
    d[tuple(lo)] = f[tuple(hi)] - f[tuple(lo)]
    return d


def _bwd(f, axis):
    """Backward difference along ``axis``; zero on the first plane."""
    d = np.zeros_like(f)
    hi = [slice(None)] * 3
    lo = [slice(None)] * 3
    hi[axis] = slice(1, None)
    lo[axis] = slice(None, -1)
    d[tuple(hi)] = f[tuple(hi)] - f[tuple(lo)]
    return d


def _bcast(v, axis):
    shape = [1, 1, 1]
    shape[axis] = -1
    return v.reshape(shape)


class NumPyFaceCPML:
    """CPU FDTD with the reference's NumPy face-CPML arithmetic."""

    def __init__(self, shape, dl, npml=20, dtype=np.float32, courant=None, slab=None):
        self.slab = slab
        self.global_shape = tuple(int(v) for v in shape)
        self.Nx, self.Ny, self.Nz = self.global_shape
        # x-planes of the local grid: global [x0, x0 + Nx); CPML layers per x side
        self.x0, self.pml_x = 0, (int(npml), int(npml))
        if slab is not None:
            self.Nx, self.x0, self.pml_x = slab.nx_local, slab.l0, (slab.pml_lo, slab.pml_hi)
        self.shape = (self.Nx, self.Ny, self.Nz)
        self.dl = float(dl)
        self.npml = int(npml)
        self.dtype = np.dtype(dtype)
        self.t = 0.0
        self.step_num = 0
        self.dt = (0.99 * dl / (hm.C0 * np.sqrt(3.0)) if courant is None
                   else float(courant) * self.dl / hm.C0)
        for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            setattr(self, n, np.zeros(self.shape, self.dtype))
        self.set_epsilon(np.ones(self.global_shape, self.dtype))
        self._sources = []
        self._monitors = []
        self._build_cpml()

    # ------------------------------------------------------------ set-up
    def set_epsilon(self, eps):
        """εr of the whole grid (``global_shape``); a slab takes its planes."""
        if eps.shape != self.global_shape:
            raise ValueError(f"Epsilon shape mismatch: expected {self.global_shape}, "
                             f"got {eps.shape}")
        eps_r = eps[self.x0:self.x0 + self.Nx].astype(self.dtype)
        self.ce = list(hm.edge_ce(eps_r, self.dt, self.dtype))

    def _sides(self, axis):
        """CPML layers (low, high) along ``axis`` on the local grid."""
        return self.pml_x if axis == 0 else (self.npml, self.npml)

    def _build_cpml(self):
        prof = hm.cpml_all(self.global_shape, self.npml, self.dl, self.dt, self.dtype)
        sel = slice(self.x0, self.x0 + self.Nx)  # the local planes of the x profiles
        # per stagger and axis: b, c on the axis and κ broadcast for the volume curls
        self._prof = {}
        for st in ("h", "e"):
            axes = []
            for a, (b, c, _ik, kap) in enumerate(prof[st]):
                if a == 0:
                    b, c, kap = b[sel], c[sel], kap[sel]
                axes.append((b, c, _bcast(kap, a)))
            self._prof[st] = axes
        self._psi = {}
        for a in range(3):
            lo, hi = self._sides(a)
            shp = list(self.shape)
            shp[a] = lo + hi
            for name, _d, _s in _H_TERMS[a] + _E_TERMS[a]:
                self._psi[(name, a)] = np.zeros(shp if self.npml > 0 else (0,), self.dtype)

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

    # ------------------------------------------------------------ sources
    def _span(self, i0, i1, j0, j1):
        """Sheet bounds in global indices (defaults: the whole global plane)."""
        return (0 if i0 is None else int(i0), self.global_shape[0] if i1 is None else int(i1),
                0 if j0 is None else int(j0), self.Ny if j1 is None else int(j1))

    def _local_rows(self, a0, a1):
        """The sheet rows [a0, a1) (global) that lie on the local grid: the local
        slice and the matching slice of the sheet's own row index."""
        l0, l1 = max(a0, self.x0), min(a1, self.x0 + self.Nx)
        if l1 <= l0:
            return slice(0, 0), slice(0, 0)
        return slice(l0 - self.x0, l1 - self.x0), slice(l0 - a0, l1 - a0)

    def add_source_Ex(self, z_src, amp, i0=None, i1=None, j0=None, j1=None):
        a0, a1, b0, b1 = self._span(i0, i1, j0, j1)
        loc, _ = self._local_rows(a0, a1)
        self.Ex[loc, b0:b1, int(z_src)] += self.dtype.type(amp)

    def add_source_Jx(self, z_src, Jx, i0=None, i1=None, j0=None, j1=None, *,
                      rim_taper=False, rim_edge=0.8, rim_renorm=True):
        a0, a1, b0, b1 = self._span(i0, i1, j0, j1)
        z, jx, re = int(z_src), float(Jx), float(rim_edge)
        na, nb = max(0, a1 - a0), max(0, b1 - b0)
        if rim_taper and rim_renorm and na >= 2 and nb >= 2:
            inner_a, inner_b = na - 2, nb - 2
            total = inner_a * inner_b + re * (2 * inner_a + 2 * inner_b) + (re * re) * 4
            jx *= (na * nb) / total
        loc, rows = self._local_rows(a0, a1)
        inj = -self.ce[0][loc, b0:b1, z] * jx
        if rim_taper:
            w = np.ones((na, nb), self.dtype)
            if na >= 1:
                w[0, :] *= re
                w[-1, :] *= re
            if nb >= 1:
                w[:, 0] *= re
                w[:, -1] *= re
            inj = inj * w[rows]
        self.Ex[loc, b0:b1, z] += inj.astype(self.dtype, copy=False)

    # ------------------------------------------------------------ update
    def _faces(self, axis):
        """(domain slice, stripe slice) of the low then the high stripe."""
        n = self.shape[axis]
        lo, hi = self._sides(axis)
        out = []
        if lo > 0:
            out.append((slice(0, lo), slice(0, lo)))
        if hi > 0:
            out.append((slice(n - hi, n), slice(lo, lo + hi)))
        return out

    def _stripe_terms(self, terms, stag, diffs, apply):
        for a in range(3):
            b_all, c_all, _ = self._prof[stag][a]
            for dom, stripe in self._faces(a):
                b = _bcast(b_all[dom], a)
                c = _bcast(c_all[dom], a)
                sel_d = [slice(None)] * 3
                sel_s = [slice(None)] * 3
                sel_d[a], sel_s[a] = dom, stripe
                sel_d, sel_s = tuple(sel_d), tuple(sel_s)
                for name, dname, _sign in terms[a]:
                    psi = self._psi[(name, a)]
                    psi[sel_s] = b * psi[sel_s] + c * diffs[dname][sel_d]
                for name, _dname, sign in terms[a]:
                    psi = self._psi[(name, a)][sel_s]
                    apply(name, sel_d, psi if sign > 0 else -psi)

    def _update_H(self):
        dtm, dl = self.dt / hm.MU0, self.dl
        E = {"x": self.Ex, "y": self.Ey, "z": self.Ez}
        d = {f"dE{f}_d{'xyz'[a]}": _fwd(E[f], a) for f, a in
             (("z", 1), ("y", 2), ("x", 2), ("z", 0), ("y", 0), ("x", 1))}
        kx, ky, kz = (self._prof["h"][a][2] for a in range(3))
        self.Hx -= dtm * (d["dEz_dy"] / (ky * dl) - d["dEy_dz"] / (kz * dl))
        self.Hy -= dtm * (d["dEx_dz"] / (kz * dl) - d["dEz_dx"] / (kx * dl))
        self.Hz -= dtm * (d["dEy_dx"] / (kx * dl) - d["dEx_dy"] / (ky * dl))
        if self.npml <= 0:
            return

        def apply(name, sel, term):
            getattr(self, name)[sel] -= dtm * term

        self._stripe_terms(_H_TERMS, "h", d, apply)

    def _update_E(self):
        dl = self.dl
        H = {"x": self.Hx, "y": self.Hy, "z": self.Hz}
        d = {f"dH{f}_d{'xyz'[a]}": _bwd(H[f], a) for f, a in
             (("z", 1), ("y", 2), ("x", 2), ("z", 0), ("y", 0), ("x", 1))}
        kx, ky, kz = (self._prof["e"][a][2] for a in range(3))
        cex, cey, cez = self.ce
        self.Ex += cex * (d["dHz_dy"] / (ky * dl) - d["dHy_dz"] / (kz * dl))
        self.Ey += cey * (d["dHx_dz"] / (kz * dl) - d["dHz_dx"] / (kx * dl))
        self.Ez += cez * (d["dHy_dx"] / (kx * dl) - d["dHx_dy"] / (ky * dl))
        if self.npml <= 0:
            return
        ce = {"Ex": cex, "Ey": cey, "Ez": cez}

        def apply(name, sel, term):
            getattr(self, name)[sel] += ce[name][sel] * term

        self._stripe_terms(_E_TERMS, "e", d, apply)

    def step(self):
        self._update_H()
        t_int = self.t
        self.t = t_int + 0.5 * self.dt
        for src in self._sources:
            src(self)
        self.t = t_int
        self._update_E()
        self.t += self.dt
        self.step_num += 1
        for mon in self._monitors:
            mon(self)

    def run(self, n_steps):
        for _ in range(int(n_steps)):
            self.step()
