"""CPU restatement of the discrete adjoint ε-gradient (TEST INFRASTRUCTURE).

The reference has no gradient; this module states, in NumPy, the transpose of the
reference's Yee/CPML step (``opencl_fdtd_solver/kernels/yee_update.cl:11-238``,
restated by ``fdtd_oracle.c``) and the chain rule through the Yee-edge ε average
(``opencl_fdtd_solver/materials.py:28-56``), in the operation order of the CUDA
kernels in ``opencl_fdtd_solver_b200/csrc/adjoint.cu``.  Its own correctness is
pinned by ``oracle/torch_fdtd.py`` (torch autograd through an FP64 transcription of
``opencl_fdtd_solver/numpy_engine.py:193-297``), independently of this derivation.

Notation (for a lossless grid, ca ≡ 1):

* E pairs p = Ex_y, Ex_z, Ey_x, Ey_z, Ez_x, Ez_y with derivative axis d and sign
  s = +,−,−,+,+,−:  P_p ← b_e,d·P_p + s·ce·Ē,   ḡ_p = s·ce·ik_e,d·Ē + c_e,d·P_p
  (P terms on the d slabs only);  H̄ += B_d^T ḡ_p.
* H pairs p = Hx_y … Hz_y, sign −s:  P_p ← b_h,d·P_p − s·dtm·H̄,
  ā_p = −s·dtm·ik_h,d·H̄ + c_h,d·P_p;  Ē += F_d^T ā_p.
* (B^T v)(x) = [x≥1]·v(x) − [x≤n−2]·v(x+1);  (F^T v)(x) = [x≥1]·v(x−1) − [x≤n−2]·v(x).
* ce·∂J/∂ce = Σ_n Ē^{n+1}·(E^{n+1} − E^n) (float64), so ∂J/∂ε_edge = −that/ε_edge;
  each cell collects ½ of its two edges per axis (the last plane keeps the cell).

Only tests and the smoke check import this module.
"""

from __future__ import annotations

import numpy as np

from . import host_math as hm

E_PAIRS = ((0, 1, True), (0, 2, False), (1, 0, False), (1, 2, True), (2, 0, True), (2, 1, False))
"""(component, derivative axis, positive in the E update) for ψ_E order Ex_y … Ez_y."""


def _bc(v, axis):
    shp = [1, 1, 1]
    shp[axis] = -1
    return v.reshape(shp)


def _slab_mask(shape, axis, npml):
    n = shape[axis]
    x = np.arange(n)
    m = (x < npml) | (x >= n - npml) if npml > 0 else np.zeros(n, bool)
    return _bc(m, axis)


def _bt(g, axis):
    """(B^T g)(x) = [x≥1]·g(x) − [x≤n−2]·g(x+1), evaluated as the kernel does."""
    lo = np.zeros_like(g)
    hi = np.zeros_like(g)
    sl = [slice(None)] * 3
    sl[axis] = slice(1, None)
    lo[tuple(sl)] = g[tuple(sl)]
    a = [slice(None)] * 3
    b = [slice(None)] * 3
    a[axis] = slice(0, -1)
    b[axis] = slice(1, None)
    hi[tuple(a)] = g[tuple(b)]
    return lo - hi


def _ft(g, axis):
    """(F^T g)(x) = [x≥1]·g(x−1) − [x≤n−2]·g(x)."""
    lo = np.zeros_like(g)
    hi = np.zeros_like(g)
    a = [slice(None)] * 3
    b = [slice(None)] * 3
    a[axis] = slice(1, None)
    b[axis] = slice(0, -1)
    lo[tuple(a)] = g[tuple(b)]
    hi[tuple(b)] = g[tuple(b)]
    return lo - hi


class OracleAdjoint:
    """Reverse sweep state (Ē, H̄, P_E, P_H on full-grid arrays) for one oracle engine."""

    def __init__(self, fd):
        self.fd = fd
        self.dtype = fd.dtype
        self.shape = (fd.Nx, fd.Ny, fd.Nz)
        z = lambda: np.zeros(self.shape, self.dtype)  # noqa: E731
        self.E = [z() for _ in range(3)]
        self.H = [z() for _ in range(3)]
        self.PE = [z() for _ in range(6)]
        self.PH = [z() for _ in range(6)]
        r = fd.real
        self.dtm = r(fd.dt / hm.MU0)
        self.ce = [np.asarray(c) for c in fd.ce]
        self.cpe = fd.cpml["e"]
        self.cph = fd.cpml["h"]
        self.masks = [_slab_mask(self.shape, a, fd.npml) for a in range(3)]

    def add_seed(self, axis, index, patch, seed, phase):
        """Ē_c += Σ_f Re(seed)·Re(phase) + Im(seed)·Im(phase) on the patch.

        ``seed``: complex128 ``(ncomp, nfreq, na, nb)`` for the E components in
        ``self.seed_comps`` order; ``phase``: complex128 ``(nfreq,)``.
        """
        (a0, a1), (b0, b1) = patch
        sl = [slice(a0, a1), slice(b0, b1)]
        sl.insert(axis, index)
        sl = tuple(sl)
        for slot, c in enumerate(self.seed_comps):
            acc = np.zeros((a1 - a0, b1 - b0), np.float64)
            for f in range(seed.shape[1]):
                s = seed[slot, f]
                acc = acc + (s.real * phase[f].real + s.imag * phase[f].imag)
            self.E[c][sl] = self.E[c][sl] + acc.astype(self.dtype)

    def _e_pair(self, p):
        c, d, pos = E_PAIRS[p]
        b, cc, ik, _ = self.cpe[d]
        t = self.ce[c] * _bc(ik, d) * self.E[c]
        g = t if pos else -t
        u = self.ce[c] * self.E[c]
        pn = _bc(b, d) * self.PE[p] + (u if pos else -u)
        m = self.masks[d]
        g = np.where(m, g + _bc(cc, d) * pn, g)
        return g, np.where(m, pn, self.PE[p])

    def _h_pair(self, p):
        c, d, pos_e = E_PAIRS[p]
        pos = not pos_e
        b, cc, ik, _ = self.cph[d]
        t = self.dtm * _bc(ik, d) * self.H[c]
        g = t if pos else -t
        u = self.dtm * self.H[c]
        pn = _bc(b, d) * self.PH[p] + (u if pos else -u)
        m = self.masks[d]
        g = np.where(m, g + _bc(cc, d) * pn, g)
        return g, np.where(m, pn, self.PH[p])

    def step(self, box=None, e_next=None, e_prev=None, G=None):
        """One reverse step (transposed E update with gradient, transposed H update)."""
        res = [self._e_pair(p) for p in range(6)]
        g = [r[0] for r in res]
        if box is not None:
            sl = tuple(slice(lo, hi) for lo, hi in box)
            for c in range(3):
                de = e_next[c].astype(np.float64) - e_prev[c].astype(np.float64)
                G[c] = G[c] + self.E[c][sl].astype(np.float64) * de
        self.PE = [r[1] for r in res]
        self.H[0] = self.H[0] + (_bt(g[3], 2) + _bt(g[5], 1))
        self.H[1] = self.H[1] + (_bt(g[1], 2) + _bt(g[4], 0))
        self.H[2] = self.H[2] + (_bt(g[0], 1) + _bt(g[2], 0))
        res = [self._h_pair(p) for p in range(6)]
        a = [r[0] for r in res]
        self.PH = [r[1] for r in res]
        self.E[0] = self.E[0] + (_ft(a[3], 2) + _ft(a[5], 1))
        self.E[1] = self.E[1] + (_ft(a[1], 2) + _ft(a[4], 0))
        self.E[2] = self.E[2] + (_ft(a[0], 1) + _ft(a[2], 0))


def phase_sequence(freqs, dt, n_steps, t_first):
    """The plane monitor's E phases φ_n (complex128 ``(n_steps, nfreq)``): φ_0 =
    e^{jωt_first}·dt, φ_n = φ_{n−1}·e^{jωdt}, the recurrence of
    ``opencl_fdtd_solver/monitors.py:571-577``."""
    omega = 2.0 * np.pi * np.asarray(freqs, np.float64)
    d = np.exp(1j * omega * float(dt))
    out = np.empty((int(n_steps), omega.size), np.complex128)
    p = np.exp(1j * omega * float(t_first)) * float(dt)
    for n in range(int(n_steps)):
        if n > 0:
            p = p * d
        out[n] = p
    return out


def grad_box(shape, design):
    """Edge box [d0−1, d1) ∩ [0, n) per axis covering every edge a design cell touches."""
    return tuple((max(0, lo - 1), hi) for (lo, hi) in design)


def edge_to_cell(G, eps_full, design, box):
    """∂J/∂ε over the design cells from ce·∂J/∂ce on the edge box (float64)."""
    eps_e = hm.edge_eps(eps_full)
    shape = eps_full.shape
    bsl = tuple(slice(lo, hi) for lo, hi in box)
    out = np.zeros(tuple(hi - lo for lo, hi in design), np.float64)
    for c in range(3):
        ge = np.zeros(shape, np.float64)
        ge[bsl] = -G[c] / eps_e[c][bsl]
        n = shape[c]
        cell = np.zeros(shape, np.float64)
        a = [slice(None)] * 3
        b = [slice(None)] * 3
        a[c] = slice(0, n - 1)
        cell[tuple(a)] += 0.5 * ge[tuple(a)]
        a[c] = slice(1, n)
        b[c] = slice(0, n - 1)
        cell[tuple(a)] += 0.5 * ge[tuple(b)]
        a[c] = slice(n - 1, n)
        cell[tuple(a)] += ge[tuple(a)]
        out += cell[tuple(slice(lo, hi) for lo, hi in design)]
    return out


def gradient(fd, n_steps, objective, design, eps_full):
    """Forward ``n_steps`` on the oracle engine ``fd`` (sources registered, fields
    zero, ``set_epsilon(eps_full)`` done) and return ``(J, dJ/dε_design, D)``.

    ``objective``: dict with ``axis, index, patch ((a0,a1),(b0,b1)), freqs,
    components`` (E names); J = Σ|D|² over the patch, D the plane DFT.
    """
    axis, index, patch = objective["axis"], objective["index"], objective["patch"]
    comps = [("Ex", "Ey", "Ez").index(c) for c in objective.get("components", ("Ex",))]
    comps.sort()
    phases = phase_sequence(objective["freqs"], fd.dt, n_steps, fd.t + fd.dt)
    (a0, a1), (b0, b1) = patch
    sl = [slice(a0, a1), slice(b0, b1)]
    sl.insert(axis, index)
    sl = tuple(sl)
    box = grad_box(fd.Ex.shape, design)
    bsl = tuple(slice(lo, hi) for lo, hi in box)
    nf = phases.shape[1]
    acc = np.zeros((len(comps), nf, a1 - a0, b1 - b0), np.complex128)
    re = acc.real.copy()
    im = acc.imag.copy()
    caps = [[fd.fields()[n][bsl].copy() for n in ("Ex", "Ey", "Ez")]]
    for n in range(n_steps):
        fd.step()
        E = (fd.Ex, fd.Ey, fd.Ez)
        for s, c in enumerate(comps):
            v = E[c][sl].astype(np.float64)
            for f in range(nf):
                re[s, f] = re[s, f] + v * phases[n, f].real
                im[s, f] = im[s, f] + v * phases[n, f].imag
        caps.append([E[c][bsl].copy() for c in range(3)])
    D = re + 1j * im
    J = float(np.sum(re * re + im * im))
    seed = 2.0 * D
    adj = OracleAdjoint(fd)
    adj.seed_comps = comps
    G = [np.zeros(tuple(hi - lo for lo, hi in box), np.float64) for _ in range(3)]
    adj.add_seed(axis, index, patch, seed, phases[n_steps - 1])
    for n in range(n_steps - 1, -1, -1):
        adj.step(box, caps[n + 1], caps[n], G)
        if n >= 1:
            adj.add_seed(axis, index, patch, seed, phases[n - 1])
    return J, edge_to_cell(G, np.asarray(eps_full, np.float64), design, box), D
