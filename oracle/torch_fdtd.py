"""FP64 PyTorch transcription of the reference NumPy engine, for autograd (TEST INFRASTRUCTURE).

Each step transcribes ``opencl_fdtd_solver/numpy_engine.py``:

* forward / backward differences, zero at the last / first index: ``:193-211``
* ``_update_H`` with full-grid ψ and ``dE/(κ·dl)``: ``:213-248``
* ``_update_E``: ``:250-284``
* ``add_source_Jx`` (``soft = −ce_x·Jx·w``, rim weights and renorm): ``:93-153``
* ``step`` order H → sources at t+dt/2 → E → t += dt: ``:286-297``
* ``ce = dt/(ε0·ε_edge)`` with the two-cell edge average: ``materials.py:28-56``

ε is a torch tensor, so ``torch.autograd`` differentiates the whole run; that
gradient is the independent check of the hand-derived adjoint.  The CPML
profiles are the oracle's restatement (``host_math.cpml_axis``).  The plane DFT
uses the monitor phase recurrence (``adjoint_oracle.phase_sequence``).

Only tests import this module.
"""

from __future__ import annotations

import numpy as np

from . import host_math as hm
from .adjoint_oracle import phase_sequence


def _fwd(torch, F, axis):
    d = torch.zeros_like(F)
    n = F.shape[axis]
    d.narrow(axis, 0, n - 1).copy_(F.narrow(axis, 1, n - 1) - F.narrow(axis, 0, n - 1))
    return d


def _bwd(torch, F, axis):
    d = torch.zeros_like(F)
    n = F.shape[axis]
    d.narrow(axis, 1, n - 1).copy_(F.narrow(axis, 1, n - 1) - F.narrow(axis, 0, n - 1))
    return d


def edge_ce(torch, eps, dt):
    """Differentiable ``yee_edge_ce`` (``materials.py:28-56``) in float64."""
    ex = torch.cat([0.5 * (eps[:-1] + eps[1:]), eps[-1:]], 0)
    ey = torch.cat([0.5 * (eps[:, :-1] + eps[:, 1:]), eps[:, -1:]], 1)
    ez = torch.cat([0.5 * (eps[:, :, :-1] + eps[:, :, 1:]), eps[:, :, -1:]], 2)
    scale = float(dt) / hm.EPS0
    return scale / ex, scale / ey, scale / ez


def dft_objective(eps, *, shape, dl, npml, dt, n_steps, sources, objective):
    """Run ``n_steps`` from rest with ``ε = eps`` (float64 tensor) and return
    ``(J, D)`` with D the plane DFT over the objective patch and ``J = Σ|D|²``.

    ``sources``: callable ``(t) -> list of (z, Jx, i0, i1, j0, j1, rim_taper,
    rim_edge, rim_renorm)`` evaluated at ``t + dt/2``.
    """
    import torch

    dev, f64 = eps.device, torch.float64
    nx, ny, nz = shape
    cp = hm.cpml_all(shape, npml, dl, dt, np.float64)

    def bc(v, axis):
        s = [1, 1, 1]
        s[axis] = -1
        return torch.as_tensor(np.asarray(v, np.float64), device=dev).reshape(s)

    bh = [bc(cp["h"][a][0], a) for a in range(3)]
    chh = [bc(cp["h"][a][1], a) for a in range(3)]
    kh = [bc(cp["h"][a][3], a) for a in range(3)]
    be = [bc(cp["e"][a][0], a) for a in range(3)]
    che = [bc(cp["e"][a][1], a) for a in range(3)]
    ke = [bc(cp["e"][a][3], a) for a in range(3)]
    cex, cey, cez = edge_ce(torch, eps, dt)
    z = lambda: torch.zeros(shape, dtype=f64, device=dev)  # noqa: E731
    Ex, Ey, Ez, Hx, Hy, Hz = (z() for _ in range(6))
    pH = [z() for _ in range(6)]  # Hx_y, Hx_z, Hy_x, Hy_z, Hz_x, Hz_y
    pE = [z() for _ in range(6)]  # Ex_y, Ex_z, Ey_x, Ey_z, Ez_x, Ez_y
    dtm = float(dt) / hm.MU0
    axis, index = objective["axis"], objective["index"]
    (a0, a1), (b0, b1) = objective["patch"]
    comps = sorted(("Ex", "Ey", "Ez").index(c) for c in objective.get("components", ("Ex",)))
    phases = phase_sequence(objective["freqs"], dt, n_steps, dt)
    sl = [slice(a0, a1), slice(b0, b1)]
    sl.insert(axis, index)
    sl = tuple(sl)
    nf = phases.shape[1]
    re = [[0.0] * nf for _ in comps]
    im = [[0.0] * nf for _ in comps]
    t = 0.0
    for n in range(int(n_steps)):
        dEz_dy, dEy_dz = _fwd(torch, Ez, 1), _fwd(torch, Ey, 2)
        dEx_dz, dEz_dx = _fwd(torch, Ex, 2), _fwd(torch, Ez, 0)
        dEy_dx, dEx_dy = _fwd(torch, Ey, 0), _fwd(torch, Ex, 1)
        pH[0] = bh[1] * pH[0] + chh[1] * dEz_dy
        pH[1] = bh[2] * pH[1] + chh[2] * dEy_dz
        pH[2] = bh[0] * pH[2] + chh[0] * dEz_dx
        pH[3] = bh[2] * pH[3] + chh[2] * dEx_dz
        pH[4] = bh[0] * pH[4] + chh[0] * dEy_dx
        pH[5] = bh[1] * pH[5] + chh[1] * dEx_dy
        Hx = Hx - dtm * (dEz_dy / (kh[1] * dl) + pH[0] - dEy_dz / (kh[2] * dl) - pH[1])
        Hy = Hy - dtm * (dEx_dz / (kh[2] * dl) + pH[3] - dEz_dx / (kh[0] * dl) - pH[2])
        Hz = Hz - dtm * (dEy_dx / (kh[0] * dl) + pH[4] - dEx_dy / (kh[1] * dl) - pH[5])
        for (zs, jx, i0, i1, j0, j1, rim_taper, rim_edge, rim_renorm) in sources(t + 0.5 * dt):
            jx = float(jx)
            if rim_taper and rim_renorm:
                nxs, nys = max(0, i1 - i0), max(0, j1 - j0)
                if nxs >= 2 and nys >= 2:
                    ni, nj = nxs - 2, nys - 2
                    jx *= (nxs * nys) / (ni * nj + rim_edge * (2 * ni + 2 * nj)
                                         + rim_edge * rim_edge * 4)
            soft = -cex[i0:i1, j0:j1, zs] * jx
            if rim_taper:
                w = np.ones((i1 - i0, j1 - j0))
                w[0, :] *= rim_edge
                w[-1, :] *= rim_edge
                w[:, 0] *= rim_edge
                w[:, -1] *= rim_edge
                soft = soft * torch.as_tensor(w, device=dev)
            add = torch.zeros_like(Ex)
            add[i0:i1, j0:j1, zs] = soft
            Ex = Ex + add
        dHz_dy, dHy_dz = _bwd(torch, Hz, 1), _bwd(torch, Hy, 2)
        dHx_dz, dHz_dx = _bwd(torch, Hx, 2), _bwd(torch, Hz, 0)
        dHy_dx, dHx_dy = _bwd(torch, Hy, 0), _bwd(torch, Hx, 1)
        pE[0] = be[1] * pE[0] + che[1] * dHz_dy
        pE[1] = be[2] * pE[1] + che[2] * dHy_dz
        pE[2] = be[0] * pE[2] + che[0] * dHz_dx
        pE[3] = be[2] * pE[3] + che[2] * dHx_dz
        pE[4] = be[0] * pE[4] + che[0] * dHy_dx
        pE[5] = be[1] * pE[5] + che[1] * dHx_dy
        Ex = Ex + cex * (dHz_dy / (ke[1] * dl) + pE[0] - dHy_dz / (ke[2] * dl) - pE[1])
        Ey = Ey + cey * (dHx_dz / (ke[2] * dl) + pE[3] - dHz_dx / (ke[0] * dl) - pE[2])
        Ez = Ez + cez * (dHy_dx / (ke[0] * dl) + pE[4] - dHx_dy / (ke[1] * dl) - pE[5])
        t += dt
        E = (Ex, Ey, Ez)
        for s, c in enumerate(comps):
            v = E[c][sl]
            for f in range(nf):
                re[s][f] = re[s][f] + v * float(phases[n, f].real)
                im[s][f] = im[s][f] + v * float(phases[n, f].imag)
    J = 0.0
    for s in range(len(comps)):
        for f in range(nf):
            J = J + (re[s][f] ** 2 + im[s][f] ** 2).sum()
    D = torch.stack([torch.stack([torch.complex(re[s][f], im[s][f]) for f in range(nf)])
                     for s in range(len(comps))])
    return J, D
