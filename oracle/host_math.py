"""Oracle restatement of the reference host-side coefficient math (TEST INFRASTRUCTURE).

Written independently of the product package so that the product's own host math
(``opencl_fdtd_solver_b200/cpml.py``, ``materials.py``) is checked against it:

* CFS-CPML profiles: reference ``opencl_fdtd_solver/cpml.py:52-134``
* ``1/(κ·dl)``: reference ``opencl_fdtd_solver/engine.py:264-266``
* Yee-edge ε and ``ce``/``ca,cb``: reference ``opencl_fdtd_solver/materials.py:28-88``
* constants: reference ``opencl_fdtd_solver/constants.py:11-14``
"""

from __future__ import annotations

import numpy as np

C0 = 299_792_458.0
MU0 = 4e-7 * np.pi
EPS0 = 1.0 / (MU0 * C0**2)
ETA0 = np.sqrt(MU0 / EPS0)  # numpy float64 scalar, as in the reference


def cpml_axis(n, npml, dl, dt, node_offset, dtype, m=3, kappa_max=15.0):
    """Return ``(b, c, kappa)`` for one axis and stagger, in the reference loop order."""
    b = np.ones(n, dtype=dtype)
    c = np.zeros(n, dtype=dtype)
    kappa = np.ones(n, dtype=dtype)
    if npml <= 0 or n <= 0:
        return b, c, kappa
    sig_max = 0.8 * (m + 1) / (ETA0 * float(dl))
    alpha_max = 0.05 / ETA0
    for i in range(npml):
        for lo, idx in ((True, i), (False, n - npml + i)):
            if idx < 0 or idx >= n:
                continue
            xi = (npml - i - node_offset) / npml if lo else (i + 1 - node_offset) / npml
            xi = max(xi, 0.0)
            sig = sig_max * xi**m
            kap = 1.0 + (kappa_max - 1.0) * xi**m
            alp = alpha_max * (1.0 - xi)
            b[idx] = np.exp(-((sig / kap + alp) * dt / EPS0))
            denom = sig + kap * alp
            c[idx] = 0.0 if denom == 0 else sig / kap * (b[idx] - 1.0) / denom / dl
            kappa[idx] = kap
    return b, c, kappa


def cpml_all(shape, npml, dl, dt, dtype):
    """``{'e': [(b, c, ik) x3], 'h': [...]}`` with ``ik = 1/(κ·dl)`` rounded once."""
    out = {}
    for stag, off in (("e", 0.0), ("h", 0.5)):
        axes = []
        for n in shape:
            b, c, kap = cpml_axis(int(n), npml, dl, dt, off, dtype)
            ik = (1.0 / (kap.astype(np.float64) * dl)).astype(dtype)
            axes.append((b, c, ik, kap))
        out[stag] = axes
    return out


def edge_eps(eps):
    eps = np.asarray(eps, dtype=np.float64)
    ex = eps.copy()
    ex[:-1] = 0.5 * (eps[:-1] + eps[1:])
    ey = eps.copy()
    ey[:, :-1] = 0.5 * (eps[:, :-1] + eps[:, 1:])
    ez = eps.copy()
    ez[:, :, :-1] = 0.5 * (eps[:, :, :-1] + eps[:, :, 1:])
    return ex, ey, ez


def edge_ce(eps, dt, dtype):
    scale = float(dt) / EPS0
    return tuple((scale / e).astype(dtype) for e in edge_eps(eps))


def edge_ca_cb(eps, sigma, dt, dtype):
    cas, cbs = [], []
    for e, s in zip(edge_eps(eps), edge_eps(sigma)):
        loss = s * float(dt) / (2.0 * EPS0 * e)
        cas.append(((1.0 - loss) / (1.0 + loss)).astype(dtype))
        cbs.append(((float(dt) / (EPS0 * e)) / (1.0 + loss)).astype(dtype))
    return tuple(cas), tuple(cbs)
