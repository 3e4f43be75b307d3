"""Yee-edge material coefficients (host side).

Cell-centred ``εr`` (and optional conductivity ``σ``) are sampled onto the three
E-edge staggers by the two-cell arithmetic mean used by the reference
(``opencl_fdtd_solver/materials.py:28-41``): ``Ex`` at ``(i+½, j, k)`` averages
cells ``i`` and ``i+1``; the last plane along the stagger axis keeps the cell
value.  Coefficients are evaluated in float64 and rounded once to the field
dtype (``materials.py:45-55`` and ``:59-88``).

The same map is differentiated by the adjoint: ``ce = dt/(ε0·ε_edge)`` so
``∂ce/∂ε_edge = −ce/ε_edge`` and each cell feeds ½ of that into the (up to) two
edges of each component that it touches.
"""

from __future__ import annotations

import numpy as np

from .constants import EPS0


def _edge_mean(a: np.ndarray, axis: int) -> np.ndarray:
    out = np.array(a, dtype=np.float64, copy=True)
    lo = [slice(None)] * 3
    hi = [slice(None)] * 3
    lo[axis] = slice(0, -1)
    hi[axis] = slice(1, None)
    out[tuple(lo)] = 0.5 * (out[tuple(lo)] + np.asarray(a, dtype=np.float64)[tuple(hi)])
    return out


def yee_edge_eps(eps_r: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Edge permittivities ``(εx, εy, εz)`` in float64."""
    eps = np.asarray(eps_r, dtype=np.float64)
    return _edge_mean(eps, 0), _edge_mean(eps, 1), _edge_mean(eps, 2)


def yee_edge_ce(eps_r: np.ndarray, dt: float, dtype=np.float32):
    """Lossless E-update coefficients ``ce = dt/(ε0·ε_edge)`` per component."""
    scale = float(dt) / EPS0
    dt_t = np.dtype(dtype)
    return tuple((scale / e).astype(dt_t) for e in yee_edge_eps(eps_r))


def yee_edge_ca_cb(eps_r: np.ndarray, sigma: np.ndarray, dt: float, dtype=np.float32):
    """Lossy (trapezoidal) coefficients ``((ca_x, ca_y, ca_z), (cb_x, cb_y, cb_z))``.

    ``E ← ca·E + cb·curl H`` with ``loss = σ·dt/(2ε0·ε)``, ``ca = (1−loss)/(1+loss)``
    and ``cb = dt/(ε0·ε)/(1+loss)``; ``σ ≡ 0`` gives ``ca = 1`` and ``cb = ce``.
    """
    dt_f = float(dt)
    dt_t = np.dtype(dtype)
    cas, cbs = [], []
    for e, s in zip(yee_edge_eps(eps_r), yee_edge_eps(sigma)):
        loss = s * dt_f / (2.0 * EPS0 * e)
        denom = 1.0 + loss
        cas.append(((1.0 - loss) / denom).astype(dt_t))
        cbs.append(((dt_f / (EPS0 * e)) / denom).astype(dt_t))
    return tuple(cas), tuple(cbs)
