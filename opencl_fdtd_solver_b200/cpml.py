"""CFS-CPML 1-D coefficient profiles (host side, computed once per engine).

The profile arithmetic follows the reference ``opencl_fdtd_solver/cpml.py:52-134``
operation for operation, including its dtype behaviour: ``b`` is evaluated in
float64 and rounded to the field dtype, and ``c`` is then formed from the
*rounded* ``b`` (``b − 1`` in field dtype, the remaining products in float64,
one final rounding; that is what NumPy's scalar promotion does in the reference
loop at ``cpml.py:104-106``).  Getting this bit-identical
matters: ``c`` multiplies every ψ update, so a one-ulp difference in ``c`` shows
up as a field difference after a few hundred steps.

Depth convention (``cpml.py:57-65``): ``node_offset`` is 0 for E-aligned samples
and ½ for H-aligned samples; depth ξ is 1 at the outer wall and 0 at the vacuum
interface.
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np

from .constants import EPS0, ETA0

# Polynomial grading order, κ stretch at the wall and CFS α at the interface
# (reference ``cpml.py:30-34``).
CPML_M = 3
CPML_KAPPA_MAX = 15.0
CPML_ALPHA_MAX_OVER_ETA0 = 0.05


class CpmlAxisProfile(NamedTuple):
    """Per-axis CPML arrays ``b``, ``c``, ``κ`` sampled on one Yee stagger."""

    b: np.ndarray
    c: np.ndarray
    kappa: np.ndarray


class CpmlProfiles(NamedTuple):
    """E-node (offset 0) and H-node (offset ½) profiles for x, y, z."""

    e: tuple[CpmlAxisProfile, CpmlAxisProfile, CpmlAxisProfile]
    h: tuple[CpmlAxisProfile, CpmlAxisProfile, CpmlAxisProfile]


def sigma_max(dl: float, *, m: int = CPML_M) -> float:
    """Taflove's optimum conductivity at the outer PML cell, ``0.8(m+1)/(η0·dl)``."""
    return 0.8 * (m + 1) / (ETA0 * float(dl))


def _depth(npml: int, layer: int, lo: bool, node_offset: float) -> float:
    # Normalised depth of layer ``layer`` (0-based from the wall on the low side,
    # from the interface on the high side).
    if lo:
        return (npml - layer - node_offset) / npml
    return (layer + 1 - node_offset) / npml


def build_cpml_1d(
    n: int,
    *,
    npml: int,
    dl: float,
    dt: float,
    node_offset: float,
    dtype=np.float32,
    m: int | None = None,
    kappa_max: float | None = None,
    alpha_max: float | None = None,
) -> CpmlAxisProfile:
    """1-D ``(b, c, κ)`` of length ``n`` for one stagger (reference ``cpml.py:68-108``)."""
    dtype = np.dtype(dtype)
    m = CPML_M if m is None else m
    kappa_max = CPML_KAPPA_MAX if kappa_max is None else kappa_max
    b = np.ones(n, dtype=dtype)
    c = np.zeros(n, dtype=dtype)
    kappa = np.ones(n, dtype=dtype)
    if npml <= 0 or n <= 0:
        return CpmlAxisProfile(b, c, kappa)
    smax = sigma_max(dl, m=m)
    amax = CPML_ALPHA_MAX_OVER_ETA0 / ETA0 if alpha_max is None else alpha_max
    one = dtype.type(1.0)
    # Cells are visited in the reference order (low face then high face, per
    # layer) so that overlapping faces on grids thinner than 2·npml resolve the
    # same way.
    for layer in range(npml):
        for lo, idx in ((True, layer), (False, n - npml + layer)):
            if idx < 0 or idx >= n:
                continue
            xi = max(_depth(npml, layer, lo, node_offset), 0.0)
            grade = xi**m
            sig = smax * grade
            kap = 1.0 + (kappa_max - 1.0) * grade
            alp = amax * (1.0 - xi)
            bval = dtype.type(np.exp(-((sig / kap + alp) * dt / EPS0)))
            b[idx] = bval
            denom = sig + kap * alp
            if denom == 0:
                c[idx] = 0.0
            else:
                # (b − 1) is taken on the rounded b in field dtype, the rest in
                # float64, then rounded once (see module docstring)
                c[idx] = sig / kap * float(bval - one) / denom / float(dl)
            kappa[idx] = kap
    return CpmlAxisProfile(b, c, kappa)


def build_cpml_profiles(
    shape: tuple[int, int, int],
    *,
    npml: int,
    dl: float,
    dt: float,
    dtype=np.float32,
    m: int | None = None,
    kappa_max: float | None = None,
) -> CpmlProfiles:
    """E-node and H-node profiles for all three axes (reference ``cpml.py:111-134``)."""
    kw = dict(npml=npml, dl=dl, dt=dt, dtype=dtype, m=m, kappa_max=kappa_max)
    dims = [int(v) for v in shape]
    e = tuple(build_cpml_1d(d, node_offset=0.0, **kw) for d in dims)
    h = tuple(build_cpml_1d(d, node_offset=0.5, **kw) for d in dims)
    return CpmlProfiles(e=e, h=h)  # type: ignore[arg-type]


def inverse_kappa_dl(kappa: np.ndarray, dl: float, dtype) -> np.ndarray:
    """``1/(κ·dl)`` evaluated in float64 and rounded once (reference ``engine.py:264-266``)."""
    return (1.0 / (kappa.astype(np.float64) * dl)).astype(dtype)
