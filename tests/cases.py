"""Case builders shared by the oracle and the CUDA parity tests.

Each mirrors a reference test or fixture case (cited per function); the same
builder drives both engines so that inputs are identical.
"""

from __future__ import annotations

import numpy as np


def gaussian_sine(t, f0, fwidth):
    """Reference waveform ``tests/meep_validation/harness.py:70-73``."""
    t0 = 5.0 / (np.pi * fwidth)
    sigma = 1.0 / (np.pi * fwidth)
    return float(np.exp(-0.5 * ((t - t0) / sigma) ** 2) * np.sin(2 * np.pi * f0 * t))


def gaussian_pulse(t, fwidth):
    """Gaussian envelope of ``gaussian_sine`` without the carrier."""
    t0 = 5.0 / (np.pi * fwidth)
    sigma = 1.0 / (np.pi * fwidth)
    return float(np.exp(-0.5 * ((t - t0) / sigma) ** 2))


def sphere_eps(shape, ctr, rad, eps_r):
    """Staircased sphere on cell centres (``<`` test), reference ``tests/test_solver.py:39-46``."""
    ii, jj, kk = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    eps = np.ones(shape, np.float32)
    eps[(ii - ctr) ** 2 + (jj - ctr) ** 2 + (kk - ctr) ** 2 < rad**2] = eps_r
    return eps


def block_eps(shape, half, eps_r):
    """Centred block, reference ``tests/meep_validation/plane_cases.py:98-111``."""
    eps = np.ones(shape, np.float32)
    nx, ny, nz = shape
    hx, hy, hz = half
    ci, cj, ck = nx // 2, ny // 2, nz // 2
    eps[ci - hx:ci + hx + 1, cj - hy:cj + hy + 1, ck - hz:ck + hz + 1] = eps_r
    return eps


def blocky_eps(shape, block=8, lo=1.0, hi=12.0, seed=1234):
    """εr ~ U[lo, hi] per ``block``³ cells (seeded), the bandwidth-roofline medium."""
    rng = np.random.default_rng(seed)
    nb = [-(-n // block) for n in shape]
    vals = rng.uniform(lo, hi, nb).astype(np.float32)
    e = np.repeat(np.repeat(np.repeat(vals, block, 0), block, 1), block, 2)
    return np.ascontiguousarray(e[: shape[0], : shape[1], : shape[2]])


PLANE_CASES = {
    # reference tests/meep_validation/plane_cases.py:62-91
    "vacuum_sheet": dict(shape=(32, 32, 40), dl=2.5e-3, npml=4, block=None),
    "dielectric_block": dict(shape=(32, 32, 40), dl=2.5e-3, npml=4, block=(6, 6, 4)),
}


def drive_plane_case(sim, name, steps=(20, 40, 60, 80)):
    """Run a golden plane case on ``sim``; return ``{step: Ex[:, Ny//2, :]}``."""
    c = PLANE_CASES[name]
    nx, ny, nz = c["shape"]
    p = c["npml"]
    if c["block"] is not None:
        sim.set_epsilon(block_eps(c["shape"], c["block"], 4.0))
    z_src = nz - p - 2

    def src(f):
        f.add_source_Jx(z_src, gaussian_sine(f.t, 5e9, 1e9), i0=p, i1=nx - p, j0=p, j1=ny - p,
                        rim_taper=True)

    sim.add_source(src)
    out = {}
    for s in range(1, max(steps) + 1):
        sim.step()
        if s in steps:
            out[s] = np.asarray(sim.Ex)[:, ny // 2, :].astype(np.float64)
    return out


def farfield_case_setup(sim, dielectric):
    """Reference ``tests/meep_validation/cases.py:24-83``: 30³, 5×5 soft Ex patch at the centre."""
    if dielectric:
        sim.set_epsilon(sphere_eps((30, 30, 30), 15, 4, 4.0))
    sim.add_source(lambda f: f.add_source_Ex(15, gaussian_sine(f.t, 5e9, 1e9),
                                             i0=13, i1=18, j0=13, j1=18))


def peak_err(a, b):
    """``max|a − b| / max|b|`` (peak-normalised), 0 when both are zero."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = float(np.max(np.abs(b)))
    num = float(np.max(np.abs(a - b)))
    return num / den if den > 0 else num


class SyntheticFieldSequence:
    """Engine stand-in that serves seeded random fields, one set per step.

    It has the attributes a host monitor reads (``Nx, Ny, Nz, dl, dt, t``,
    ``Ex … Hz``, ``add_monitor``), so the reference's ``NumPyNear2FarMonitor``
    and this package's can be driven by identical inputs without a solver.
    Step ``n`` draws from ``default_rng([seed, n])``.
    """

    FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")

    def __init__(self, shape, dl, dt, seed, dtype=np.float32):
        self.Nx, self.Ny, self.Nz = (int(v) for v in shape)
        self.dl, self.dt, self.t = float(dl), float(dt), 0.0
        self.dtype = np.dtype(dtype)
        self.seed = int(seed)
        self.step_num = 0
        self._monitors = []
        for n in self.FIELDS:
            setattr(self, n, np.zeros((self.Nx, self.Ny, self.Nz), self.dtype))

    def add_monitor(self, mon):
        self._monitors.append(mon)
        return mon

    def step(self):
        rng = np.random.default_rng([self.seed, self.step_num])
        for n in self.FIELDS:
            setattr(self, n, rng.standard_normal((self.Nx, self.Ny, self.Nz)).astype(self.dtype))
        self.step_num += 1
        self.t += self.dt
        for mon in self._monitors:
            mon(self)


# Host-monitor fixture cases: (tag, shape, dl, dt, seed, center, size, freq, steps).
# "inner" keeps the box away from the grid edges; "edge" snaps it to the whole
# grid, so every clamp of the co-location means (i+1, j+1, k+1 at the high edge,
# i-1 at index 0) is exercised.
HOST_MONITOR_CASES = (
    ("inner", (12, 14, 16), 2e-3, 3.1e-12, 11, (12e-3, 14e-3, 16e-3), (10e-3, 12e-3, 14e-3),
     5e9, 6),
    ("edge", (9, 10, 11), 1e-3, 1.7e-12, 12, (4.5e-3, 5e-3, 5.5e-3), (20e-3, 20e-3, 20e-3),
     8e9, 5),
)
