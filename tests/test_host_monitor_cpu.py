"""Host Huygens-box monitor (reference ``NumPyNear2FarMonitor``) on the CPU.

The package's vectorised ``NumPyNear2FarMonitor`` is driven by the seeded field
sequences that produced ``tests/golden/host_monitor.npz`` from the reference's
own per-sample loop (``opencl_fdtd_solver/monitors.py:229-295``); the face
arrays must agree bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

from opencl_fdtd_solver_b200 import NumPyNear2FarMonitor
from tests.cases import HOST_MONITOR_CASES, SyntheticFieldSequence
from tests.conftest import GOLDEN

FIELDS = SyntheticFieldSequence.FIELDS


@pytest.fixture(scope="module")
def fixture():
    return np.load(GOLDEN / "host_monitor.npz")


@pytest.mark.parametrize("case", HOST_MONITOR_CASES, ids=[c[0] for c in HOST_MONITOR_CASES])
def test_vectorised_monitor_matches_reference_loop_bitwise(case, fixture):
    tag, shape, dl, dt, seed, center, size, freq, steps = case
    seq = SyntheticFieldSequence(shape, dl, dt, seed)
    mon = NumPyNear2FarMonitor(seq, center, size, freq)
    assert mon._box == tuple(int(v) for v in fixture[f"{tag}_box"])
    for _ in range(steps):
        seq.step()
    for n in FIELDS:
        got = getattr(mon, f"{n}_dft_f")
        want = fixture[f"{tag}_{n}_dft_f"]
        assert got.dtype == np.complex64
        assert np.array_equal(got, want), n
        assert np.abs(want).max() > 0


def test_host_regions_cover_every_read(fixture):
    """Serving reads only inside ``host_regions`` (NaN elsewhere) gives the same sums."""
    tag, shape, dl, dt, seed, center, size, freq, steps = HOST_MONITOR_CASES[1]

    class Windowed(SyntheticFieldSequence):
        def step(self):
            rng = np.random.default_rng([self.seed, self.step_num])
            for n in self.FIELDS:
                full = rng.standard_normal(shape).astype(self.dtype)
                masked = np.full(shape, np.nan, self.dtype)
                for box in mon.host_regions():
                    sl = tuple(slice(a, b) for a, b in box)
                    masked[sl] = full[sl]
                setattr(self, n, masked)
            self.step_num += 1
            self.t += self.dt
            for m in self._monitors:
                m(self)

    seq = Windowed(shape, dl, dt, seed)
    mon = NumPyNear2FarMonitor(seq, center, size, freq)
    for _ in range(steps):
        seq.step()
    for n in FIELDS:
        assert np.array_equal(getattr(mon, f"{n}_dft_f"), fixture[f"{tag}_{n}_dft_f"]), n


def test_empty_box_raises():
    seq = SyntheticFieldSequence((8, 8, 8), 1e-3, 1e-12, 0)
    with pytest.raises(ValueError):
        NumPyNear2FarMonitor(seq, (-50e-3, 4e-3, 4e-3), (1e-3, 1e-3, 1e-3), 1e9)
