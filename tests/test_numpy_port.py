"""The NumPy face-CPML restatement (``oracle/numpy_face_cpml.py``) against the
reference's own ``NumPyFDTD_FaceCPML`` (CPU).

The fixtures in ``tests/golden/numpy_ref.npz`` were made by importing the
reference engine (``tests/golden/make_golden.py``): the FP32 sphere case of
reference ``tests/test_solver.py:48-85`` (50 steps, soft Ex sheet) and the small
configuration (64³, npml 8, Courant 0.5, Jx point at the centre, 500 steps,
z = 32 plane DFT at 25/30/35 GHz).  The restatement keeps the reference's array
operations and their order, so the fields are equal bit for bit.  This is the
engine ``bench.py`` times as the NumPy CPU baseline and runs in FP64 for the
FP32-vs-FP64 error statements.
"""

from __future__ import annotations

import numpy as np

from oracle.numpy_face_cpml import NumPyFaceCPML
from tests.cases import gaussian_sine, sphere_eps

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def test_sphere_case_bit_identical(golden):
    ref = golden["numpy"]
    shape, npml = (30, 30, 30), 6
    sim = NumPyFaceCPML(shape, 2e-3, npml=npml)
    sim.set_epsilon(sphere_eps(shape, 15, 6, 4.0))
    z = shape[2] - npml - 2
    sim.add_source(lambda f: f.add_source_Ex(z, np.sin(2 * np.pi * 5e9 * f.t)))
    sim.run(50)
    for n in FIELDS:
        want = ref[f"npface_sphere_{n}"]
        assert np.abs(want).max() > 0, n
        assert np.array_equal(getattr(sim, n), want), n


def test_small_config_bit_identical(golden):
    ref = golden["numpy"]
    sim = NumPyFaceCPML((64, 64, 64), 1e-3, npml=8, courant=0.5)
    assert sim.dt == float(ref["small_dt"])
    sim.add_source(lambda f: f.add_source_Jx(32, gaussian_sine(f.t, 30e9, 20e9),
                                             i0=32, i1=33, j0=32, j1=33))
    omega = 2 * np.pi * np.array([25e9, 30e9, 35e9])
    acc = {c: np.zeros((3, 64, 64), np.complex128) for c in ("Ex", "Hy")}
    st = {"p": None}

    def plane(f):
        st["p"] = (np.exp(1j * omega * f.t) * f.dt if st["p"] is None
                   else st["p"] * np.exp(1j * omega * f.dt))
        ph = st["p"] * np.exp(-0.5j * omega * f.dt)
        acc["Ex"] += st["p"][:, None, None] * f.Ex[:, :, 32].astype(np.float64)[None]
        acc["Hy"] += ph[:, None, None] * f.Hy[:, :, 32].astype(np.float64)[None]

    sim.add_monitor(plane)
    sim.run(500)
    assert np.array_equal(sim.Ex, ref["small_Ex"])
    assert np.array_equal(sim.Hy, ref["small_Hy"])
    assert np.array_equal(acc["Ex"], ref["small_dft_Ex"])
    assert np.array_equal(acc["Hy"], ref["small_dft_Hy"])
