"""Pin the CPU oracle against the reference's golden vectors (CPU only).

The oracle is the checker for every CUDA parity test, so it is itself pinned
here: against the reference's committed OpenCL arrays, against fields produced
by the reference's own NumPy engines, and (when ``oracle/_ref`` was built from
the reference tree) bit-for-bit against the reference kernels compiled as C.
"""

from __future__ import annotations

import warnings

import numpy as np
import pytest

from oracle import dft_oracle as D
from oracle import host_math as hm
from oracle.cpu_fdtd import OracleFDTD, ref_available
from tests.cases import (
    PLANE_CASES,
    drive_plane_case,
    farfield_case_setup,
    gaussian_sine,
    peak_err,
    sphere_eps,
)

warnings.simplefilter("ignore", DeprecationWarning)
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


@pytest.mark.parametrize("case", sorted(PLANE_CASES))
def test_oracle_matches_opencl_golden_planes(golden, case):
    c = PLANE_CASES[case]
    sim = OracleFDTD(c["shape"], c["dl"], npml=c["npml"])
    got = drive_plane_case(sim, case)
    for step, plane in got.items():
        ref = golden["planes"][f"{case}_{step:04d}"]
        # POCL fused multiply-adds; this oracle rounds every operation: ≤ 4e-7 seen
        assert peak_err(plane, ref) < 1e-6, (case, step)


@pytest.mark.parametrize("dielectric", [False, True])
def test_oracle_matches_opencl_golden_farfield(golden, dielectric):
    tag = "dielectric_sphere_farfield" if dielectric else "vacuum_farfield"
    sim = OracleFDTD((30, 30, 30), 2e-3, npml=6)
    farfield_case_setup(sim, dielectric)
    mon = D.OracleNear2FarMonitor(sim, (30e-3,) * 3, (20e-3,) * 3, 5e9)
    sim.run(500)
    g = golden["farfield"]
    for key, pt in (("ocl_eh_plus_z", (0, 0, 10.0)), ("ocl_eh_plus_x", (10.0, 0, 0))):
        ref = g[f"{tag}_{key}"]
        # with the reference's float32 k·r prefactor the restatement matches to ~4e-7
        assert peak_err(mon.get_farfield(pt, reference_fp32_k=True), ref) < 2e-6
        # in float64 the only difference is that global phase: ≤ 3e-5 (reference gate 1e-4)
        assert peak_err(mon.get_farfield(pt), ref) < 1e-4
    ang, db = mon.farfield_polar_xz(distance_m=10.0, n_angles=19)
    np.testing.assert_allclose(ang, g[f"{tag}_angles_deg"], atol=1e-12)
    np.testing.assert_allclose(db, g[f"{tag}_ocl_S_db"], rtol=1e-5, atol=1e-4)


def test_oracle_matches_numpy_reference_sphere(golden):
    """Reference ``tests/test_solver.py:48-111`` case against the reference NumPy engines."""
    shape, npml = (30, 30, 30), 6
    sim = OracleFDTD(shape, 2e-3, npml=npml)
    sim.set_epsilon(sphere_eps(shape, 15, 6, 4.0))
    z_src = shape[2] - npml - 2
    sim.add_source(lambda f: f.add_source_Ex(z_src, np.sin(2 * np.pi * 5e9 * f.t)))
    sim.run(50)
    for name in FIELDS:
        for tag in ("np_sphere", "npface_sphere"):
            ref = golden["numpy"][f"{tag}_{name}"]
            assert peak_err(getattr(sim, name), ref) < 1e-5, (tag, name)
            assert np.max(np.abs(getattr(sim, name) - ref)) < 1e-4  # reference gate


def test_oracle_fp64_matches_numpy_reference(golden):
    """Reference ``tests/test_unit_engine.py:340-370``: FP64 within 1e-12 absolute."""
    shape, npml = (24, 24, 24), 4
    sim = OracleFDTD(shape, 2e-3, npml=npml, dtype=np.float64)
    z = shape[2] - npml - 2
    sim.add_source(lambda f: f.add_source_Jx(z, np.sin(2 * np.pi * 4e9 * f.t)))
    sim.run(40)
    for name in FIELDS:
        ref = golden["numpy"][f"np64_jx_{name}"]
        assert np.max(np.abs(getattr(sim, name) - ref)) < 1e-12, name


def test_oracle_taper_matches_numpy_reference(golden):
    """Reference ``tests/test_unit_engine.py:438-474`` (Jx rim taper + renorm)."""
    shape, z = (20, 20, 20), 10
    eps = np.ones(shape, np.float32)
    eps[8:12, 8:12, z] = 2.5
    sim = OracleFDTD(shape, 1e-3, npml=3)
    sim.set_epsilon(eps)
    sim.add_source(lambda f: f.add_source_Jx(z, 0.4, i0=3, i1=17, j0=3, j1=17, rim_taper=True,
                                             rim_edge=0.8, rim_renorm=True))
    sim.run(15)
    for name in FIELDS:
        ref = golden["numpy"][f"np_taper_{name}"]
        assert peak_err(getattr(sim, name), ref) < 1e-5, name


def test_oracle_small_config_with_plane_dft(golden):
    """64³ vacuum, npml 8, Courant 0.5, Jx point, 500 steps, z=32 DFT at 25/30/35 GHz."""
    sim = OracleFDTD((64, 64, 64), 1e-3, npml=8, courant=0.5)
    assert sim.dt == float(golden["numpy"]["small_dt"])
    sim.add_source(lambda f: f.add_source_Jx(32, gaussian_sine(f.t, 30e9, 20e9),
                                             i0=32, i1=33, j0=32, j1=33))
    mon = D.OraclePlaneDFTMonitor(sim, "z", 32, [25e9, 30e9, 35e9], ("Ex", "Hy"))
    run_peak = {"Ex": 0.0, "Hy": 0.0}

    def track(f):
        for c in run_peak:
            run_peak[c] = max(run_peak[c], float(np.max(np.abs(getattr(f, c)))))

    sim.add_monitor(track)
    sim.run(500)
    g = golden["numpy"]
    # By step 500 the pulse has left the box (|Hy| has decayed ~4000x from its peak),
    # so errors are normalised by each field's peak over the run.  The NumPy engine
    # divides by κ·dl where the OpenCL kernels multiply by 1/(κ·dl); that alone
    # separates the two reference engines at the 1e-7 level.
    for c in ("Ex", "Hy"):
        err = np.max(np.abs(getattr(sim, c) - g[f"small_{c}"])) / run_peak[c]
        assert err < 1e-5, (c, err)
    for c in ("Ex", "Hy"):
        for f in range(3):
            assert peak_err(mon.dft[c][f], g[f"small_dft_{c}"][f]) < 1e-5, (c, f)


@pytest.mark.skipif(not ref_available(), reason="reference kernels were not compiled here")
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("npml", [0, 1, 5])
def test_oracle_bit_exact_vs_reference_kernels(dtype, npml):
    """C restatement vs the reference's yee_update.cl/sources.cl compiled as C: identical bits."""
    shape = (19, 23, 17)
    eps = sphere_eps(shape, 9, 5, 3.0)
    sims = [OracleFDTD(shape, 2e-3, npml=npml, dtype=dtype, backend=b) for b in ("oracle", "ref")]
    for s in sims:
        s.set_epsilon(eps)
        s.add_source(lambda f: f.add_source_Jx(8, gaussian_sine(f.t, 5e9, 1e9), i0=2, i1=15,
                                               j0=3, j1=20, rim_taper=True))
        s.add_source(lambda f: f.add_source_Ex(11, 0.01 * np.sin(1e10 * f.t), i0=4, i1=9))
        s.run(30)
    for name in FIELDS:
        assert np.array_equal(getattr(sims[0], name), getattr(sims[1], name)), name


@pytest.mark.skipif(not ref_available(), reason="reference kernels were not compiled here")
def test_oracle_bit_exact_vs_reference_kernels_lossy():
    shape = (16, 14, 18)
    rng = np.random.default_rng(3)
    eps = rng.uniform(1, 6, shape).astype(np.float32)
    sig = rng.uniform(0, 30, shape)
    sims = [OracleFDTD(shape, 1e-3, npml=3, backend=b) for b in ("oracle", "ref")]
    for s in sims:
        s.set_epsilon(eps, sigma_array=sig)
        s.add_source(lambda f: f.add_source_Jx(7, gaussian_sine(f.t, 30e9, 20e9)))
        s.run(25)
    for name in FIELDS:
        assert np.array_equal(getattr(sims[0], name), getattr(sims[1], name)), name


def test_oracle_host_math_matches_reference_arrays(golden):
    g = golden["numpy"]
    for tag in ("p0", "p1", "p2", "p3"):
        meta = g[f"cpml_{tag}_meta"]
        shape = tuple(int(v) for v in meta[:3])
        npml, dl, dt = int(meta[3]), float(meta[4]), float(meta[5])
        dtype = np.float64 if meta[6] else np.float32
        prof = hm.cpml_all(shape, npml, dl, dt, dtype)
        for st in ("e", "h"):
            for ax in range(3):
                b, c, _, kap = prof[st][ax]
                assert np.array_equal(b, g[f"cpml_{tag}_{st}{ax}_b"])
                assert np.array_equal(c, g[f"cpml_{tag}_{st}{ax}_c"])
                assert np.array_equal(kap, g[f"cpml_{tag}_{st}{ax}_kappa"])
    for dtype, tag in ((np.float32, "f32"), (np.float64, "f64")):
        ce = hm.edge_ce(g["mat_eps"], 1e-12, dtype)
        ca, cb = hm.edge_ca_cb(g["mat_eps"], g["mat_sig"], 1e-12, dtype)
        for ax in range(3):
            assert np.array_equal(ce[ax], g[f"mat_ce_{tag}_{ax}"])
            assert np.array_equal(ca[ax], g[f"mat_ca_{tag}_{ax}"])
            assert np.array_equal(cb[ax], g[f"mat_cb_{tag}_{ax}"])


def test_plane_dft_phase_recurrence_matches_closed_form():
    """Reference ``tests/test_unit_monitors.py:95-109``: recurrence stays ≈ e^{jωt}·dt."""
    rec = D.PhaseRecurrence([3e9], 1.9e-12)
    t = 0.0
    for _ in range(5000):
        t += 1.9e-12
        pe, _ = rec.next(t)
    expect = np.exp(1j * 2 * np.pi * 3e9 * t) * 1.9e-12
    assert abs(pe[0] - expect) / abs(expect) < 1e-9
