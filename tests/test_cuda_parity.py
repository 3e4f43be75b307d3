"""CUDA engine parity against the CPU oracle and the reference's golden vectors (GPU).

Every case is driven identically on ``CUDAFDTD`` (through the C ABI of
``libfdtd_b200.so``) and on ``OracleFDTD`` (the C restatement of the reference
kernels).  The Yee kernels are compiled without FMA contraction, so FP32 and
FP64 fields are expected to be bit-identical to the oracle; the north-star
tolerance (peak-normalised 1e-5 FP32, 1e-12 FP64) is asserted against the
reference's own arrays.
"""

from __future__ import annotations

import logging
import warnings

import numpy as np
import pytest

from oracle import dft_oracle as D
from oracle.cpu_fdtd import OracleFDTD
from tests.cases import (
    PLANE_CASES,
    block_eps,
    blocky_eps,
    drive_plane_case,
    farfield_case_setup,
    gaussian_pulse,
    gaussian_sine,
    peak_err,
    sphere_eps,
)

pytestmark = pytest.mark.gpu
warnings.simplefilter("ignore", DeprecationWarning)
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import opencl_fdtd_solver_b200 as pkg

    return pkg


def both(cuda, shape, dl, npml, dtype=np.float32, courant=None, fused=True):
    g = cuda.CUDAFDTD(shape, dl, npml=npml, dtype=dtype, courant=courant, fused=fused)
    o = OracleFDTD(shape, dl, npml=npml, dtype=dtype, courant=courant)
    return g, o


def assert_same(g, o, exact=True, tol=0.0):
    for n in FIELDS:
        a, b = getattr(g, n), getattr(o, n)
        assert a.dtype == b.dtype and a.shape == b.shape
        if exact:
            d = np.max(np.abs(a.astype(np.float64) - b))
            assert np.array_equal(a, b), f"{n}: max |diff| {d:.3e}"
        else:
            assert peak_err(a, b) <= tol, (n, peak_err(a, b))


@pytest.mark.parametrize("case", sorted(PLANE_CASES))
def test_golden_planes(cuda, case):
    c = PLANE_CASES[case]
    g, o = both(cuda, c["shape"], c["dl"], c["npml"])
    got = drive_plane_case(g, case)
    ref = drive_plane_case(o, case)
    for step in got:
        assert np.array_equal(got[step], ref[step]), (case, step)
    import tests.conftest as cf

    gold = np.load(cf.GOLDEN / "ocl_planes.npz")
    for step, plane in got.items():
        assert peak_err(plane, gold[f"{case}_{step:04d}"]) < 1e-6


@pytest.mark.parametrize("fused", [True, False])
def test_sphere_ex_sheet_vs_oracle_and_numpy(cuda, golden, fused):
    """Reference ``tests/test_solver.py:48-111``: εr=4 sphere, full-sheet Ex source, 50 steps."""
    shape, npml = (30, 30, 30), 6
    g, o = both(cuda, shape, 2e-3, npml, fused=fused)
    eps = sphere_eps(shape, 15, 6, 4.0)
    z_src = shape[2] - npml - 2
    for s in (g, o):
        s.set_epsilon(eps)
        s.add_source(lambda f: f.add_source_Ex(z_src, np.sin(2 * np.pi * 5e9 * f.t)))
        s.run(50)
    assert_same(g, o)
    for n in FIELDS:
        ref = golden["numpy"][f"np_sphere_{n}"]
        assert peak_err(getattr(g, n), ref) < 1e-5
        assert np.max(np.abs(getattr(g, n) - ref)) < 1e-4


def test_fp64_jx_vs_numpy_reference(cuda, golden):
    """Reference ``tests/test_unit_engine.py:340-370``: FP64 within 1e-12 absolute."""
    shape, npml = (24, 24, 24), 4
    g, o = both(cuda, shape, 2e-3, npml, dtype=np.float64)
    z = shape[2] - npml - 2
    for s in (g, o):
        s.add_source(lambda f: f.add_source_Jx(z, np.sin(2 * np.pi * 4e9 * f.t)))
        s.run(40)
    assert_same(g, o)
    for n in FIELDS:
        assert np.max(np.abs(getattr(g, n) - golden["numpy"][f"np64_jx_{n}"])) < 1e-12


def test_rim_taper_renorm_vs_numpy_reference(cuda, golden):
    """Reference ``tests/test_unit_engine.py:438-474``."""
    shape, z = (20, 20, 20), 10
    eps = np.ones(shape, np.float32)
    eps[8:12, 8:12, z] = 2.5
    g, o = both(cuda, shape, 1e-3, 3)
    for s in (g, o):
        s.set_epsilon(eps)
        s.add_source(lambda f: f.add_source_Jx(z, 0.4, i0=3, i1=17, j0=3, j1=17, rim_taper=True,
                                               rim_edge=0.8, rim_renorm=True))
        s.run(15)
    assert_same(g, o)
    for n in FIELDS:
        assert peak_err(getattr(g, n), golden["numpy"][f"np_taper_{n}"]) < 1e-5


def test_jx_known_answer(cuda):
    """Reference ``tests/test_unit_engine.py:183-207``: −dt/(ε0·2.5)·J at an averaged edge."""
    from opencl_fdtd_solver_b200.constants import EPS0

    shape, z, Jx, p = (16, 16, 16), 8, 0.25, 2
    g = cuda.CUDAFDTD(shape, 1e-3, npml=p)
    eps = np.ones(shape, np.float32)
    eps[8, 8, z] = 4.0
    g.set_epsilon(eps)
    g.add_source(lambda f: f.add_source_Jx(z, Jx, i0=p, i1=shape[0] - p, j0=p, j1=shape[1] - p))
    g.step()
    ex = g.Ex
    assert ex[8, 8, z] == pytest.approx(-g.dt / (EPS0 * 2.5) * Jx, abs=1e-6)
    assert ex[p, p, z] == pytest.approx(-g.dt / EPS0 * Jx, abs=1e-6)
    assert ex[0, 0, z] == 0.0


def test_rim_taper_weights(cuda):
    """Reference ``tests/test_unit_engine.py:209-243``: 1, r, r² without renorm."""
    from opencl_fdtd_solver_b200.constants import EPS0

    shape, p, z, ew = (16, 16, 16), 2, 8, 0.5
    i1, j1 = shape[0] - p, shape[1] - p
    g = cuda.CUDAFDTD(shape, 1e-3, npml=p)
    g.add_source(lambda f: f.add_source_Jx(z, 1.0, i0=p, i1=i1, j0=p, j1=j1, rim_taper=True,
                                           rim_edge=ew, rim_renorm=False))
    g.step()
    ex = g.Ex
    base = -g.dt / EPS0
    assert ex[p + 2, p + 2, z] == pytest.approx(base, abs=1e-6)
    assert ex[p, p + 2, z] == pytest.approx(ew * base, abs=1e-6)
    assert ex[p + 2, p, z] == pytest.approx(ew * base, abs=1e-6)
    assert ex[p, p, z] == pytest.approx(ew * ew * base, abs=1e-6)
    assert ex[i1 - 1, j1 - 1, z] == pytest.approx(ew * ew * base, abs=1e-6)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape,npml", [((37, 41, 53), 3), ((19, 23, 17), 1), ((20, 20, 20), 0),
                                        ((9, 7, 5), 2), ((33, 8, 64), 5)])
def test_odd_shapes_vs_oracle(cuda, shape, npml, dtype):
    g, o = both(cuda, shape, 1e-3, npml, dtype=dtype)
    rng = np.random.default_rng(11)
    eps = rng.uniform(1, 5, shape).astype(np.float32)
    zc = shape[2] // 2
    for s in (g, o):
        s.set_epsilon(eps)
        s.add_source(lambda f: f.add_source_Jx(zc, gaussian_sine(f.t, 40e9, 30e9),
                                               i0=1, i1=shape[0] - 1, j0=1, j1=shape[1] - 1,
                                               rim_taper=True))
        s.add_source(lambda f: f.add_source_Ex(max(0, zc - 1), 1e-3 * np.cos(3e10 * f.t),
                                               i0=2, i1=4, j0=0, j1=2))
        s.run(25)
    assert_same(g, o)


@pytest.mark.parametrize("fused", [True, False])
def test_lossy_vs_oracle(cuda, fused):
    """Lossy E update (``materials.py:59-88``, ``engine.py:242-254``)."""
    shape = (24, 24, 60)
    sig = np.zeros(shape)
    sig[:, :, 40:] = 100.0
    eps = np.ones(shape, np.float32)
    g, o = both(cuda, shape, 1e-3, 8, fused=fused)
    for s in (g, o):
        s.set_epsilon(eps, sigma_array=sig)
        s.add_source(lambda f: f.add_source_Ex(15, 0.1 * np.sin(2 * np.pi * 10e9 * f.t)))
        s.run(120)
    assert_same(g, o)


def test_sigma_zero_matches_lossless(cuda):
    """Reference ``tests/test_materials_lossy.py:133-145``."""
    shape = (24, 24, 60)
    a = cuda.CUDAFDTD(shape, 1e-3, npml=8)
    b = cuda.CUDAFDTD(shape, 1e-3, npml=8)
    eps = np.ones(shape, np.float32)
    a.set_epsilon(eps, sigma_array=np.zeros(shape))
    b.set_epsilon(eps)
    for s in (a, b):
        s.add_source(lambda f: f.add_source_Ex(15, 0.1 * np.sin(2 * np.pi * 10e9 * f.t)))
        s.run(100)
    np.testing.assert_allclose(a.Ex, b.Ex, atol=1e-12)


def test_lossy_reflection_monotone(cuda):
    """Reference ``tests/test_materials_lossy.py:147-176``."""
    before, inside = [], []
    for sv in (20.0, 100.0, 300.0):
        g = cuda.CUDAFDTD((24, 24, 60), 1e-3, npml=8)
        sig = np.zeros((24, 24, 60))
        sig[:, :, 40:] = sv
        g.set_epsilon(np.ones((24, 24, 60), np.float32), sigma_array=sig)
        g.add_source(lambda f: f.add_source_Ex(15, 0.1 * np.sin(2 * np.pi * 10e9 * f.t)))
        g.run(400)
        ex = g.Ex
        before.append(abs(ex[12, 12, 35]))
        inside.append(abs(ex[12, 12, 55]))
    assert before == sorted(before)
    assert inside[0] > inside[1] > inside[2]


def test_fused_equals_split(cuda):
    shape = (40, 36, 64)
    eps = blocky_eps(shape, block=4, seed=5)
    runs = []
    for fused in (True, False):
        g = cuda.CUDAFDTD(shape, 1e-3, npml=6, fused=fused)
        g.set_epsilon(eps)
        g.add_source(lambda f: f.add_source_Jx(30, gaussian_sine(f.t, 30e9, 20e9), i0=18, i1=19,
                                               j0=17, j1=18))
        m = cuda.CUDAPlaneDFTMonitor(g, "x", 20, [25e9, 35e9], ("Ez", "Hx"))
        g.run(60)
        runs.append(({n: getattr(g, n) for n in FIELDS}, m.dft("Ez"), m.dft("Hx")))
    for n in FIELDS:
        assert np.array_equal(runs[0][0][n], runs[1][0][n]), n
    assert np.array_equal(runs[0][1], runs[1][1])
    assert np.array_equal(runs[0][2], runs[1][2])


def test_callback_touching_fields_uses_split_step(cuda):
    """A source callback that reads and writes E (host read-modify-write, as in reference
    ``tests/meep_validation/cases.py:57-66``) sees the reference state."""
    shape = (30, 30, 30)
    g, o = both(cuda, shape, 2e-3, 6)

    def rmw(f):
        ex = f.Ex
        ex[13:18, 13:18, 15] += np.float32(gaussian_sine(f.t, 5e9, 1e9))
        f.Ex = ex

    def rmw_oracle(f):
        f.Ex[13:18, 13:18, 15] += np.float32(gaussian_sine(f.t, 5e9, 1e9))

    g.add_source(rmw)
    o.add_source(rmw_oracle)
    g.run(40)
    o.run(40)
    assert_same(g, o)


def test_small_config_fields_and_plane_dft(cuda, golden):
    """64³ vacuum, npml 8, Courant 0.5, Jx point, 500 steps, z=32 DFT at 25/30/35 GHz."""
    g, o = both(cuda, (64, 64, 64), 1e-3, 8, courant=0.5)
    mons = []
    for s in (g, o):
        s.add_source(lambda f: f.add_source_Jx(32, gaussian_sine(f.t, 30e9, 20e9),
                                               i0=32, i1=33, j0=32, j1=33))
    mg = cuda.CUDAPlaneDFTMonitor(g, "z", 32, [25e9, 30e9, 35e9], ("Ex", "Hy"))
    mo = D.OraclePlaneDFTMonitor(o, "z", 32, [25e9, 30e9, 35e9], ("Ex", "Hy"))
    peak = {"Ex": 0.0, "Hy": 0.0}

    def track(f):
        for c in peak:
            peak[c] = max(peak[c], float(f.field_tensor(c).abs().max()))

    g.add_monitor(track)
    g.run(500)
    o.run(500)
    assert_same(g, o)
    nref = golden["numpy"]
    for c in ("Ex", "Hy"):
        assert np.array_equal(mg.dft(c), mo.dft[c])
        assert np.max(np.abs(getattr(g, c) - nref[f"small_{c}"])) / peak[c] < 1e-5
        for f in range(3):
            assert peak_err(mg.dft(c)[f], nref[f"small_dft_{c}"][f]) < 1e-5


@pytest.mark.parametrize("axis,comps", [(0, ("Ey", "Hz")), (1, ("Ex", "Ez", "Hx")),
                                        (2, FIELDS)])
def test_plane_dft_axes_vs_oracle(cuda, axis, comps):
    shape = (28, 30, 32)
    g, o = both(cuda, shape, 1e-3, 4)
    for s in (g, o):
        s.set_epsilon(blocky_eps(shape, block=4, lo=1, hi=4, seed=2))
        s.add_source(lambda f: f.add_source_Jx(16, gaussian_sine(f.t, 40e9, 30e9), i0=13, i1=15,
                                               j0=14, j1=16))
    idx = (9, 15, 20)[axis]
    mg = cuda.CUDAPlaneDFTMonitor(g, axis, idx, [30e9, 45e9], comps)
    mo = D.OraclePlaneDFTMonitor(o, axis, idx, [30e9, 45e9], comps)
    g.run(80)
    o.run(80)
    for c in comps:
        assert np.array_equal(mg.dft(c), mo.dft[c]), c


@pytest.mark.parametrize("dielectric", [False, True])
def test_farfield_goldens(cuda, golden, dielectric):
    """Reference far-field goldens (``tests/meep_validation/cases.py:24-83,249-265``)."""
    tag = "dielectric_sphere_farfield" if dielectric else "vacuum_farfield"
    g, o = both(cuda, (30, 30, 30), 2e-3, 6)
    farfield_case_setup(g, dielectric)
    farfield_case_setup(o, dielectric)
    mg = cuda.CUDANear2FarMonitor(g, (30e-3,) * 3, (20e-3,) * 3, 5e9)
    mo = D.OracleNear2FarMonitor(o, (30e-3,) * 3, (20e-3,) * 3, 5e9)
    g.run(500)
    o.run(500)
    assert_same(g, o)
    faces = mg.face_dft()
    for n in FIELDS:
        assert np.array_equal(faces[n], mo.dft[n][0]), n
    gold = golden["farfield"]
    for key, pt in (("ocl_eh_plus_z", (0, 0, 10.0)), ("ocl_eh_plus_x", (10.0, 0, 0))):
        eh = mg.get_farfield(pt)
        assert peak_err(eh, mo.get_farfield(pt)) < 1e-9
        assert peak_err(eh, gold[f"{tag}_{key}"]) < 1e-4
    ang, db = mg.farfield_polar_xz(distance_m=10.0, n_angles=19)
    np.testing.assert_allclose(db, gold[f"{tag}_ocl_S_db"], rtol=1e-5, atol=1e-4)


def test_near2far_monitor_api(cuda):
    """Reference ``tests/test_unit_monitors.py:52-173``."""
    shape, dl, npml = (24, 24, 24), 2e-3, 4
    g = cuda.CUDAFDTD(shape, dl, npml=npml)
    z = shape[2] - npml - 2
    g.add_source(lambda f: f.add_source_Ex(z, np.sin(2 * np.pi * 5e9 * f.t)))
    mon = cuda.CUDANear2FarMonitor(g, (24e-3,) * 3, (24e-3,) * 3, 5e9)
    assert mon._phase is None
    assert mon.dft_relative_change() == 1.0
    g.run(40)
    eh = mon.get_farfields(np.array([[0.0, 0.0, 10.0], [10.0, 0.0, 0.0]], np.float32))
    assert eh.shape == (2, 6)
    assert mon.get_farfields(np.array([0.0, 0.0, 10.0], np.float32)).shape == (1, 6)
    with pytest.raises(ValueError):
        mon.get_farfields(np.ones((3, 2), np.float32))
    with pytest.raises(ValueError):
        mon.farfield_polar_xz(distance_m=0.0)
    expected = np.exp(1j * mon.omega * g.t) * g.dt
    assert abs(mon._phase) == pytest.approx(abs(expected), rel=1e-9)
    assert abs(np.angle(mon._phase / expected)) < 1e-6
    faces = mon.fetch_dft_fields()
    assert set(faces) == set(FIELDS)
    assert mon.Ex_dft.shape == shape and mon.Ex_dft.dtype == np.complex64
    mon.snapshot_dft()
    assert mon.dft_relative_change() < 1e-12
    prev = mon.face_dft()
    g.run(30)
    cur = mon.face_dft()
    num = sum(float(np.vdot(cur[k] - prev[k], cur[k] - prev[k]).real) for k in FIELDS)
    den = sum(float(np.vdot(cur[k], cur[k]).real) for k in FIELDS)
    host = np.sqrt(num / den)
    gpu = mon.dft_relative_change()
    assert 1e-3 < gpu < 1.0
    assert gpu == pytest.approx(host, rel=1e-10)


def test_tiny_box_farfield(cuda):
    g = cuda.CUDAFDTD((16, 16, 16), 1e-3, npml=2)
    g.add_source(lambda f: f.add_source_Ex(8, 0.05))
    mon = cuda.CUDANear2FarMonitor(g, (8e-3,) * 3, (2e-3,) * 3, 5e9)
    assert mon.n_face_samples < 256
    g.run(15)
    assert mon.get_farfields([(0.0, 0.0, 5.0)]).shape == (1, 6)


def test_engine_api_surface(cuda, caplog):
    """Reference ``tests/test_unit_engine.py:137-181, 259-275``."""
    g = cuda.CUDAFDTD((16, 16, 16), 1e-3, npml=4)
    assert g.dt == 0.99 * 1e-3 / (299_792_458.0 * np.sqrt(3.0))
    with caplog.at_level(logging.INFO, logger="opencl_fdtd_solver_b200.engine"):
        g.run(3, progress_every=1)
    assert "step 0/3" in caplog.text
    assert g.step_num == 3
    h = cuda.CUDAFDTD((14, 15, 16), 1e-3, npml=3)
    for n in FIELDS:
        arr = getattr(h, n)
        assert arr.shape == (14, 15, 16) and arr.dtype == np.float32
    r = cuda.CUDAFDTD((12, 12, 12), 1e-3, npml=2)
    r.add_source(lambda f: f.add_source_Ex(5, 0.37))
    r.step()
    assert r.read_point("Ex", 6, 7, 5) == float(r.Ex[6, 7, 5])
    with pytest.raises(ValueError, match="Epsilon shape mismatch"):
        r.set_epsilon(np.ones((8, 8, 8), np.float32))
    z = cuda.CUDAFDTD((20, 20, 20), 1e-3, npml=0)
    assert z.psi_x_size == 0
    z.add_source(lambda f: f.add_source_Ex(10, 0.1))
    z.run(5)
    assert np.all(np.isfinite(z.Ex)) and np.max(np.abs(z.Ex)) > 0
    with pytest.raises(ValueError):
        z.add_source_Jx(20, 1.0)
    hits = []
    z.add_monitor(lambda f: hits.append(f.step_num))
    z.run(2)
    assert hits == [6, 7]


def test_roofline_config_short_vs_oracle(cuda):
    """Bandwidth config construction (blocky εr∈[1,12], npml 16, Jx point, Gaussian pulse,
    z-plane DFT at 4 frequencies) on a 192³ grid for 12 steps, bit-compared with the oracle."""
    shape = (192, 192, 192)
    g, o = both(cuda, shape, 1e-3, 16, courant=0.5)
    eps = blocky_eps(shape, block=8, seed=1234)
    c = shape[0] // 2
    freqs = [20e9, 25e9, 30e9, 35e9]
    for s in (g, o):
        s.set_epsilon(eps)
        s.add_source(lambda f: f.add_source_Jx(c, gaussian_pulse(f.t, 20e9) + 0.5,
                                               i0=c, i1=c + 1, j0=c, j1=c + 1))
    mg = cuda.CUDAPlaneDFTMonitor(g, "z", c, freqs, ("Ex",))
    mo = D.OraclePlaneDFTMonitor(o, "z", c, freqs, ("Ex",))
    g.run(12)
    o.run(12)
    assert_same(g, o)
    assert np.array_equal(mg.dft("Ex"), mo.dft["Ex"])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape,npml,lossy", [((40, 37, 36), 4, False), ((70, 13, 100), 5, True),
                                              ((65, 65, 68), 6, False), ((12, 9, 8), 0, False),
                                              ((300, 20, 20), 3, False)])
def test_fused_kernel_shapes_vs_oracle(cuda, shape, npml, lossy, dtype):
    """Partial tiles in j and k, several i-chunks, lossy and npml = 0 on the fused path."""
    g, o = both(cuda, shape, 1e-3, npml, dtype=dtype)
    rng = np.random.default_rng(21)
    eps = rng.uniform(1, 6, shape).astype(np.float32)
    sig = rng.uniform(0, 50, shape) if lossy else None
    zc = shape[2] // 2
    for s in (g, o):
        s.set_epsilon(eps, sigma_array=sig)
        s.add_source(lambda f: f.add_source_Jx(zc, gaussian_sine(f.t, 40e9, 30e9),
                                               i0=1, i1=shape[0] - 1, j0=0, j1=shape[1],
                                               rim_taper=True))
        s.add_source(lambda f: f.add_source_Ex(0, 1e-3 * np.cos(3e10 * f.t), i0=0, i1=3))
    mg = cuda.CUDAPlaneDFTMonitor(g, "y", shape[1] // 2, [30e9], ("Ez", "Hy"))
    mo = D.OraclePlaneDFTMonitor(o, "y", shape[1] // 2, [30e9], ("Ez", "Hy"))
    g.run(20)
    o.run(20)
    assert g._fused_enabled, "the aligned shape should run the fused kernel"
    assert_same(g, o)
    for c in ("Ez", "Hy"):
        assert np.array_equal(mg.dft(c), mo.dft[c])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("shape,npml,lossy", [((48, 40, 44), 4, False), ((40, 52, 48), 8, True),
                                              ((56, 44, 64), 12, False), ((66, 70, 72), 20, False),
                                              ((44, 40, 40), 16, True)])
def test_cpml_face_kernels_vs_oracle(cuda, shape, npml, lossy, dtype, monkeypatch):
    """Shell E through the CPML face marches (npml a multiple of 16 bytes of
    elements; forced on, since by default they take only shells of 20 M cells
    and more): z tiles masked (npml 4, 12) or two per face (npml 20), the x-rim
    plane and z-rim column, sources and plane DFTs inside the CPML faces, lossy
    coefficients."""
    monkeypatch.setenv("FDTD_B200_FACE_E", "1")
    g, o = both(cuda, shape, 1e-3, npml, dtype=dtype)
    rng = np.random.default_rng(5)
    eps = rng.uniform(1, 6, shape).astype(np.float32)
    sig = rng.uniform(0, 50, shape) if lossy else None
    nx, ny, nz = shape
    for s in (g, o):
        s.set_epsilon(eps, sigma_array=sig)
        # a full-plane sheet crossing the x and y faces, one inside the low z face
        s.add_source(lambda f: f.add_source_Jx(nz // 2, gaussian_sine(f.t, 40e9, 30e9),
                                               i0=0, i1=nx, j0=0, j1=ny, rim_taper=True))
        s.add_source(lambda f: f.add_source_Jx(1, 0.3 * gaussian_sine(f.t, 30e9, 30e9),
                                               i0=npml + 2, i1=nx - npml - 2, j0=npml + 3,
                                               j1=ny - npml - 1))
    planes = [("x", 2, ("Ey", "Hz")), ("y", ny - 3, ("Ex", "Hx")), ("z", 1, ("Ez", "Hy")),
              ("x", npml, ("Ex", "Ez"))]
    mg = [cuda.CUDAPlaneDFTMonitor(g, ax, i, [30e9, 35e9], c) for ax, i, c in planes]
    mo = [D.OraclePlaneDFTMonitor(o, ax, i, [30e9, 35e9], c) for ax, i, c in planes]
    g.run(30)
    o.run(30)
    assert g._fused_enabled
    assert_same(g, o)
    for (ax, i, comps), a, b in zip(planes, mg, mo):
        for c in comps:
            assert np.array_equal(a.dft(c), b.dft[c]), (ax, i, c)


def test_device_status_clean(cuda):
    import ctypes

    from opencl_fdtd_solver_b200 import _capi as capi

    flags = ctypes.c_int32(-1)
    capi.run("fdtd_device_status", ctypes.byref(flags), 1)
    assert flags.value == 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("src_dtype", [np.float32, np.float64])
@pytest.mark.parametrize("lossy", [False, True])
def test_device_set_epsilon_equals_host_math(cuda, dtype, src_dtype, lossy):
    """Coefficients from fdtd_set_epsilon equal the host float64 math bit for bit
    (reference materials.py:28-88), for float32 and float64 inputs."""
    from opencl_fdtd_solver_b200 import materials

    rng = np.random.default_rng(11)
    shape = (13, 17, 24)
    eps = (1 + 11 * rng.random(shape)).astype(src_dtype)
    sig = (0.5 * rng.random(shape)).astype(src_dtype) if lossy else None
    g = cuda.CUDAFDTD(shape, 1e-3, npml=3, dtype=dtype)
    g.set_epsilon(eps, sigma_array=sig)
    co = g.coefficient_tensors()
    g.synchronize()
    if lossy:
        ca, cb = materials.yee_edge_ca_cb(eps, sig, g.dt, dtype)
        for a in range(3):
            assert np.array_equal(co["ca"][a].cpu().numpy(), ca[a])
            assert np.array_equal(co["ce"][a].cpu().numpy(), cb[a])
    else:
        ce = materials.yee_edge_ce(eps, g.dt, dtype)
        assert co["ca"] is None
        for a in range(3):
            assert np.array_equal(co["ce"][a].cpu().numpy(), ce[a])


@pytest.mark.parametrize("npml,faces,per_step", [(6, None, 4), (8, None, 4), (8, "1", 5)])
def test_launch_counter_and_step_profile(cuda, npml, faces, per_step, monkeypatch):
    import ctypes

    from opencl_fdtd_solver_b200 import _capi as capi

    if faces is not None:
        monkeypatch.setenv("FDTD_B200_FACE_E", faces)
    g = cuda.CUDAFDTD((40, 36, 48), 1e-3, npml=npml)
    cuda.CUDAPlaneDFTMonitor(g, 2, 20, [30e9])
    g.run(2)
    g.synchronize()
    n0 = capi.lib().fdtd_launch_count()
    capi.run("fdtd_profile_steps", 1)
    g.run(5)
    capi.run("fdtd_profile_steps", 0)
    ms = (ctypes.c_double * 5)()
    n = ctypes.c_int32()
    capi.run("fdtd_profile_read", ms, ctypes.byref(n))
    assert n.value == 5
    assert ms[0] > 0 and ms[2] > 0 and ms[3] > 0 and ms[4] > 0
    # shell H, interior, then either the plane DFT of the interior and one
    # per-cell shell E launch (the default for a shell this small), or the
    # face marches, the per-cell kernel for the edges and rims and the plane
    # DFT (forced on; npml 8 is a multiple of four FP32 cells)
    assert capi.lib().fdtd_launch_count() - n0 == per_step * 5


@pytest.mark.parametrize("steps", [200, 2000], ids=["200_steps", "full_2000_steps"])
def test_medium_config_sphere_box_farfield(cuda, steps):
    """The medium configuration: 256³ FP32, npml 12, εr = 4 sphere of radius 40
    cells, rim-tapered Jx sheet at z = npml + 8 trimmed out of the PML,
    Gaussian-modulated sine, a closed 6-face DFT box (half-width 44 cells) at 8
    frequencies, far field on a 181 (θ) x 91 (φ) grid at R = 1 m; 200 steps and
    the configuration's full 2000.  Fields and box DFTs against the C oracle; far
    fields direct and through the tensor-core contraction against the oracle's
    float64 transform."""
    from oracle.dft_oracle import OracleNear2FarMonitor

    n, npml, dl = 256, 12, 1e-3
    shape = (n, n, n)
    eps = sphere_eps(shape, n // 2, 40, 4.0)
    freqs = np.linspace(20e9, 40e9, 8)
    g, o = both(cuda, shape, dl, npml)
    g.set_epsilon(eps)
    o.set_epsilon(eps)
    z = npml + 8

    def drive(f):
        f.add_source_Jx(z, gaussian_sine(f.t, 30e9, 20e9), npml, n - npml, npml, n - npml,
                        rim_taper=True)

    g.add_source(drive)
    o.add_source(drive)
    ctr, size = (n // 2 * dl,) * 3, (88 * dl,) * 3
    mg = cuda.CUDANear2FarMonitor(g, ctr, size, freqs)
    mo = OracleNear2FarMonitor(o, ctr, size, freqs)
    g.run(steps)
    o.run(steps)
    assert_same(g, o)
    for fi in range(freqs.size):
        a = mg.face_dft(fi)
        for c in FIELDS:
            b = mo.dft[c][fi]
            assert np.abs(a[c] - b).max() <= 1e-9 * np.abs(b).max(), (fi, c)
    th = np.deg2rad(np.linspace(0.0, 180.0, 181))
    ph = np.deg2rad(np.linspace(0.0, 180.0, 91, endpoint=False))
    T, P = np.meshgrid(th, ph, indexing="ij")
    pts = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    # get_farfields rounds observation points to the engine dtype (reference
    # monitors.py:653); the oracle gets the same rounded points
    pts32 = pts.astype(np.float32).astype(np.float64)
    for fi in (0, 7):
        ref = mo.get_farfields(pts32, fi)
        d = mg.get_farfields(pts, fi)
        t = mg.get_farfields(pts, fi, method="bf16x3")
        scale = np.abs(ref).max()
        assert np.abs(d - ref).max() <= 1e-9 * scale, fi
        # split-BF16 is held to the FP32-mode far-field tolerance, 1e-5 of peak
        assert np.abs(t - ref).max() <= 1e-5 * scale, fi
