"""Sub-box host reads and the host Huygens-box monitor on ``CUDAFDTD`` (GPU).

* ``read_region`` / ``read_plane`` / ``host_window`` (``fdtd_read_regions``) return
  exactly the cells of a full read (reference ``engine.py:747-789``).
* ``NumPyNear2FarMonitor`` on ``CUDAFDTD`` (windowed reads of the face slabs only)
  accumulates bit-for-bit what it accumulates on the CPU oracle engine with full
  reads, and its far field is the oracle's ``η·N⊥ − r̂×L`` transform of its face
  arrays.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import dft_oracle as D
from oracle.cpu_fdtd import OracleFDTD
from tests.cases import gaussian_sine

pytestmark = pytest.mark.gpu
FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


@pytest.fixture(scope="module")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import opencl_fdtd_solver_b200 as pkg

    return pkg


def driven(engine, shape, npml):
    c = [n // 2 for n in shape]
    engine.add_source(lambda f: f.add_source_Jx(c[2], gaussian_sine(f.t, 30e9, 20e9),
                                                i0=c[0], i1=c[0] + 1, j0=c[1], j1=c[1] + 1))
    return engine


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_read_region_and_plane_equal_full_reads(cuda, dtype):
    shape = (20, 22, 24)
    g = driven(cuda.CUDAFDTD(shape, 1e-3, npml=5, dtype=dtype), shape, 5)
    g.run(30)
    boxes = [((0, 20), (0, 22), (0, 24)), ((3, 4), (5, 6), (7, 8)), ((19, 20), (0, 22), (23, 24)),
             ((2, 9), (21, 22), (0, 24)), ((0, 20), (4, 4), (0, 24))]
    for n in FIELDS:
        full = getattr(g, n)
        for box in boxes:
            lo, hi = [a for a, _ in box], [b for _, b in box]
            got = g.read_region(n, lo, hi)
            assert got.dtype == np.dtype(dtype)
            assert np.array_equal(got, full[tuple(slice(a, b) for a, b in box)]), (n, box)
        assert np.array_equal(g.read_plane(n, "x", 7), full[7])
        assert np.array_equal(g.read_plane(n, 1, 21), full[:, 21])
        assert np.array_equal(g.read_plane(n, "z", 0), full[:, :, 0])
    with pytest.raises(ValueError):
        g.read_region("Ex", (0, 0, 0), (21, 1, 1))
    with pytest.raises(ValueError):
        g.read_plane("Ex", "z", 24)
    with pytest.raises(ValueError):
        g.read_region("Bx", (0, 0, 0), (1, 1, 1))


def test_host_window_many_boxes_and_restore(cuda):
    """More boxes than one call takes (chunked), a read-only mirror inside the
    window, full writable reads again outside it."""
    shape = (16, 18, 40)
    g = driven(cuda.CUDAFDTD(shape, 1e-3, npml=4), shape, 4)
    g.run(25)
    full = {n: getattr(g, n) for n in FIELDS}
    boxes = [((i % 16, i % 16 + 1), (0, 18), (i, i + 1)) for i in range(40)]
    with g.host_window(boxes):
        for n in FIELDS:
            win = getattr(g, n)
            assert not win.flags.writeable and win.shape == shape
            for box in boxes:
                sl = tuple(slice(a, b) for a, b in box)
                assert np.array_equal(win[sl], full[n][sl])
    out = g.Ex
    assert out.flags.writeable and np.array_equal(out, full["Ex"])


def test_host_monitor_bitwise_vs_oracle_engine(cuda):
    shape, npml, dl, freq = (26, 24, 28), 5, 1e-3, 30e9
    center = tuple(n * dl / 2 for n in shape)
    size = (12e-3, 10e-3, 14e-3)
    g = driven(cuda.CUDAFDTD(shape, dl, npml=npml), shape, npml)
    o = driven(OracleFDTD(shape, dl, npml=npml), shape, npml)
    mg = cuda.NumPyNear2FarMonitor(g, center, size, freq)
    mo = cuda.NumPyNear2FarMonitor(o, center, size, freq)

    class FullReads(cuda.NumPyNear2FarMonitor):
        host_regions = None

    mf = FullReads(g, center, size, freq)
    from opencl_fdtd_solver_b200 import _capi

    n0 = _capi.lib().fdtd_launch_count()
    g.run(60)
    launches = _capi.lib().fdtd_launch_count() - n0
    o.run(60)
    for n in FIELDS:
        a, b, c = (getattr(m, f"{n}_dft_f") for m in (mg, mo, mf))
        assert np.abs(b).max() > 0, n
        assert np.array_equal(a, b), n
        assert np.array_equal(c, b), n
    # the windowed monitor issues one gather launch per field per step
    assert launches >= 60 * 6
    # after the run, properties are full reads of the engine state
    assert np.array_equal(g.Hz, o.Hz)


def test_host_monitor_farfield_matches_oracle_transform(cuda):
    shape, npml, dl, freq = (26, 24, 28), 5, 1e-3, 30e9
    center = tuple(n * dl / 2 for n in shape)
    g = driven(cuda.CUDAFDTD(shape, dl, npml=npml), shape, npml)
    mon = cuda.NumPyNear2FarMonitor(g, center, (12e-3, 10e-3, 14e-3), freq)
    ref_mon = cuda.CUDANear2FarMonitor(g, center, (12e-3, 10e-3, 14e-3), freq)
    g.run(80)
    pts = np.array([[0.0, 0.0, 1.0], [1.0, 0.0, 0.0], [0.3, -0.4, 0.866], [-1.0, 0.2, -0.5]])
    got = mon.get_farfields(pts)
    dft = {n: getattr(mon, f"{n}_dft_f").astype(np.complex128)[None] for n in FIELDS}
    want = D.farfield_eh(dft, mon._box, dl, freq, pts.astype(np.float32).astype(np.float64))
    scale = np.abs(want).max()
    assert scale > 0
    assert np.abs(got - want).max() <= 1e-9 * scale
    assert np.allclose(mon.get_farfield(pts[2]), got[2])
    # the device-accumulated monitor (complex128 sums) agrees to complex64 rounding
    dev = ref_mon.get_farfields(pts)
    assert np.abs(dev - got).max() <= 1e-5 * scale
