"""FP32 results against FP64 runs of the same configuration (GPU).

The FP32 engine's results carry the rounding of FP32 time stepping, exactly as
the reference's FP32 kernels do.  These tests state how far they are from FP64
runs and hold them to bounds a few times above the measured values:

* small configuration (64³, npml 8, Courant 0.5, Jx point, 500 steps, z = 32
  plane DFT at 25/30/35 GHz) against the FP64 NumPy face-CPML engine (the
  reference's NumPy algorithm, bit-identical to it on its fixtures): Ex to its
  peak, Hy to η0 times the E peak (a static charge field stays in E near the
  source and H is a difference of those values), and the plane DFTs;
* medium configuration (256³ sphere, rim-tapered sheet, 2000 steps, 89³ box at
  8 frequencies) against the FP64 CUDA engine (itself within 1e-12 of FP64
  NumPy on the parity tests): box DFTs, far fields direct and split-BF16.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from tests.cases import gaussian_sine, sphere_eps  # noqa: E402


def _err(a, b):
    return float(np.abs(np.asarray(a, np.complex128) - b).max() / np.abs(b).max())


def test_small_config_fp32_vs_fp64_numpy():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opencl_fdtd_solver_b200 import ETA0, CUDAFDTD, CUDAPlaneDFTMonitor
    from oracle.numpy_face_cpml import NumPyFaceCPML

    freqs = [25e9, 30e9, 35e9]

    def src(f):
        f.add_source_Jx(32, gaussian_sine(f.t, 30e9, 20e9), i0=32, i1=33, j0=32, j1=33)

    g = CUDAFDTD((64,) * 3, 1e-3, npml=8, courant=0.5)
    g.add_source(src)
    m = CUDAPlaneDFTMonitor(g, "z", 32, freqs, ("Ex", "Hy"))
    g.run(500)
    o = NumPyFaceCPML((64,) * 3, 1e-3, npml=8, dtype=np.float64, courant=0.5)
    o.add_source(src)
    om = 2 * np.pi * np.array(freqs)
    acc = {c: np.zeros((3, 64, 64), np.complex128) for c in ("Ex", "Hy")}
    st = {"p": None}

    def plane(f):
        st["p"] = (np.exp(1j * om * f.t) * f.dt if st["p"] is None
                   else st["p"] * np.exp(1j * om * f.dt))
        ph = st["p"] * np.exp(-0.5j * om * f.dt)
        acc["Ex"] += st["p"][:, None, None] * f.Ex[:, :, 32][None]
        acc["Hy"] += ph[:, None, None] * f.Hy[:, :, 32][None]

    o.add_monitor(plane)
    o.run(500)
    e_peak = np.abs(o.Ex).max()
    assert _err(g.Ex, o.Ex) <= 1e-5          # measured 2.2e-6
    assert ETA0 * np.abs(g.Hy.astype(np.float64) - o.Hy).max() <= 1e-5 * e_peak
    assert _err(m.dft("Ex"), acc["Ex"]) <= 1e-6   # measured 8.6e-8
    assert _err(m.dft("Hy"), acc["Hy"]) <= 1e-6   # measured 1.5e-8


def test_medium_config_fp32_vs_fp64_box_and_far_field():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import bench

    th = np.deg2rad(np.linspace(0.0, 180.0, 181))
    ph = np.deg2rad(np.linspace(0.0, 180.0, 91, endpoint=False))
    T, P = np.meshgrid(th, ph, indexing="ij")
    pts = np.stack([np.sin(T) * np.cos(P), np.sin(T) * np.sin(P), np.cos(T)], -1).reshape(-1, 3)
    res = {}
    for dt in (np.float32, np.float64):
        g, mon = bench.medium_engine(box=True, dtype=dt)
        g.run(2000)
        res[dt] = ([mon.face_dft(fi) for fi in range(bench.MED_FREQS.size)],
                   {fi: mon.get_farfields(pts, fi) for fi in (0, 7)},
                   {fi: mon.get_farfields(pts, fi, method="bf16x3") for fi in (0, 7)}
                   if dt == np.float32 else None)
        del g, mon
        torch.cuda.empty_cache()
    (box32, ff32, tc32), (box64, ff64, _) = res[np.float32], res[np.float64]
    for fi in range(bench.MED_FREQS.size):
        for c in box64[fi]:
            assert _err(box32[fi][c], box64[fi][c]) <= 1e-5, (fi, c)  # measured ≤ 1.8e-6
    for fi in (0, 7):
        assert _err(ff32[fi], ff64[fi]) <= 5e-5, fi      # measured 8.7e-6 / 1.2e-5
        assert _err(tc32[fi], ff64[fi]) <= 5e-5, fi      # measured 9.1e-6 / 1.2e-5
