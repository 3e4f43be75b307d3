"""Near-to-far contraction on the tensor cores (GPU) against float64 transforms.

The float64 direct kernel (``mode="fp64"``) is held to the CPU direct sum
(``oracle/n2f_oracle.py``); the split-BF16 and TF32 tensor-core modes to the
float64 kernel, on faces whose sample counts are not multiples of the tile
sizes and direction counts that leave a partial last tile.  The monitor path
(``box_faces`` of a running simulation) is held to the engine's float64 far field.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from oracle import n2f_oracle  # noqa: E402


def _faces(rng, shape, dl, nfreq, dtype=np.complex64):
    """A closed box of faces with random currents under a smooth envelope."""
    out = []
    for normal in range(3):
        a, b = [x for x in range(3) if x != normal]
        na, nb = shape[a], shape[b]
        for side in (0, 1):
            cur = (rng.standard_normal((nfreq, na, nb, 4)) +
                   1j * rng.standard_normal((nfreq, na, nb, 4)))
            ra = (np.arange(na) - na / 2) / (na / 3)
            rb = (np.arange(nb) - nb / 2) / (nb / 3)
            env = np.exp(-(ra[:, None] ** 2 + rb[None, :] ** 2))
            cur = (cur * env[None, :, :, None] * dl * dl).astype(dtype)
            out.append(dict(normal=normal, x_n=(side * shape[normal]) * dl,
                            o_p=0.5 * dl, o_q=0.5 * dl, pitch=dl, cur=cur))
    return out


def _dirs(n, rng):
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _to_dev(faces):
    from opencl_fdtd_solver_b200.n2f import N2FFace

    return [N2FFace(normal=f["normal"], x_n=f["x_n"], o_p=f["o_p"], o_q=f["o_q"],
                    pitch=f["pitch"], cur=torch.as_tensor(f["cur"], device="cuda")) for f in faces]


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def small():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(3)
    dl = 2e-3
    faces = _faces(rng, (37, 45, 40), dl, 3)
    dirs = _dirs(300, rng)
    freqs = [20e9, 31e9, 44e9]
    ref = n2f_oracle.contract(faces, freqs, dirs)
    return faces, dirs, freqs, ref


def test_fp64_kernel_matches_cpu_direct_sum(small):
    from opencl_fdtd_solver_b200.n2f import near2far_contract

    faces, dirs, freqs, ref = small
    got = near2far_contract(_to_dev(faces), freqs, dirs, mode="fp64").cpu().numpy()
    assert _rel(got, ref) <= 1e-12


@pytest.mark.parametrize("mode,tol", [("bf16x3", 2e-5), ("tf32", 2e-3)])
def test_tensor_core_modes_vs_fp64(small, mode, tol):
    import ctypes

    from opencl_fdtd_solver_b200 import _capi as capi
    from opencl_fdtd_solver_b200.n2f import near2far_contract

    faces, dirs, freqs, ref = small
    got = near2far_contract(_to_dev(faces), freqs, dirs, mode=mode).cpu().numpy()
    flags = ctypes.c_int32(-1)
    capi.run("fdtd_device_status", ctypes.byref(flags), 1)
    assert flags.value == 0
    err = _rel(got.astype(np.complex128), ref)
    assert err <= tol, err
    for f in range(len(freqs)):
        assert _rel(got[f].astype(np.complex128), ref[f]) <= 2 * tol


def test_single_face_and_tiny_counts():
    from opencl_fdtd_solver_b200.n2f import near2far_contract

    rng = np.random.default_rng(9)
    cur = (rng.standard_normal((2, 3, 5, 4)) + 1j * rng.standard_normal((2, 3, 5, 4)))
    f = dict(normal=1, x_n=0.01, o_p=-0.002, o_q=0.003, pitch=1e-3, cur=cur.astype(np.complex128))
    dirs = _dirs(7, rng)
    ref = n2f_oracle.contract([f], [30e9, 60e9], dirs)
    for mode, tol in (("fp64", 1e-12), ("bf16x3", 2e-5), ("tf32", 2e-3)):
        got = near2far_contract(_to_dev([f]), [30e9, 60e9], dirs, mode=mode).cpu().numpy()
        assert _rel(got.astype(np.complex128), ref) <= tol, mode


def test_monitor_faces_reproduce_engine_far_field():
    """box_faces of a running simulation through the contraction equals the NL
    sums of the engine's float64 far-field kernel (get_farfields)."""
    import opencl_fdtd_solver_b200 as pkg
    from opencl_fdtd_solver_b200.n2f import box_faces, near2far_contract

    g = pkg.CUDAFDTD((40, 36, 44), 1e-3, npml=6)
    g.add_source(lambda f: f.add_source_Jx(22, np.sin(2 * np.pi * 30e9 * f.t), i0=15, i1=25,
                                           j0=14, j1=22))
    mon = pkg.CUDANear2FarMonitor(g, (20e-3, 18e-3, 22e-3), (20e-3, 18e-3, 20e-3), [25e9, 30e9])
    g.run(60)
    rng = np.random.default_rng(4)
    dirs = _dirs(50, rng)
    faces = box_faces(mon, dtype=torch.complex128)
    nl64 = near2far_contract(faces, mon.freqs, dirs, mode="fp64").cpu().numpy()
    nl16 = near2far_contract(box_faces(mon), mon.freqs, dirs, mode="bf16x3").cpu().numpy()
    # the same sums from the CPU restatement of the monitor's surface currents
    from oracle import dft_oracle

    acc = mon.acc.cpu().numpy()
    for fi, fr in enumerate(mon.freqs):
        k = 2 * np.pi * fr / dft_oracle.C0
        fields = {n: acc[c][fi:fi + 1, :, 0] + 1j * acc[c][fi:fi + 1, :, 1]
                  for c, n in enumerate(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"))}
        pos, wda, cur = dft_oracle.surface_currents(fields, mon._box, mon.dl, 0)
        ref = dft_oracle.nl_integrals(pos, wda, cur, k, dirs * 10.0)
        assert _rel(nl64[fi], ref) <= 1e-10
        assert _rel(nl16[fi].astype(np.complex128), ref) <= 5e-5


@pytest.mark.parametrize("mode", ["bf16x3", "tf32"])
def test_a_operand_in_tensor_memory_equals_shared_memory_form(small, mode, monkeypatch):
    """The A operand (phases) written to tensor memory and read from there by
    the MMAs gives the shared-memory form's result bit for bit: the same values,
    the same K order, the same MMAs in the same order."""
    from opencl_fdtd_solver_b200.n2f import near2far_contract

    faces, dirs, freqs, _ = small
    dev = _to_dev(faces)
    out = {}
    for where in ("smem", "tmem"):
        monkeypatch.setenv("FDTD_B200_N2F_A", where)
        out[where] = near2far_contract(dev, freqs, dirs, mode=mode).cpu().numpy()
    assert np.abs(out["smem"]).max() > 0
    assert np.array_equal(out["smem"], out["tmem"])
