"""The bounded device waits give up, report and recover (GPU).

The fused step's interior kernel and CPML face marches and the tensor-core
near-to-far contraction wait on mbarriers for their bulk copies and MMAs.  Each wait has a budget, and
``fdtd_set_wait_budget`` lowers it for later launches.  With a budget of zero a
wait gives up unless its phase is already complete, which is certain for the
first plane of the interior march and for the contraction's first accumulator
tile.  The kernel then raises its bit in ``fdtd_device_status``, still waits
(with the default bound) for every copy and MMA it issued, frees its tensor
memory and returns.

Each test checks that the call returns, that the bit is set and clears on reset,
and that the next launch with the default budget is correct again: the step
against the CPU oracle bit for bit, the contraction against the float64 direct
sum.  Nothing here faults, traps or hangs the device: the waits that run out
are bounded, and every drain keeps its normal bound.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture
def capi():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opencl_fdtd_solver_b200 import _capi

    flags = ctypes.c_int32(-1)
    _capi.run("fdtd_device_status", ctypes.byref(flags), 1)
    yield _capi
    _capi.run("fdtd_set_wait_budget", _capi.FDTD_WAIT_INTERIOR, -1)
    _capi.run("fdtd_set_wait_budget", _capi.FDTD_WAIT_N2F, -1)
    _capi.run("fdtd_device_status", ctypes.byref(flags), 1)


def _status(capi, reset):
    flags = ctypes.c_int32(-1)
    capi.run("fdtd_device_status", ctypes.byref(flags), reset)
    return flags.value


def _engines(npml=6):
    from opencl_fdtd_solver_b200 import CUDAFDTD
    from oracle.cpu_fdtd import OracleFDTD

    shape = (40, 36, 48)
    g = CUDAFDTD(shape, 1e-3, npml=npml)
    o = OracleFDTD(shape, 1e-3, npml=npml)

    def src(f):
        f.add_source_Jx(24, np.sin(2 * np.pi * 30e9 * f.t), i0=10, i1=30, j0=8, j1=28)

    for s in (g, o):
        s.add_source(src)
    return g, o


@pytest.mark.parametrize("npml", [6, 8])
def test_interior_wait_timeout_reports_and_recovers(capi, npml, monkeypatch):
    """npml 6: the interior march gives up; npml 8 (a multiple of four FP32
    cells, the CPML face marches forced on): the face marches of the shell E
    step give up as well."""
    if npml == 8:
        monkeypatch.setenv("FDTD_B200_FACE_E", "1")
    assert capi.call("fdtd_set_wait_budget", 7, 0) == capi.FDTD_ERR_INVALID
    g, _ = _engines(npml)
    g.run(3)
    assert g._fused_enabled
    capi.run("fdtd_set_wait_budget", capi.FDTD_WAIT_INTERIOR, 0)
    g.step()  # returns: the interior kernel gave up at its first plane
    g.synchronize()
    assert _status(capi, 0) & 1
    assert _status(capi, 1) & 1  # read and clear
    assert _status(capi, 0) == 0
    capi.run("fdtd_set_wait_budget", capi.FDTD_WAIT_INTERIOR, -1)
    # a fresh engine with the default budget matches the oracle bit for bit
    g, o = _engines(npml)
    g.run(30)
    o.run(30)
    assert _status(capi, 0) == 0
    for n in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        ref = getattr(o, n)
        assert np.abs(ref).max() > 0, n
        assert np.array_equal(getattr(g, n), ref), n


def test_n2f_wait_timeout_reports_and_recovers(capi):
    from opencl_fdtd_solver_b200.n2f import N2FFace, near2far_contract

    rng = np.random.default_rng(5)
    dl, nfreq = 2e-3, 2
    faces = []
    for normal in range(3):
        a, b = [x for x in range(3) if x != normal]
        for side in (0, 1):
            cur = (rng.standard_normal((nfreq, 40, 36, 4)) +
                   1j * rng.standard_normal((nfreq, 40, 36, 4))).astype(np.complex64)
            faces.append(N2FFace(normal=normal, x_n=side * 40 * dl, o_p=0.5 * dl, o_q=0.5 * dl,
                                 pitch=dl, cur=torch.as_tensor(cur * dl * dl, device="cuda")))
    v = rng.standard_normal((200, 3))
    dirs = v / np.linalg.norm(v, axis=1, keepdims=True)
    freqs = [20e9, 33e9]
    capi.run("fdtd_set_wait_budget", capi.FDTD_WAIT_N2F, 0)
    near2far_contract(faces, freqs, dirs, mode="bf16x3")  # returns; its output is undefined
    torch.cuda.synchronize()
    assert _status(capi, 1) & 2
    assert _status(capi, 0) == 0
    capi.run("fdtd_set_wait_budget", capi.FDTD_WAIT_N2F, -1)
    got = near2far_contract(faces, freqs, dirs, mode="bf16x3").cpu().numpy()
    ref = near2far_contract(faces, freqs, dirs, mode="fp64").cpu().numpy()
    assert _status(capi, 0) == 0
    err = np.abs(got.astype(np.complex128) - ref).max() / np.abs(ref).max()
    assert err <= 1e-5, err
