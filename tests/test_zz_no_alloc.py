"""The allocation-free relative-change entry point (GPU).

``fdtd_dft_rel_change_noalloc`` serves callers that must not allocate device
memory while a simulation runs: drivers that keep the device busy with
asynchronous steps (``cudaMalloc``/``cudaFree`` can synchronise the device and
would stall the step stream), and hosts that hand out device memory from a pool
fixed at start-up.  It keeps its partial sums in an array built into the
library instead of a buffer the caller passes.  This test checks it, through
the C ABI, against the entry point that takes a caller buffer, on two calls in
a row (the built-in array keeps the previous call's contents), and checks that
a box larger than the array's stated capacity is refused.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from opencl_fdtd_solver_b200 import CUDAFDTD, CUDANear2FarMonitor
    from opencl_fdtd_solver_b200 import _capi as capi

    return torch, CUDAFDTD, CUDANear2FarMonitor, capi


def _with_caller_buffer(torch, capi, mon, fi):
    q = mon.fdtd.queue
    nblk = int(capi.lib().fdtd_rel_change_blocks(mon.n_face_samples))
    scratch = torch.empty(2 * nblk, dtype=torch.float64, device=mon.fdtd.device)
    out = torch.empty(2, dtype=torch.float64, device=mon.fdtd.device)
    capi.run("fdtd_dft_rel_change", mon.acc.data_ptr(), mon._dft_snap.data_ptr(),
             mon.n_face_samples, mon.freqs.size, fi, scratch.data_ptr(), out.data_ptr(),
             q.cuda_stream)
    q.synchronize()
    return out.cpu().numpy()


def _allocation_free(torch, capi, mon, fi, out):
    q = mon.fdtd.queue
    capi.run("fdtd_dft_rel_change_noalloc", mon.acc.data_ptr(), mon._dft_snap.data_ptr(),
             mon.n_face_samples, mon.freqs.size, fi, out.data_ptr(), q.cuda_stream)
    q.synchronize()
    return out.cpu().numpy()


def test_noalloc_rel_change_matches_caller_buffer_twice(setup):
    torch, CUDAFDTD, CUDANear2FarMonitor, capi = setup
    g = CUDAFDTD((40, 36, 44), 1e-3, npml=6)
    g.add_source(lambda f: f.add_source_Jx(22, np.sin(2 * np.pi * 30e9 * f.t), i0=15, i1=25,
                                           j0=14, j1=22))
    mon = CUDANear2FarMonitor(g, (20e-3, 18e-3, 22e-3), (20e-3, 18e-3, 20e-3), [25e9, 30e9])
    g.run(30)
    mon.snapshot_dft()
    g.run(25)
    out = torch.empty(2, dtype=torch.float64, device=g.device)
    for call in range(2):
        for fi in (0, 1):
            ref = _with_caller_buffer(torch, capi, mon, fi)
            got = _allocation_free(torch, capi, mon, fi, out)
            assert ref[1] > 0 and ref[0] > 0, (call, fi, ref)
            np.testing.assert_allclose(got, ref, rtol=1e-12, atol=0.0)
        g.run(5)  # the next call sees new data, and the array still holds this call's sums


def _header_capacity():
    """FDTD_NOALLOC_MAX_FACE as the C header defines it (the library's own
    static_assert ties its built-in array to the same macro)."""
    hdr = (Path(__file__).resolve().parents[1] / "include" / "fdtd_b200.h").read_text()
    m = re.search(r"#define\s+FDTD_NOALLOC_MAX_FACE\s+\(([^)]*)\)", hdr)
    assert m, "FDTD_NOALLOC_MAX_FACE not found in include/fdtd_b200.h"
    return int(eval(m.group(1), {"__builtins__": {}}))


def test_noalloc_at_exact_capacity_matches_caller_buffer(setup):
    """A box of exactly FDTD_NOALLOC_MAX_FACE samples uses every partial the
    built-in array holds; two calls on different data both match the
    caller-buffer entry point."""
    torch, _, _, capi = setup
    n = _header_capacity()
    assert capi.FDTD_NOALLOC_MAX_FACE == n
    nfreq = 2
    gen = torch.Generator(device="cuda")
    gen.manual_seed(99)
    out = torch.empty(2, dtype=torch.float64, device="cuda")
    ref = torch.empty(2, dtype=torch.float64, device="cuda")
    nblk = int(capi.lib().fdtd_rel_change_blocks(n))
    scratch = torch.empty(2 * nblk, dtype=torch.float64, device="cuda")
    for call in range(2):
        cur = torch.randn((6, nfreq, n, 2), dtype=torch.float64, device="cuda", generator=gen)
        prev = cur + 1e-3 * (call + 1) * torch.randn(cur.shape, dtype=torch.float64,
                                                     device="cuda", generator=gen)
        for fi in range(nfreq):
            capi.run("fdtd_dft_rel_change", cur.data_ptr(), prev.data_ptr(), n, nfreq, fi,
                     scratch.data_ptr(), ref.data_ptr(), None)
            capi.run("fdtd_dft_rel_change_noalloc", cur.data_ptr(), prev.data_ptr(), n, nfreq,
                     fi, out.data_ptr(), None)
            torch.cuda.synchronize()
            a, b = out.cpu().numpy(), ref.cpu().numpy()
            assert b[0] > 0 and b[1] > 0, (call, fi, b)
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=0.0)


def test_noalloc_rejects_boxes_beyond_capacity(setup):
    torch, _, _, capi = setup
    dummy = torch.zeros(2, dtype=torch.float64, device="cuda")
    too_many = _header_capacity() + 1
    rc = capi.call("fdtd_dft_rel_change_noalloc", dummy.data_ptr(), dummy.data_ptr(), too_many,
                   1, 0, dummy.data_ptr(), None)
    assert rc == capi.FDTD_ERR_INVALID
    assert "exceeds" in capi.last_error()
    flags = ctypes.c_int32(-1)
    capi.run("fdtd_device_status", ctypes.byref(flags), 0)
    assert flags.value == 0
