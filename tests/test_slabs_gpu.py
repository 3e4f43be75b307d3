"""x-slab decomposition on the GPU: slabs of one grid equal the single domain.

Two or three slabs of one grid are held by this process on one device (a run
gets one GPU here, and ranks whose kernels wait on one another must not share a
GPU); after every step their ghost planes are copied directly
(``slabs.local_exchange``), which is the exchange ``SlabFDTD`` makes over NCCL
between GPUs.  The owned planes of all slabs must equal the single-domain run
bit for bit, through the fused step (interior kernel, shell kernels with the
x-CPML only on global faces, ghost planes) and through the split kernels, in
FP32 and FP64, with a rim-tapered sheet and a dielectric block that cross slab
boundaries and a CPML on every global face.  The multi-process exchange itself
is covered on CPU with gloo ranks (``tests/test_slabs_cpu.py``).
"""

from __future__ import annotations

import numpy as np
import pytest

from opencl_fdtd_solver_b200 import slabs
from tests.cases import gaussian_sine

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FIELDS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import opencl_fdtd_solver_b200 as pkg

    return pkg


def _case(shape):
    eps = np.ones(shape, np.float32)
    nx, ny, nz = shape
    eps[nx // 3:2 * nx // 3 + 2, ny // 4:ny // 2, nz // 3:nz // 2] = 3.5

    def src(f):
        f.add_source_Jx(nz // 4, gaussian_sine(f.t, 60e9, 40e9), i0=4, i1=nx - 5, j0=5,
                        j1=ny - 6, rim_taper=True)

    return eps, src


@pytest.mark.parametrize("ranks", [2, 3])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("fused", [True, False], ids=["fused", "split"])
def test_slabs_equal_single_domain(cuda, ranks, dtype, fused):
    shape, npml, steps = (48, 36, 40), 5, 60
    eps, src = _case(shape)
    ref = cuda.CUDAFDTD(shape, 1e-3, npml=npml, dtype=dtype, fused=fused)
    ref.set_epsilon(eps)
    ref.add_source(src)
    ref.run(steps)
    plan = slabs.partition(shape[0], ranks, npml)
    engines = []
    for s in plan:
        g = cuda.CUDAFDTD(shape, 1e-3, npml=npml, dtype=dtype, fused=fused, slab=s)
        g.set_epsilon(eps)
        g.add_source(src)
        engines.append(g)
    views = lambda r: (lambda n, i: engines[r].field_tensor(n)[i])
    for _ in range(steps):
        for g in engines:
            g.step()
        slabs.local_exchange(plan, views)
    for g in engines:
        assert g._fused_enabled == fused
    for n in FIELDS:
        want = getattr(ref, n)
        got = np.concatenate([engines[r].field_tensor(n)[s.owned].cpu().numpy()
                              for r, s in enumerate(plan)])
        assert np.abs(want).max() > 0, n
        assert np.array_equal(got, want), n


def test_slab_refuses_box_monitor_and_adjoint_grid(cuda):
    from opencl_fdtd_solver_b200 import CUDANear2FarMonitor

    s = slabs.partition(48, 2, 5)[1]
    g = cuda.CUDAFDTD((48, 36, 40), 1e-3, npml=5, slab=s)
    assert g.Nx == s.nx_local and g.x0 == s.l0
    with pytest.raises(NotImplementedError):
        CUDANear2FarMonitor(g, (24e-3, 18e-3, 20e-3), (10e-3, 10e-3, 10e-3), 30e9)
