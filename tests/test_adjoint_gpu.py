"""Adjoint ε-gradient on the GPU (``EpsilonAdjoint`` through the C ABI).

Checks, in order of strength:

* the CUDA sweep against the CPU restatement of the same transposed step
  (``oracle/adjoint_oracle.py``), FP64 and FP32, same inputs;
* against torch autograd through the FP64 transcription of the reference NumPy
  engine (``oracle/torch_fdtd.py``) on a 48³ grid;
* against central finite differences (h = 1e-3) of the CUDA forward solve;
* checkpoint spacing and the capture mode do not change the result; the
  autograd wrapper returns the same gradient; lossy grids are refused.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from opencl_fdtd_solver_b200 import (CUDAFDTD, DFTObjective, EpsilonAdjoint,  # noqa: E402
                                     epsilon_objective)
from oracle import adjoint_oracle as ao  # noqa: E402
from oracle import torch_fdtd as tf  # noqa: E402
from oracle.cpu_fdtd import OracleFDTD  # noqa: E402

DL = 1e-3


def _drive(t):
    return float(np.sin(2 * np.pi * 30e9 * t) * np.exp(-((t - 60e-12) / 30e-12) ** 2))


SMALL = dict(shape=(14, 12, 16), npml=3, design=((5, 9), (4, 8), (6, 9)),
             src=(4, 4, 10, 3, 9), obj=dict(axis=2, index=11, patch=((4, 10), (3, 9)),
                                            freqs=[30e9, 25e9], components=("Ex", "Ez")))


def _eps_design(design, seed):
    rng = np.random.default_rng(seed)
    return 1 + 3 * rng.random(tuple(hi - lo for lo, hi in design))


def _full(shape, design, eps_d):
    eps = np.ones(shape)
    eps[tuple(slice(lo, hi) for lo, hi in design)] = eps_d
    return eps


def _cuda_adjoint(case, dtype, n_steps, K, **kw):
    z, i0, i1, j0, j1 = case["src"]
    fd = CUDAFDTD(case["shape"], DL, npml=case["npml"], dtype=dtype)
    fd.add_source(lambda f: f.add_source_Jx(z, _drive(f.t), i0, i1, j0, j1, rim_taper=True))
    o = case["obj"]
    obj = DFTObjective(o["axis"], o["index"], o["patch"], o["freqs"], o["components"])
    return EpsilonAdjoint(fd, case["design"], n_steps, obj, checkpoint_every=K, **kw)


def _oracle(case, dtype, n_steps, eps_d):
    z, i0, i1, j0, j1 = case["src"]
    eps = _full(case["shape"], case["design"], eps_d)
    fd = OracleFDTD(case["shape"], DL, case["npml"], dtype)
    fd.set_epsilon(eps)
    fd.add_source(lambda f: f.add_source_Jx(z, _drive(f.t), i0, i1, j0, j1, rim_taper=True))
    return ao.gradient(fd, n_steps, case["obj"], case["design"], eps)


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-13), (np.float32, 1e-6)])
def test_cuda_adjoint_matches_oracle(dtype, tol):
    eps_d = _eps_design(SMALL["design"], 1)
    adj = _cuda_adjoint(SMALL, dtype, 160, 37)
    J, g = adj.value_and_grad(eps_d)
    Jo, go, Do = _oracle(SMALL, dtype, 160, eps_d)
    D = adj.D.cpu().numpy()
    assert np.abs(D - Do).max() <= tol * np.abs(Do).max()
    assert abs(J - Jo) <= 10 * tol * Jo
    err = np.abs(g - go).max() / np.abs(go).max()
    assert err <= tol, err


def test_checkpoint_spacing_does_not_change_gradient():
    """Replay from checkpoints every K steps (K = 1000, 7, 1) and the forward
    capture of every step give the same gradient bit for bit."""
    eps_d = _eps_design(SMALL["design"], 2)
    g = []
    for K in (1000, 7, 1):
        adj = _cuda_adjoint(SMALL, np.float32, 90, K, capture="replay")
        g.append(adj.value_and_grad(eps_d)[1])
        assert not adj._captured and adj._cap_all is None
    adj = _cuda_adjoint(SMALL, np.float32, 90, 7, capture="all")
    g.append(adj.value_and_grad(eps_d)[1])
    assert adj._captured
    for other in g[1:]:
        np.testing.assert_array_equal(g[0], other)


def test_capture_mode_follows_the_budget():
    eps_d = _eps_design(SMALL["design"], 4)
    roomy = _cuda_adjoint(SMALL, np.float64, 60, 10)
    J0, g0 = roomy.value_and_grad(eps_d)
    assert roomy._captured  # a few MB: within a quarter of free memory
    tight = _cuda_adjoint(SMALL, np.float64, 60, 10, capture_budget=0)
    J1, g1 = tight.value_and_grad(eps_d)
    assert not tight._captured and tight._cap_all is None
    assert J0 == J1
    np.testing.assert_array_equal(g0, g1)
    with pytest.raises(ValueError):
        _cuda_adjoint(SMALL, np.float64, 60, 10, capture="sometimes")


def test_autograd_function_returns_adjoint_gradient():
    eps_d = _eps_design(SMALL["design"], 3)
    adj = _cuda_adjoint(SMALL, np.float64, 80, 25)
    J0, g0 = adj.value_and_grad(eps_d)
    e = torch.tensor(eps_d, dtype=torch.float64, device="cuda", requires_grad=True)
    J = epsilon_objective(e, adj)
    (2.0 * J).backward()
    assert float(J) == J0
    np.testing.assert_allclose(e.grad.cpu().numpy(), 2.0 * g0, rtol=0, atol=0)


def test_cuda_adjoint_vs_torch_autograd_48cube():
    """48³, npml 8, FP64: CUDA adjoint against autograd of the NumPy-engine transcription."""
    shape, npml, n = (48, 48, 48), 8, 240
    design = ((16, 32), (16, 32), (20, 28))
    src = (12, 10, 38, 10, 38)
    obj = dict(axis=2, index=36, patch=((16, 32), (16, 32)), freqs=[30e9], components=("Ex",))
    case = dict(shape=shape, npml=npml, design=design, src=src, obj=obj)
    eps_d = _eps_design(design, 4)
    adj = _cuda_adjoint(case, np.float64, n, 100)
    J, g = adj.value_and_grad(eps_d)
    et = torch.tensor(_full(shape, design, eps_d), device="cuda", requires_grad=True)
    z, i0, i1, j0, j1 = src
    Jt, _ = tf.dft_objective(et, shape=shape, dl=DL, npml=npml, dt=adj.fdtd.dt, n_steps=n,
                             sources=lambda t: [(z, _drive(t), i0, i1, j0, j1, True, 0.8, True)],
                             objective=obj)
    Jt.backward()
    gt = et.grad[tuple(slice(lo, hi) for lo, hi in design)].cpu().numpy()
    del et, Jt
    torch.cuda.empty_cache()
    assert np.isfinite(J) and J > 0
    err = np.linalg.norm(g - gt) / np.linalg.norm(gt)
    assert err <= 1e-10, err


def test_gradient_vs_central_differences():
    """FP64 CUDA solves: central differences (h = 1e-3) at 6 seeded design voxels."""
    shape, npml, n = (32, 32, 28), 6, 300
    design = ((10, 22), (10, 22), (10, 14))
    src = (7, 7, 25, 7, 25)
    obj = dict(axis=2, index=20, patch=((10, 22), (10, 22)), freqs=[30e9], components=("Ex",))
    case = dict(shape=shape, npml=npml, design=design, src=src, obj=obj)
    eps_d = _eps_design(design, 5)
    adj = _cuda_adjoint(case, np.float64, n, 64)
    _, g = adj.value_and_grad(eps_d)
    rng = np.random.default_rng(6)
    dims = tuple(hi - lo for lo, hi in design)
    idx = [tuple(int(rng.integers(0, d)) for d in dims) for _ in range(6)]
    h = 1e-3
    fd_g, ad_g = [], []
    for v in idx:
        ep = eps_d.copy()
        ep[v] += h
        Jp = adj.forward(ep)
        ep[v] -= 2 * h
        Jm = adj.forward(ep)
        fd_g.append((Jp - Jm) / (2 * h))
        ad_g.append(g[v])
    fd_g, ad_g = np.array(fd_g), np.array(ad_g)
    err = np.linalg.norm(ad_g - fd_g) / np.linalg.norm(fd_g)
    assert err <= 1e-3, (err, ad_g, fd_g)


def test_lossy_grid_is_refused():
    adj = _cuda_adjoint(SMALL, np.float32, 10, 5)
    adj.forward(_eps_design(SMALL["design"], 1))
    adj.fdtd.set_epsilon(np.ones(SMALL["shape"]), sigma_array=np.full(SMALL["shape"], 0.1))
    with pytest.raises(NotImplementedError):
        adj.backward()


MEDIUM = dict(shape=(44, 38, 76), npml=5, design=((14, 30), (12, 26), (30, 42)),
              src=(20, 6, 38, 6, 32), obj=dict(axis=2, index=50, patch=((10, 34), (9, 29)),
                                               freqs=[30e9], components=("Ex", "Ey")))


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("capture", ["all", "replay"])
def test_fused_reverse_step_equals_per_cell_kernels(dtype, capture):
    """The fused reverse step (interior plane march beside the CPML-shell kernels,
    ping-pong buffers) gives the per-cell in-place sweep's gradient and final
    adjoint state bit for bit, on a grid with several march tiles and chunks."""
    eps_d = _eps_design(MEDIUM["design"], 3)
    out = []
    for fused in (True, False):
        adj = _cuda_adjoint(MEDIUM, dtype, 240, 60, capture=capture, fused_reverse=fused)
        J, g = adj.value_and_grad(eps_d)
        Eb, Hb = adj._adjoint_state
        out.append((J, g, [t.cpu().numpy() for t in Eb + Hb]))
    (J1, g1, s1), (J2, g2, s2) = out
    assert J1 == J2
    assert np.abs(g2).max() > 0
    assert np.array_equal(g1, g2)
    for a, b in zip(s1, s2):
        assert np.abs(b).max() > 0
        assert np.array_equal(a, b)
