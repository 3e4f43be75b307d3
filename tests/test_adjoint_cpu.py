"""Adjoint ε-gradient: the CPU restatement against torch autograd, and host logic.

The reference has no gradient, so the discrete adjoint is pinned by automatic
differentiation of an FP64 PyTorch transcription of the reference NumPy engine
(``opencl_fdtd_solver/numpy_engine.py:193-297``), run here on the CPU: the hand
derivation in ``oracle/adjoint_oracle.py`` (the statement the CUDA kernels follow
operation for operation) must agree with it to rounding, CPML, rim-tapered sheet
source (whose ``ce`` depends on ε) and several frequencies and components included.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import adjoint_oracle as ao  # noqa: E402
from oracle import host_math as hm  # noqa: E402
from oracle import torch_fdtd as tf  # noqa: E402
from oracle.cpu_fdtd import OracleFDTD  # noqa: E402

SHAPE = (14, 12, 16)
DL = 1e-3
NPML = 3
DESIGN = ((5, 9), (4, 8), (6, 9))
SRC = dict(z=4, i0=4, i1=10, j0=3, j1=9)


def _drive(t):
    return float(np.sin(2 * np.pi * 30e9 * t) * np.exp(-((t - 60e-12) / 30e-12) ** 2))


def _eps(seed=1):
    rng = np.random.default_rng(seed)
    eps = np.ones(SHAPE)
    (i0, i1), (j0, j1), (k0, k1) = DESIGN
    eps[i0:i1, j0:j1, k0:k1] = 1 + 3 * rng.random((i1 - i0, j1 - j0, k1 - k0))
    return eps


def _oracle_grad(eps, n, obj, design=DESIGN, src=SRC, dtype=np.float64):
    fd = OracleFDTD(SHAPE, DL, NPML, dtype)
    fd.set_epsilon(eps)
    fd.add_source(lambda f: f.add_source_Jx(src["z"], _drive(f.t), src["i0"], src["i1"],
                                            src["j0"], src["j1"], rim_taper=True))
    return fd.dt, ao.gradient(fd, n, obj, design, eps)


def _torch_grad(eps, n, obj, dt, src=SRC):
    et = torch.tensor(eps, requires_grad=True)
    sources = lambda t: [(src["z"], _drive(t), src["i0"], src["i1"], src["j0"],  # noqa: E731
                          src["j1"], True, 0.8, True)]
    J, D = tf.dft_objective(et, shape=SHAPE, dl=DL, npml=NPML, dt=dt, n_steps=n,
                            sources=sources, objective=obj)
    J.backward()
    return float(J.detach()), et.grad.numpy(), D.detach().numpy()


@pytest.mark.parametrize("n_steps", [40, 160])
def test_oracle_adjoint_matches_torch_autograd(n_steps):
    obj = dict(axis=2, index=11, patch=((4, 10), (3, 9)), freqs=[30e9, 25e9],
               components=("Ex", "Ez"))
    eps = _eps()
    dt, (J, g, D) = _oracle_grad(eps, n_steps, obj)
    Jt, gt, Dt = _torch_grad(eps, n_steps, obj, dt)
    sl = tuple(slice(lo, hi) for lo, hi in DESIGN)
    gt = gt[sl]
    assert abs(J - Jt) <= 1e-13 * abs(Jt)
    assert np.abs(D - Dt).max() <= 1e-13 * np.abs(Dt).max()
    assert np.abs(g - gt).max() <= 1e-12 * np.abs(gt).max()


def test_oracle_adjoint_design_overlapping_source_and_pml():
    """Design box touching the PML and containing the sheet: the sheet's ce term
    and the ψ adjoints enter the gradient."""
    design = ((1, 12), (2, 10), (2, 7))
    obj = dict(axis=1, index=9, patch=((3, 11), (8, 14)), freqs=[28e9], components=("Ex", "Ey"))
    rng = np.random.default_rng(5)
    eps = np.ones(SHAPE)
    eps[1:12, 2:10, 2:7] = 1 + 2 * rng.random((11, 8, 5))
    fd = OracleFDTD(SHAPE, DL, NPML, np.float64)
    fd.set_epsilon(eps)
    fd.add_source(lambda f: f.add_source_Jx(4, _drive(f.t), 3, 11, 3, 9, rim_taper=True))
    J, g, _ = ao.gradient(fd, 90, obj, design, eps)
    et = torch.tensor(eps, requires_grad=True)
    Jt, _ = tf.dft_objective(et, shape=SHAPE, dl=DL, npml=NPML, dt=fd.dt, n_steps=90,
                             sources=lambda t: [(4, _drive(t), 3, 11, 3, 9, True, 0.8, True)],
                             objective=obj)
    Jt.backward()
    gt = et.grad.numpy()[1:12, 2:10, 2:7]
    assert abs(J - float(Jt.detach())) <= 1e-13 * J
    assert np.abs(g - gt).max() <= 1e-12 * np.abs(gt).max()


def test_transcription_forward_matches_c_oracle():
    """The torch transcription's fields equal the C restatement (FP64) on the same run."""
    eps = _eps(3)
    fd = OracleFDTD(SHAPE, DL, NPML, np.float64)
    fd.set_epsilon(eps)
    fd.add_source(lambda f: f.add_source_Jx(SRC["z"], _drive(f.t), SRC["i0"], SRC["i1"],
                                            SRC["j0"], SRC["j1"], rim_taper=True))
    obj = dict(axis=0, index=7, patch=((0, SHAPE[1]), (0, SHAPE[2])), freqs=[30e9],
               components=("Ex", "Ey", "Ez"))
    J, _, D = ao.gradient(fd, 60, obj, DESIGN, eps)
    _, _, Dt = _torch_grad(eps, 60, obj, fd.dt)
    assert np.abs(D - Dt).max() <= 1e-12 * np.abs(D).max()


def test_product_chain_rule_and_phases_match_oracle():
    from opencl_fdtd_solver_b200 import adjoint as pa

    rng = np.random.default_rng(7)
    shape = (9, 8, 7)
    eps = 1 + 3 * rng.random(shape)
    for design in (((2, 6), (1, 5), (3, 7)), ((0, 9), (0, 8), (0, 7)), ((8, 9), (0, 1), (6, 7))):
        box = ao.grad_box(shape, design)
        G = [rng.standard_normal(tuple(hi - lo for lo, hi in box)) for _ in range(3)]
        want = ao.edge_to_cell(G, eps, design, box)
        got = pa.edge_to_cells(np.stack(G), eps, design, box)
        np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(pa._phase_sequence([25e9, 31e9], 1.7e-12, 700, 1.7e-12),
                                  ao.phase_sequence([25e9, 31e9], 1.7e-12, 700, 1.7e-12))


def test_product_phases_match_plane_monitor_table():
    from opencl_fdtd_solver_b200 import adjoint as pa
    from opencl_fdtd_solver_b200.monitors import _PhaseTable

    dt = 1.9e-12
    tab = _PhaseTable([30e9, 12e9], dt, "cpu")
    got = []
    for n in range(1100):  # crosses two chunk refills
        tab.next_ptr(dt * (n + 1))
        got.append(tab.phase.copy())
    np.testing.assert_array_equal(np.array(got), pa._phase_sequence([30e9, 12e9], dt, 1100, dt))


def test_objective_validation():
    from opencl_fdtd_solver_b200 import DFTObjective

    with pytest.raises(ValueError):
        DFTObjective(3, 0, ((0, 1), (0, 1)), [1e9])
    with pytest.raises(ValueError):
        DFTObjective(2, 0, ((0, 1), (0, 1)), [1e9], components=("Hx",))
    with pytest.raises(ValueError):
        DFTObjective(2, 0, ((0, 1), (0, 1)), [])
    o = DFTObjective("z", 4, ((0, 2), (1, 3)), 1e9, components=("Ez", "Ex"))
    assert o.components == ("Ex", "Ez") and o.comp_mask == 5 and o.axis == 2


def test_edge_eps_restatement_agrees():
    from opencl_fdtd_solver_b200 import adjoint as pa

    eps = 1 + np.random.default_rng(2).random((5, 6, 7))
    for a, b in zip(pa._edge_eps(eps), hm.edge_eps(eps)):
        np.testing.assert_array_equal(a, b)
