"""Generate the golden fixtures under tests/golden/ from the reference package.

Run in a container where the reference tree is present (it is not needed on a GPU
host; the fixtures it writes are committed)::

    python tests/golden/make_golden.py --reference <reference checkout>

(``--reference`` defaults to the ``FDTD_REFERENCE_ROOT`` environment variable.)

Outputs:

* ``ocl_planes.npz``   — the reference's committed OpenCL (POCL) mid-plane ``Ex``
  arrays for its ``vacuum_sheet`` and ``dielectric_block`` cases
  (``tests/meep_validation/baselines/*/ocl_ex_step*.npy``), case parameters from
  ``tests/meep_validation/plane_cases.py:62-91,116-146``.
* ``ocl_farfield.npz`` — the reference's committed OpenCL far-field arrays
  (``ocl_eh_plus_{z,x}``, ``ocl_S_db``, ``angles_deg``) for ``vacuum_farfield`` and
  ``dielectric_sphere_farfield`` (case: ``tests/meep_validation/cases.py:24-83``).
* ``host_monitor.npz`` — face-packed DFT arrays ``*_dft_f`` of the reference's
  ``NumPyNear2FarMonitor`` (``opencl_fdtd_solver/monitors.py:186-295``) driven by
  the seeded field sequences of ``tests/cases.py`` (``HOST_MONITOR_CASES``).
* ``numpy_ref.npz``    — fields produced by importing the reference's own
  ``NumPyFDTD`` / ``NumPyFDTD_FaceCPML`` (with a stub ``pyopencl`` module, which the
  reference imports at top level but only uses at call time) on small cases, plus
  its CPML profile arrays and ``ce`` maps.
"""

from __future__ import annotations

import argparse
import os
import sys
import types
import warnings
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def gaussian_sine(t, f0, fwidth):
    """Reference waveform ``tests/meep_validation/harness.py:70-73``."""
    t0 = 5.0 / (np.pi * fwidth)
    sigma = 1.0 / (np.pi * fwidth)
    return float(np.exp(-0.5 * ((t - t0) / sigma) ** 2) * np.sin(2 * np.pi * f0 * t))


def import_reference(root: Path):
    sys.modules.setdefault("pyopencl", types.ModuleType("pyopencl"))
    sys.path.insert(0, str(root))
    import opencl_fdtd_solver as ref  # noqa: E402

    return ref


def sphere_eps(shape, ctr, rad, eps_r):
    ii, jj, kk = np.meshgrid(*[np.arange(n) for n in shape], indexing="ij")
    eps = np.ones(shape, np.float32)
    eps[(ii - ctr) ** 2 + (jj - ctr) ** 2 + (kk - ctr) ** 2 < rad**2] = eps_r
    return eps


def numpy_cases(ref):
    out = {}
    # (1) reference tests/test_solver.py:48-85 — FP32 sphere, full-sheet Ex soft source, 50 steps
    shape, dl, npml, freq = (30, 30, 30), 2e-3, 6, 5e9
    eps = sphere_eps(shape, 15, 6, 4.0)
    z_src = shape[2] - npml - 2
    for name, cls in (("np_sphere", ref.NumPyFDTD), ("npface_sphere", ref.NumPyFDTD_FaceCPML)):
        sim = cls(shape, dl, npml=npml)
        sim.set_epsilon(eps)
        sim.add_source(lambda f: f.add_source_Ex(z_src, np.sin(2 * np.pi * freq * f.t)))
        sim.run(50)
        for fld in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            out[f"{name}_{fld}"] = getattr(sim, fld).copy()
    # (2) reference tests/test_unit_engine.py:340-370 — FP64 vacuum, Jx full sheet, 40 steps
    shape, dl, npml, freq = (24, 24, 24), 2e-3, 4, 4e9
    sim = ref.NumPyFDTD(shape, dl, npml=npml, dtype=np.float64)
    z = shape[2] - npml - 2
    sim.add_source(lambda f: f.add_source_Jx(z, np.sin(2 * np.pi * freq * f.t)))
    sim.run(40)
    for fld in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        out[f"np64_jx_{fld}"] = getattr(sim, fld).copy()
    # (3) reference tests/test_unit_engine.py:438-474 — FP32 Jx rim taper + renorm, 15 steps
    shape, dl, npml, z = (20, 20, 20), 1e-3, 3, 10
    eps = np.ones(shape, np.float32)
    eps[8:12, 8:12, z] = 2.5
    sim = ref.NumPyFDTD(shape, dl, npml=npml)
    sim.set_epsilon(eps)
    sim.add_source(lambda f: f.add_source_Jx(z, 0.4, i0=3, i1=17, j0=3, j1=17, rim_taper=True,
                                             rim_edge=0.8, rim_renorm=True))
    sim.run(15)
    for fld in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
        out[f"np_taper_{fld}"] = getattr(sim, fld).copy()
    # (4) small config: 64^3 FP32 vacuum, npml 8, Courant 0.5, Jx point at the centre,
    #     Gaussian-modulated sine 30 GHz / 20 GHz, 500 steps, z=32 plane DFT at 25/30/35 GHz.
    #     The reference fixes Courant 0.99/sqrt(3); the override rebuilds dt, ce and CPML.
    from opencl_fdtd_solver.constants import C0, EPS0
    from opencl_fdtd_solver.materials import yee_edge_ce

    shape, dl, npml = (64, 64, 64), 1e-3, 8
    sim = ref.NumPyFDTD_FaceCPML(shape, dl, npml=npml)
    sim.dt = 0.5 * dl / C0
    sim._ce_x, sim._ce_y, sim._ce_z = yee_edge_ce(np.ones(shape), sim.dt, dtype=sim.dtype)
    sim._build_cpml()
    assert abs(sim._ce_x[0, 0, 0] - np.float32(sim.dt / EPS0)) == 0
    sim.add_source(lambda f: f.add_source_Jx(32, gaussian_sine(f.t, 30e9, 20e9),
                                             i0=32, i1=33, j0=32, j1=33))
    freqs = np.array([25e9, 30e9, 35e9])
    omega = 2 * np.pi * freqs
    acc = {c: np.zeros((3, 64, 64), np.complex128) for c in ("Ex", "Hy")}
    state = {"p": None}

    def plane_dft(f):
        # phase recurrence of monitors.py:571-584, E at t, H half a step earlier
        if state["p"] is None:
            state["p"] = np.exp(1j * omega * f.t) * f.dt
        else:
            state["p"] = state["p"] * np.exp(1j * omega * f.dt)
        pe = state["p"]
        ph = pe * np.exp(-0.5j * omega * f.dt)
        acc["Ex"] += pe[:, None, None] * f.Ex[:, :, 32].astype(np.float64)[None]
        acc["Hy"] += ph[:, None, None] * f.Hy[:, :, 32].astype(np.float64)[None]

    sim.add_monitor(plane_dft)
    sim.run(500)
    out["small_Ex"] = sim.Ex.copy()
    out["small_Hy"] = sim.Hy.copy()
    out["small_dft_Ex"] = acc["Ex"]
    out["small_dft_Hy"] = acc["Hy"]
    out["small_dt"] = np.float64(sim.dt)
    # (5) CPML profiles and ce maps straight from the reference host math
    from opencl_fdtd_solver.cpml import build_cpml_profiles
    from opencl_fdtd_solver.materials import yee_edge_ca_cb

    for tag, shape, npml, dl, cour, dt_ in (
        ("p0", (30, 26, 22), 5, 2e-3, 0.99 / np.sqrt(3), np.float32),
        ("p1", (64, 64, 64), 8, 1e-3, 0.5, np.float32),
        ("p2", (24, 24, 24), 4, 2e-3, 0.99 / np.sqrt(3), np.float64),
        ("p3", (9, 7, 5), 3, 1e-3, 0.99 / np.sqrt(3), np.float32),
    ):
        dt = cour * dl / C0
        prof = build_cpml_profiles(shape, npml=npml, dl=dl, dt=dt, dtype=dt_)
        out[f"cpml_{tag}_meta"] = np.array([*shape, npml, dl, dt, 1 if dt_ == np.float64 else 0])
        for st in ("e", "h"):
            for ax in range(3):
                p = getattr(prof, st)[ax]
                for fld in ("b", "c", "kappa"):
                    out[f"cpml_{tag}_{st}{ax}_{fld}"] = getattr(p, fld)
    rng = np.random.default_rng(7)
    eps = rng.uniform(1, 12, (9, 10, 11)).astype(np.float32)
    sig = rng.uniform(0, 5, (9, 10, 11))
    out["mat_eps"], out["mat_sig"] = eps, sig
    for dt_, tag in ((np.float32, "f32"), (np.float64, "f64")):
        ce = yee_edge_ce(eps, 1e-12, dtype=dt_)
        (ca, cb) = yee_edge_ca_cb(eps, sig, 1e-12, dtype=dt_)
        for ax in range(3):
            out[f"mat_ce_{tag}_{ax}"] = ce[ax]
            out[f"mat_ca_{tag}_{ax}"] = ca[ax]
            out[f"mat_cb_{tag}_{ax}"] = cb[ax]
    return out


def host_monitor_cases(ref):
    sys.path.insert(0, str(HERE.parents[1]))
    from tests.cases import HOST_MONITOR_CASES, SyntheticFieldSequence

    out = {}
    for tag, shape, dl, dt, seed, center, size, freq, steps in HOST_MONITOR_CASES:
        seq = SyntheticFieldSequence(shape, dl, dt, seed)
        mon = ref.NumPyNear2FarMonitor(seq, center, size, freq)
        for _ in range(steps):
            seq.step()
        out[f"{tag}_box"] = np.array(mon._box)
        for n in SyntheticFieldSequence.FIELDS:
            out[f"{tag}_{n}_dft_f"] = getattr(mon, f"{n}_dft_f").copy()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FDTD_REFERENCE_ROOT"),
                    required="FDTD_REFERENCE_ROOT" not in os.environ,
                    help="reference checkout (default: $FDTD_REFERENCE_ROOT)")
    ap.add_argument("--only", choices=("host_monitor",), default=None,
                    help="write just this fixture")
    args = ap.parse_args(argv)
    root = Path(args.reference)
    if args.only == "host_monitor":
        ref = import_reference(root)
        np.savez_compressed(HERE / "host_monitor.npz", **host_monitor_cases(ref))
        print("wrote host_monitor.npz")
        return
    base = root / "tests/meep_validation/baselines"
    planes = {}
    for case in ("vacuum_sheet", "dielectric_block"):
        for step in (20, 40, 60, 80):
            planes[f"{case}_{step:04d}"] = np.load(base / case / f"ocl_ex_step{step:04d}.npy")
    np.savez_compressed(HERE / "ocl_planes.npz", **planes)
    ff = {}
    for case in ("vacuum_farfield", "dielectric_sphere_farfield"):
        for key in ("ocl_eh_plus_z", "ocl_eh_plus_x", "ocl_S_db", "angles_deg"):
            ff[f"{case}_{key}"] = np.load(base / case / f"{key}.npy")
    np.savez_compressed(HERE / "ocl_farfield.npz", **ff)
    warnings.simplefilter("ignore", DeprecationWarning)
    ref = import_reference(root)
    np.savez_compressed(HERE / "numpy_ref.npz", **numpy_cases(ref))
    np.savez_compressed(HERE / "host_monitor.npz", **host_monitor_cases(ref))
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
