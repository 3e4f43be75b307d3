"""Host-side logic of the package and the C ABI boundary (CPU only, no kernel launches)."""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path
from unittest import mock

import numpy as np
import pytest

from opencl_fdtd_solver_b200 import _capi as capi
from opencl_fdtd_solver_b200 import cpml, materials
from opencl_fdtd_solver_b200.engine import CUDAFDTD
from opencl_fdtd_solver_b200.monitors import _poynting_db, _poynting_mag
from opencl_fdtd_solver_b200.plugin import BACKENDS, SourceMonitorMixin, get_backend

ROOT = Path(__file__).resolve().parents[1]
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(fdtd_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = capi.lib()
    names = declared_functions()
    assert "fdtd_step" in names and "fdtd_update_H" in names
    for n in names:
        assert hasattr(lib, n), n
        assert n in capi.SIGNATURES, f"{n} has no ctypes signature"
    assert lib.fdtd_version().decode().startswith("fdtd_b200")


def test_ctypes_structs_match_c_header(tmp_path):
    """sizeof/offsetof of every ABI struct, from gcc on the header, equal ctypes'."""
    structs = {"fdtd_grid": capi.Grid, "fdtd_fields": capi.Fields, "fdtd_cpml": capi.Cpml,
               "fdtd_source": capi.Source, "fdtd_plane_dft": capi.PlaneDft, "fdtd_box": capi.Box,
               "fdtd_adjoint_fields": capi.AdjointFields, "fdtd_adjoint_seed": capi.AdjointSeed,
               "fdtd_grad_box": capi.GradBox, "fdtd_n2f_face": capi.N2FFace,
               "fdtd_region": capi.Region}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fdtd_b200.h"',
             'int main(void) {']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        cname, field, val = line.split()
        got[(cname, field)] = int(val)
    for cname, py in structs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_invalid_arguments_return_status_without_launch():
    g = capi.Grid(nx=0, ny=4, nz=4, npml=0, dtype=0)
    f = capi.Fields()
    c = capi.Cpml()
    rc = capi.call("fdtd_update_H", g, f, c, None)
    assert rc == capi.FDTD_ERR_INVALID
    assert "shape" in capi.last_error()
    with pytest.raises(ValueError):
        capi.check(rc, "fdtd_update_H")
    g = capi.Grid(nx=4, ny=4, nz=4, npml=0, dtype=7)
    assert capi.call("fdtd_update_H", g, f, c, None) == capi.FDTD_ERR_INVALID
    assert "dtype" in capi.last_error()
    g = capi.Grid(nx=4, ny=4, nz=4, npml=0, dtype=0)
    assert capi.call("fdtd_update_H", g, f, c, None) == capi.FDTD_ERR_INVALID  # NULL fields
    assert capi.call("fdtd_farfield", None, None, 0, 1.0, 1.0, 1.0, None, 1, None, None,
                     None) == capi.FDTD_ERR_INVALID


def test_read_regions_validates_boxes_without_launch():
    regs = (capi.Region * 2)()
    regs[0].lo[:] = (0, 0, 0)
    regs[0].hi[:] = (4, 5, 0)          # empty along k
    regs[1].lo[:] = (2, 2, 2)
    regs[1].hi[:] = (2, 5, 6)          # empty along i
    # all boxes empty: nothing to copy, so no buffers are needed
    assert capi.call("fdtd_read_regions", None, 0, 4, 5, 6, regs, 2, None, None, None) == 0
    regs[1].lo[0] = 3                  # lo > hi
    assert capi.call("fdtd_read_regions", None, 0, 4, 5, 6, regs, 2, None, None,
                     None) == capi.FDTD_ERR_INVALID
    assert "region 1 axis 0" in capi.last_error()
    regs[1].lo[0], regs[1].hi[2] = 2, 7   # hi beyond Nz
    assert capi.call("fdtd_read_regions", None, 0, 4, 5, 6, regs, 2, None, None,
                     None) == capi.FDTD_ERR_INVALID
    regs[1].hi[:] = (3, 5, 6)          # valid, non-empty: buffers are required
    assert capi.call("fdtd_read_regions", None, 0, 4, 5, 6, regs, 2, None, None,
                     None) == capi.FDTD_ERR_INVALID
    assert "NULL" in capi.last_error()
    many = (capi.Region * (capi.FDTD_MAX_REGIONS + 1))()
    assert capi.call("fdtd_read_regions", None, 0, 4, 5, 6, many, capi.FDTD_MAX_REGIONS + 1,
                     None, None, None) == capi.FDTD_ERR_INVALID
    assert capi.call("fdtd_read_regions", None, 3, 4, 5, 6, regs, 1, None, None,
                     None) == capi.FDTD_ERR_INVALID


def test_product_host_math_matches_reference_arrays(golden):
    g = golden["numpy"]
    for tag in ("p0", "p1", "p2", "p3"):
        meta = g[f"cpml_{tag}_meta"]
        shape = tuple(int(v) for v in meta[:3])
        dtype = np.float64 if meta[6] else np.float32
        prof = cpml.build_cpml_profiles(shape, npml=int(meta[3]), dl=float(meta[4]),
                                        dt=float(meta[5]), dtype=dtype)
        for st in ("e", "h"):
            for ax in range(3):
                p = getattr(prof, st)[ax]
                for fld in ("b", "c", "kappa"):
                    ref = g[f"cpml_{tag}_{st}{ax}_{fld}"]
                    got = getattr(p, fld)
                    assert got.dtype == ref.dtype and np.array_equal(got, ref), (tag, st, ax, fld)
    for dtype, tag in ((np.float32, "f32"), (np.float64, "f64")):
        ce = materials.yee_edge_ce(g["mat_eps"], 1e-12, dtype)
        ca, cb = materials.yee_edge_ca_cb(g["mat_eps"], g["mat_sig"], 1e-12, dtype)
        for ax in range(3):
            assert np.array_equal(ce[ax], g[f"mat_ce_{tag}_{ax}"])
            assert np.array_equal(ca[ax], g[f"mat_ca_{tag}_{ax}"])
            assert np.array_equal(cb[ax], g[f"mat_cb_{tag}_{ax}"])


def test_cpml_profile_properties():
    """Reference ``tests/test_unit_cpml.py:24-49``."""
    from opencl_fdtd_solver_b200.constants import ETA0

    assert cpml.sigma_max(1e-3) == pytest.approx(0.8 * 4 / (ETA0 * 1e-3), rel=1e-15)
    e = cpml.build_cpml_1d(40, npml=8, dl=1e-3, dt=1e-12, node_offset=0.0)
    h = cpml.build_cpml_1d(40, npml=8, dl=1e-3, dt=1e-12, node_offset=0.5)
    assert float(e.kappa[0]) == pytest.approx(cpml.CPML_KAPPA_MAX, abs=1e-5)
    assert float(e.kappa[20]) == 1.0
    assert not np.allclose(e.b[:8], h.b[:8])
    prof = cpml.build_cpml_profiles((16, 20, 24), npml=6, dl=2e-3, dt=1e-12)
    assert prof.e[0].b.shape == (16,) and prof.h[2].kappa.shape == (24,)


def test_lossy_coefficients_closed_form():
    """Reference ``tests/test_materials_lossy.py:16-56``."""
    from opencl_fdtd_solver_b200.constants import EPS0

    eps = np.array([[[1.0, 2.0, 3.0]]])
    (ca, _, _), (cb, _, _) = materials.yee_edge_ca_cb(eps, np.zeros_like(eps), 1e-13, np.float64)
    assert np.array_equal(ca, np.ones_like(ca))
    np.testing.assert_allclose(cb, materials.yee_edge_ce(eps, 1e-13, np.float64)[0])
    e, s, dt = 2.5, 15.0, 3e-13
    (ca, _, _), (cb, _, _) = materials.yee_edge_ca_cb(np.full((3, 3, 3), e), np.full((3, 3, 3), s),
                                                      dt, np.float64)
    loss = s * dt / (2 * EPS0 * e)
    assert ca[1, 1, 1] == pytest.approx((1 - loss) / (1 + loss), rel=1e-12)
    assert cb[1, 1, 1] == pytest.approx(dt / (EPS0 * e) / (1 + loss), rel=1e-12)
    for sv in (100.0, 1000.0, 1e6):
        (ca, _, _), _ = materials.yee_edge_ca_cb(np.ones((2, 2, 2)), np.full((2, 2, 2), sv), 1e-12,
                                                 np.float64)
        assert np.all(ca > -1.0) and np.all(ca <= 1.0)


def test_memory_estimate_matches_reference_formula():
    """Reference ``tests/test_unit_engine.py:97-129``."""
    assert CUDAFDTD.estimate_device_memory_bytes((40, 50, 60), npml=0) == 9 * 40 * 50 * 60 * 4
    npml = 10
    psi = (4 * (2 * npml * 100 * 100) + 4 * (100 * 2 * npml * 100) + 4 * (100 * 100 * 2 * npml)) * 4
    assert CUDAFDTD.estimate_device_memory_bytes((100, 100, 100), npml) == 9 * 100**3 * 4 + psi

    class Dev:
        global_mem_size = 16 * 1024**3

    budget = CUDAFDTD.device_memory_budget_bytes(Dev())
    reserve = Dev.global_mem_size - budget
    assert reserve >= CUDAFDTD.MEMORY_HEADROOM_BYTES
    assert reserve >= int(Dev.global_mem_size * CUDAFDTD.MEMORY_HEADROOM_FRACTION)
    # the engine's own footprint: 12 field arrays + 3 ce + 12 ψ stripes when fused
    fp = CUDAFDTD.device_footprint_bytes((512, 512, 512), 16, np.float32)
    assert fp == (15 * 512**3 + 2 * 3 * 2 * 2 * 16 * 512 * 512) * 4


def test_memory_error_before_allocation():
    """Reference ``tests/test_unit_engine.py:245-257``: a 64 MiB device cannot hold 400³."""
    tiny = mock.Mock()
    tiny.global_mem_size = 64 * 1024 * 1024
    tiny.name = "MockTinyGPU"
    ctx = mock.Mock()
    ctx.devices = [tiny]
    with pytest.raises(MemoryError, match="usable"):
        CUDAFDTD((400, 400, 400), 1e-3, npml=20, ctx=ctx, queue=mock.Mock())


def test_rejects_unsupported_dtype_and_bad_args():
    with pytest.raises(ValueError, match="float32 or float64"):
        CUDAFDTD((8, 8, 8), 1e-3, npml=1, dtype=np.float16)
    with pytest.raises(ValueError):
        CUDAFDTD((8, 0, 8), 1e-3, npml=1)
    with pytest.raises(ValueError):
        CUDAFDTD((8, 8, 8), 1e-3, npml=-1)
    with pytest.raises(ValueError):
        CUDAFDTD((8, 8, 8), 1e-3, npml=1, courant=0.9)


def test_no_device_raises_runtime_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError, match="No CUDA device"):
        CUDAFDTD((8, 8, 8), 1e-3, npml=1)


def test_plugin_registration_contract():
    """Reference ``tests/test_unit_engine.py:483-513`` (mixin) plus the backend registry."""

    class Sim(SourceMonitorMixin):
        def __init__(self):
            self._sources, self._monitors = [], []

    s = Sim()
    with pytest.raises(TypeError):
        s.add_source(None)
    with pytest.raises(TypeError):
        s.add_monitor(3)
    cb = s.add_source(lambda f: None)
    assert callable(cb) and len(s._sources) == 1
    s.add_monitor(lambda f: None)
    s.clear_sources()
    s.clear_monitors()
    assert s._sources == [] and s._monitors == []
    assert BACKENDS["cuda"] is CUDAFDTD and get_backend("CUDA") is CUDAFDTD
    with pytest.raises(KeyError):
        get_backend("opencl")


def test_poynting_helpers():
    """Reference ``tests/test_unit_monitors.py:20-33``."""
    from opencl_fdtd_solver_b200.constants import ETA0

    ff = np.array([1 + 0j, 0, 0, 0, 1 / ETA0, 0], dtype=np.complex128)
    mag = _poynting_mag(ff)
    assert mag == pytest.approx(0.5 / ETA0)
    db, mag2 = _poynting_db(ff)
    assert mag2 == mag and np.isfinite(db)
    db, mag = _poynting_db(np.zeros(6, np.complex128))
    assert mag == 0.0 and db == float("-inf")


def test_public_names_are_documented():
    """Every public name is listed in INTEGRATION.md (idea of reference tests/test_api_docs.py)."""
    import opencl_fdtd_solver_b200 as pkg

    doc = (ROOT / "INTEGRATION.md").read_text()
    for name in pkg.__all__:
        if name.startswith("__"):
            continue
        assert f"`{name}" in doc, name
    for name in declared_functions():
        assert name in doc, name
