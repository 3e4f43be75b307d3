"""ctypes bindings for ``libfdtd_b200.so`` (the C ABI declared in ``include/fdtd_b200.h``).

The structures below mirror the header field for field.  Status codes map to
exceptions: ``FDTD_ERR_INVALID`` → ``ValueError``, ``FDTD_ERR_UNSUPPORTED`` →
``NotImplementedError``, anything else → ``RuntimeError`` carrying
``fdtd_last_error()``.  There is no fallback: if the library is missing the
engine fails loudly.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, Structure, c_char_p, c_double, c_int32, c_int64, c_uint64, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfdtd_b200.so"

FDTD_OK = 0
FDTD_ERR_INVALID = 1
FDTD_ERR_CUDA = 2
FDTD_ERR_DEVICE = 3
FDTD_ERR_UNSUPPORTED = 4
FDTD_F32 = 0
FDTD_F64 = 1
FDTD_MAX_SOURCES = 8
FDTD_MAX_PLANES = 4
FDTD_MAX_FREQS = 64
FDTD_MAX_REGIONS = 32
FDTD_NOALLOC_MAX_FACE = 1024 * 256
FDTD_SRC_JX = 0
FDTD_SRC_EX = 1
FDTD_N2F_BF16X3 = 0
FDTD_N2F_TF32 = 1
FDTD_N2F_FP64 = 2
FDTD_WAIT_INTERIOR = 0
FDTD_WAIT_N2F = 1

V3 = c_void_p * 3
V6 = c_void_p * 6


class Grid(Structure):
    _fields_ = [("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("npml", c_int32),
                ("dtype", c_int32), ("lossy", c_int32),
                ("dtm", c_double), ("dtm_dl", c_double), ("inv_dl", c_double),
                ("x_slab", c_int32), ("pml_x_lo", c_int32), ("pml_x_hi", c_int32),
                ("ghost_lo", c_int32), ("ghost_hi", c_int32), ("pad_", c_int32)]


class Fields(Structure):
    _fields_ = [("E", V3), ("H", V3), ("E_next", V3), ("H_next", V3), ("ce", V3), ("ca", V3)]


class Cpml(Structure):
    _fields_ = [("b_h", V3), ("c_h", V3), ("ik_h", V3), ("b_e", V3), ("c_e", V3), ("ik_e", V3),
                ("psi_h", V6), ("psi_h_next", V6), ("psi_e", V6)]


class Source(Structure):
    _fields_ = [("kind", c_int32), ("z", c_int32), ("i0", c_int32), ("i1", c_int32),
                ("j0", c_int32), ("j1", c_int32), ("rim_taper", c_int32), ("pad_", c_int32),
                ("amp", c_double), ("rim_edge", c_double)]


class PlaneDft(Structure):
    _fields_ = [("axis", c_int32), ("index", c_int32), ("comp_mask", c_int32),
                ("nfreq", c_int32), ("acc", c_void_p), ("phase", c_void_p)]


class Box(Structure):
    _fields_ = [("ix0", c_int32), ("ix1", c_int32), ("iy0", c_int32), ("iy1", c_int32),
                ("iz0", c_int32), ("iz1", c_int32), ("off", c_int32 * 6), ("n_face", c_int32),
                ("nfreq", c_int32)]


class AdjointFields(Structure):
    _fields_ = [("E", V3), ("H", V3), ("pe", V6), ("pe_next", V6), ("ph", V6), ("ph_next", V6),
                ("ce", V3), ("E_next", V3), ("H_next", V3)]


class AdjointSeed(Structure):
    _fields_ = [("axis", c_int32), ("index", c_int32), ("a0", c_int32), ("a1", c_int32),
                ("b0", c_int32), ("b1", c_int32), ("comp_mask", c_int32), ("nfreq", c_int32),
                ("seed", c_void_p), ("phase", c_void_p)]


class GradBox(Structure):
    _fields_ = [("lo", c_int32 * 3), ("hi", c_int32 * 3), ("e_next", c_void_p),
                ("e_prev", c_void_p), ("g", c_void_p)]


class Region(Structure):
    _fields_ = [("lo", c_int32 * 3), ("hi", c_int32 * 3)]


class N2FFace(Structure):
    _fields_ = [("normal", c_int32), ("np", c_int32), ("nq", c_int32), ("pad_", c_int32),
                ("x_n", c_double), ("o_p", c_double), ("o_q", c_double), ("pitch", c_double),
                ("cur", c_void_p)]


# name -> (restype, argtypes); every symbol include/fdtd_b200.h declares.
SIGNATURES = {
    "fdtd_update_H": (c_int32, [POINTER(Grid), POINTER(Fields), POINTER(Cpml), c_void_p]),
    "fdtd_update_E": (c_int32, [POINTER(Grid), POINTER(Fields), POINTER(Cpml), POINTER(Source),
                                c_int32, POINTER(PlaneDft), c_int32, c_void_p]),
    "fdtd_step": (c_int32, [POINTER(Grid), POINTER(Fields), POINTER(Cpml), POINTER(Source),
                            c_int32, POINTER(PlaneDft), c_int32, c_void_p]),
    "fdtd_add_source": (c_int32, [POINTER(Grid), c_void_p, c_void_p, POINTER(Source), c_void_p]),
    "fdtd_dft_faces": (c_int32, [POINTER(Grid), POINTER(c_void_p), POINTER(c_void_p),
                                 POINTER(Box), c_void_p, c_void_p, c_void_p]),
    "fdtd_rel_change_blocks": (c_int32, [c_int32]),
    "fdtd_dft_rel_change": (c_int32, [c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p,
                                      c_void_p, c_void_p]),
    "fdtd_dft_rel_change_noalloc": (c_int32, [c_void_p, c_void_p, c_int32, c_int32, c_int32,
                                              c_void_p, c_void_p]),
    "fdtd_farfield": (c_int32, [POINTER(Box), c_void_p, c_int32, c_double, c_double, c_double,
                                c_void_p, c_int32, c_void_p, c_void_p, c_void_p]),
    "fdtd_capture_box": (c_int32, [POINTER(Grid), POINTER(c_void_p), POINTER(c_int32),
                                   POINTER(c_int32), c_void_p, c_void_p]),
    "fdtd_read_regions": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_int32,
                                    POINTER(Region), c_int32, c_void_p, c_void_p, c_void_p]),
    "fdtd_adjoint_seed_add": (c_int32, [POINTER(Grid), POINTER(c_void_p), POINTER(AdjointSeed),
                                        c_void_p]),
    "fdtd_adjoint_step": (c_int32, [POINTER(Grid), POINTER(AdjointFields), POINTER(Cpml),
                                    POINTER(GradBox), POINTER(AdjointSeed), c_void_p]),
    "fdtd_set_epsilon": (c_int32, [POINTER(Grid), c_void_p, c_void_p, c_int32, c_double,
                                   c_double, POINTER(c_void_p), POINTER(c_void_p), c_void_p]),
    "fdtd_profile_steps": (c_int32, [c_int32]),
    "fdtd_profile_read": (c_int32, [POINTER(c_double), POINTER(c_int32)]),
    "fdtd_launch_count": (c_int64, []),
    "fdtd_farfield_eh": (c_int32, [c_void_p, c_int32, c_void_p, c_int32, c_double, c_double,
                                   c_void_p, c_void_p]),
    "fdtd_n2f_workspace": (c_int32, [POINTER(N2FFace), c_int32, c_int32, c_int32, c_int32,
                                     POINTER(c_uint64)]),
    "fdtd_n2f_contract": (c_int32, [POINTER(N2FFace), c_int32, c_int32, c_void_p, c_int32,
                                    c_void_p, c_int32, c_int32, c_void_p, c_uint64, c_void_p,
                                    c_void_p]),
    "fdtd_last_error": (c_char_p, []),
    "fdtd_device_status": (c_int32, [POINTER(c_int32), c_int32]),
    "fdtd_set_wait_budget": (c_int32, [c_int32, c_int64]),
    "fdtd_version": (c_char_p, []),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load the library once; raise ``RuntimeError`` if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built; run `python -m opencl_fdtd_solver_b200.build`")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def last_error() -> str:
    msg = lib().fdtd_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    """Raise the exception class matching status ``rc``."""
    if rc == FDTD_OK:
        return
    msg = f"{what}: {last_error()}"
    if rc == FDTD_ERR_INVALID:
        raise ValueError(msg)
    if rc == FDTD_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise RuntimeError(msg)


def call(name: str, *args) -> int:
    """Call ``name`` and return its raw status (no exception)."""
    return getattr(lib(), name)(*args)


def run(name: str, *args) -> None:
    """Call ``name`` and raise on a non-OK status."""
    check(getattr(lib(), name)(*args), name)
