"""Near-to-far contraction on the tensor cores (``fdtd_n2f_contract``).

The far-field sums of the reference kernel ``farfield_accumulate_nl``
(``opencl_fdtd_solver/kernels/dft_farfield.cl:372-556``) are

    NL[f][o] = Σ_faces Σ_{p,q} e^{+j2π f r̂_o·r'_{pq}/c0} · cur_face[f][p][q]

over every face sample r'_{pq} of a Huygens box, for each direction r̂_o and
frequency f.  :func:`near2far_contract` evaluates them for many directions and
frequencies at once.  Each face's phase separates into
``C(o)·u_p(o)·v_q(o)``, so the sum is a complex GEMM over p (directions × (q,
currents)) followed by a reduction over q.  The GEMM runs as ``tcgen05`` MMAs
(split-BF16 hi·hi + hi·lo + lo·hi, or TF32), accumulated in FP32 in TMEM, with
the q reduction fused into the epilogue.  ``mode="fp64"`` is the float64 direct
sum on the CUDA cores, the reference transform the tensor-core modes are
checked against.

:func:`box_faces` turns a :class:`CUDANear2FarMonitor`'s face DFTs into the six
faces' currents: J = n̂×H, M = −n̂×E with the trapezoid weights and dA of
``dft_farfield.cl:431-473``.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _capi as capi

MODES = {"bf16x3": capi.FDTD_N2F_BF16X3, "tf32": capi.FDTD_N2F_TF32, "fp64": capi.FDTD_N2F_FP64}


@dataclass
class N2FFace:
    """One face of sample grid ``np × nq``.

    normal : axis normal to the face (0, 1, 2); p and q run along the other two
             axes in x, y, z order
    x_n    : face coordinate along its normal (m)
    o_p, o_q : in-face coordinates of sample (0, 0) (m)
    pitch  : sample spacing (m)
    cur    : complex64/complex128 device tensor ``[nfreq][np][nq][4]`` holding
             J_p, J_q, M_p, M_q with the quadrature weights applied
    """

    normal: int
    x_n: float
    o_p: float
    o_q: float
    pitch: float
    cur: torch.Tensor


def near2far_contract(faces, freqs, directions, mode="bf16x3", *, stream=None):
    """``NL[f][o][6]`` = (Nx, Ny, Nz, Lx, Ly, Lz) for every frequency and direction.

    faces      : list of 1–6 :class:`N2FFace` on one CUDA device, same dtype and nfreq
    freqs      : frequencies (Hz), length nfreq
    directions : ``(n_obs, 3)`` directions (normalised here)
    mode       : ``"bf16x3"`` or ``"tf32"`` (tensor cores, complex64 result) or
                 ``"fp64"`` (float64 direct sum, complex128 result).  Error against
                 the float64 sums, over their peak: ``"bf16x3"`` ≤ 1e-5 (about 5e-6
                 measured); ``"tf32"`` about 3e-4, outside the 1e-5 class.
    """
    if mode not in MODES:
        raise ValueError(f"mode must be one of {sorted(MODES)}, got {mode!r}")
    faces = list(faces)
    if not 1 <= len(faces) <= 6:
        raise ValueError(f"1 to 6 faces, got {len(faces)}")
    cur0 = faces[0].cur
    if cur0.dtype not in (torch.complex64, torch.complex128):
        raise ValueError(f"currents must be complex64 or complex128, got {cur0.dtype}")
    dev = cur0.device
    if dev.type != "cuda":
        raise ValueError("currents must be on a CUDA device")
    freqs = np.atleast_1d(np.asarray(freqs, dtype=np.float64))
    nfreq = freqs.size
    arr = (capi.N2FFace * len(faces))()
    keep = []
    for i, f in enumerate(faces):
        c = f.cur
        if c.dtype != cur0.dtype or c.device != dev:
            raise ValueError("all faces must share dtype and device")
        if c.dim() != 4 or c.shape[0] != nfreq or c.shape[3] != 4:
            raise ValueError(f"face {i}: cur must be [nfreq={nfreq}][np][nq][4], got "
                             f"{tuple(c.shape)}")
        c = c.contiguous()
        keep.append(c)
        arr[i] = capi.N2FFace(normal=int(f.normal), np=int(c.shape[1]), nq=int(c.shape[2]),
                              x_n=float(f.x_n), o_p=float(f.o_p), o_q=float(f.o_q),
                              pitch=float(f.pitch), cur=c.data_ptr())
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    d = torch.as_tensor(np.asarray(directions, dtype=np.float64), device=dev).reshape(-1, 3)
    n = torch.linalg.vector_norm(d, dim=1, keepdim=True)
    if bool((n == 0).any()):
        raise ValueError("directions must be nonzero")
    d = (d / n).contiguous()
    n_obs = d.shape[0]
    m = MODES[mode]
    need = ctypes.c_uint64()
    capi.run("fdtd_n2f_workspace", arr, len(faces), nfreq, n_obs, m, ctypes.byref(need))
    with torch.cuda.stream(st):
        fr = torch.as_tensor(freqs, device=dev)
        ws = torch.empty(max(1, need.value), dtype=torch.uint8, device=dev)
        out = torch.empty((nfreq, n_obs, 6),
                          dtype=torch.complex128 if mode == "fp64" else torch.complex64,
                          device=dev)
        capi.run("fdtd_n2f_contract", arr, len(faces),
                 capi.FDTD_F32 if cur0.dtype == torch.complex64 else capi.FDTD_F64,
                 fr.data_ptr(), nfreq, d.data_ptr(), n_obs, m, ws.data_ptr(), need.value,
                 out.data_ptr(), st.cuda_stream)
    return out


def box_faces(mon, dtype=torch.complex64):
    """The six faces of a :class:`CUDANear2FarMonitor` (all its frequencies) as
    :class:`N2FFace` currents: J = n̂×H, M = −n̂×E times the trapezoid weight
    (½ on face edges, ¼ at corners) and dA = dl² (``dft_farfield.cl:431-473``),
    at the face sample positions of ``dft_farfield.cl:372-445``."""
    fd = mon.fdtd
    dl = mon.dl
    nf = mon.freqs.size
    acc = torch.view_as_complex(mon.acc)  # [6][nf][n_face]
    (ix0, ix1, iy0, iy1, iz0, iz1) = mon._box
    nx, ny, nz = mon.nxf, mon.nyf, mon.nzf
    offs = mon._face_offsets
    counts = mon._face_counts
    Ex, Ey, Ez, Hx, Hy, Hz = (acc[c] for c in range(6))

    def face(q, shape):
        sl = slice(offs[q], offs[q] + counts[q])
        return [F[:, sl].reshape(nf, *shape) for F in (Ex, Ey, Ez, Hx, Hy, Hz)]

    def weights(n_a, n_b):
        wa = torch.ones(n_a, dtype=torch.float64, device=acc.device)
        wb = torch.ones(n_b, dtype=torch.float64, device=acc.device)
        wa[0] = wa[-1] = 0.5
        wb[0] = wb[-1] = 0.5
        return (wa[:, None] * wb[None, :]) * (dl * dl)

    out = []
    for q in range(6):
        s = -1.0 if q % 2 == 0 else 1.0
        if q < 2:
            ex, ey, ez, hx, hy, hz = face(q, (ny, nz))
            cur = torch.stack([s * hz, -s * hy, -s * ez, s * ey], -1)
            w = weights(ny, nz)
            geo = (0, (ix0 if q == 0 else ix1) * dl, (iy0 + 0.5) * dl, (iz0 + 0.5) * dl)
        elif q < 4:
            ex, ey, ez, hx, hy, hz = face(q, (nx, nz))
            cur = torch.stack([-s * hz, s * hx, s * ez, -s * ex], -1)
            w = weights(nx, nz)
            geo = (1, (iy0 if q == 2 else iy1) * dl, (ix0 + 0.5) * dl, (iz0 + 0.5) * dl)
        else:
            ex, ey, ez, hx, hy, hz = face(q, (nx, ny))
            cur = torch.stack([s * hy, -s * hx, -s * ey, s * ex], -1)
            w = weights(nx, ny)
            geo = (2, (iz0 if q == 4 else iz1) * dl, (ix0 + 0.5) * dl, (iy0 + 0.5) * dl)
        cur = (cur * w[None, :, :, None]).to(dtype).contiguous()
        out.append(N2FFace(normal=geo[0], x_n=geo[1], o_p=geo[2], o_q=geo[3], pitch=dl, cur=cur))
    fd.queue.synchronize()
    return out
