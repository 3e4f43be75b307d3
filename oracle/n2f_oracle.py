"""CPU restatement of the near-to-far surface sums for arbitrary face grids (TEST INFRASTRUCTURE).

``NL[f][o][c] = Σ_faces Σ_{p,q} e^{+j2π f r̂_o·r'_{pq}/c0} cur[f][p][q][c']`` in
complex128, the sum of ``farfield_accumulate_nl``
(``opencl_fdtd_solver/kernels/dft_farfield.cl:372-556``) with the face currents
given directly: face-local currents (J_p, J_q, M_p, M_q) map to NL components
(p, q, 3+p, 3+q) for the in-face axes p < q.  A direct sum (no separation of the
phase), so it also checks the separable factorisation the GPU kernel uses.
Only tests import this module.
"""

from __future__ import annotations

import numpy as np

C0 = 299_792_458.0


def face_axes(normal):
    return [a for a in range(3) if a != normal]


def contract(faces, freqs, dirs, chunk=512):
    """faces: list of dicts ``normal, x_n, o_p, o_q, pitch, cur`` (complex
    ``[nfreq][np][nq][4]``); dirs: ``(n_obs, 3)``.  Returns complex128 ``(nfreq, n_obs, 6)``."""
    d = np.asarray(dirs, np.float64).reshape(-1, 3)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    freqs = np.atleast_1d(np.asarray(freqs, np.float64))
    out = np.zeros((freqs.size, d.shape[0], 6), np.complex128)
    for f in faces:
        cur = np.asarray(f["cur"], np.complex128)
        nf, np_, nq, _ = cur.shape
        a, b = face_axes(f["normal"])
        pos = np.zeros((np_, nq, 3))
        pos[..., f["normal"]] = f["x_n"]
        pos[..., a] = (f["o_p"] + f["pitch"] * np.arange(np_))[:, None]
        pos[..., b] = (f["o_q"] + f["pitch"] * np.arange(nq))[None, :]
        pos = pos.reshape(-1, 3)
        comp = [a, b, 3 + a, 3 + b]
        for fi, fr in enumerate(freqs):
            x = cur[fi].reshape(-1, 4)
            for o0 in range(0, d.shape[0], chunk):
                ph = np.exp(1j * 2.0 * np.pi * fr / C0 * (d[o0:o0 + chunk] @ pos.T))
                r = ph @ x
                for c in range(4):
                    out[fi, o0:o0 + chunk, comp[c]] += r[:, c]
    return out
