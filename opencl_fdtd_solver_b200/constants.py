"""SI electromagnetic constants.

Same definitions as the reference package (``opencl_fdtd_solver/constants.py:11-14``):
``MU0`` is the pre-2019 exact value ``4e-7·π`` and ``EPS0``/``ETA0`` are derived from it,
so every coefficient built from them agrees bit-for-bit with the reference.
"""

from __future__ import annotations

import math

C0 = 299_792_458.0
MU0 = 4e-7 * math.pi
EPS0 = 1.0 / (MU0 * C0**2)
ETA0 = math.sqrt(MU0 / EPS0)

__all__ = ["C0", "MU0", "EPS0", "ETA0"]
