"""B200-native FDTD engine: a CUDA drop-in for the ``OpenCLFDTD`` API.

Public surface (mirrors the reference ``opencl_fdtd_solver/__init__.py:10-21``,
with ``CUDAFDTD`` / ``CUDANear2FarMonitor`` in place of the OpenCL classes):

* constants ``C0, MU0, EPS0, ETA0``
* ``CUDAFDTD`` — Yee/CPML engine on one CUDA device
* ``CUDANear2FarMonitor`` — Huygens-box DFT + far field
* ``CUDAPlaneDFTMonitor`` — single-plane DFT fused into the E update
* ``NumPyNear2FarMonitor`` — the reference's host Huygens-box monitor; on
  ``CUDAFDTD`` its per-step reads move only the face slabs it declares
* ``StepCallback``, ``SourceMonitorMixin``, ``BACKENDS``, ``get_backend``
* ``near2far_contract``, ``N2FFace``, ``box_faces`` — near-to-far sums for many
  directions and frequencies on the tensor cores (split-BF16 / TF32) or in FP64
* ``DFTObjective``, ``EpsilonAdjoint``, ``EpsilonObjective`` — discrete-adjoint
  ε-gradient of a plane-DFT objective (``EpsilonObjective`` is the
  ``torch.autograd.Function``)

Importing the package does not touch CUDA; constructing an engine does.
"""

__version__ = "0.1.0"

from .adjoint import DFTObjective, EpsilonAdjoint, EpsilonObjective, epsilon_objective
from .constants import C0, EPS0, ETA0, MU0
from .engine import CUDAFDTD
from .monitors import CUDANear2FarMonitor, CUDAPlaneDFTMonitor, NumPyNear2FarMonitor
from .n2f import N2FFace, box_faces, near2far_contract
from .plugin import BACKENDS, SourceMonitorMixin, StepCallback, get_backend, register_backend

__all__ = [
    "C0",
    "MU0",
    "EPS0",
    "ETA0",
    "CUDAFDTD",
    "CUDANear2FarMonitor",
    "CUDAPlaneDFTMonitor",
    "NumPyNear2FarMonitor",
    "StepCallback",
    "SourceMonitorMixin",
    "BACKENDS",
    "get_backend",
    "register_backend",
    "near2far_contract",
    "N2FFace",
    "box_faces",
    "DFTObjective",
    "EpsilonAdjoint",
    "EpsilonObjective",
    "epsilon_objective",
    "__version__",
]
