"""B200-native FDTD engine: a drop-in CUDA backend for the OpenCLFDTD API."""

__version__ = "0.1.0"
