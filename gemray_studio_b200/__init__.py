"""B200 spectral-transport engine for gemray's `gpu`-feature render path.

The compute path is hand-written CUDA for sm_100a behind the C ABI in
``include/gemray_cuda.h`` (built in-tree as ``libgemray_cuda.so`` by ``build.py``).
This package is the host-side mirror of the reference's Rust backend interface
(``GpuBackend`` / ``GpuFrameRenderer``) over that ABI plus scene helpers.  There is
no CPU fallback: without the library or a device, ``GpuBackend.acquire()`` returns a
backend that declines every dispatch, as the reference's does.
"""
from . import abi  # noqa: F401
from .backend import GpuBackend, GpuFrameError, GpuFrameRenderer  # noqa: F401
from .scene import Scene  # noqa: F401
