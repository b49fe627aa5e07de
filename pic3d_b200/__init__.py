"""pic3d_b200: the PIC3D per-timestep loop (Yee FDTD, gather + Boris push,
Esirkepov deposition) as hand-written sm_100a CUDA kernels behind a C ABI
(include/pic3d_gpu.h), with a host mirror of the reference call surface."""
from . import workloads  # noqa: F401

__all__ = ["workloads", "Simulation", "load_library"]


def load_library():
    from . import _lib
    return _lib.load()


def __getattr__(name):
    if name == "Simulation":
        from .simulation import Simulation
        return Simulation
    raise AttributeError(name)
