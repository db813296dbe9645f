"""B200 pour-substep engine for PourLab's 3D teapot pour (see include/pourlab.h for the C ABI)."""
from . import abi
from .abi import gentle_pour
from .engine import EngineError, Simulation3D, lib, pcg_solve_device, pcg_solve_device_noalloc

__all__ = ["abi", "gentle_pour", "Simulation3D", "EngineError", "lib", "pcg_solve_device",
           "pcg_solve_device_noalloc"]
