"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU FP64 oracle (oracle/pourlab_oracle.cpp).

The oracle restates PourLab's src/sim3d solver on the CPU. Tests use it as the checker of the
CUDA engine, and bench.py times it as the CPU baseline. The engine itself never imports this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from teapotfluidsimulation_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpourlab_oracle.so")

_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        dp = C.POINTER(C.c_double)
        u8p = C.POINTER(C.c_uint8)
        L.plo_create.argtypes = [C.POINTER(abi.Config), C.POINTER(P)]
        L.plo_destroy.argtypes = [P]
        L.plo_get_sizes.argtypes = [P, C.POINTER(abi.Sizes)]
        L.plo_stable_dt.argtypes = [P]
        L.plo_stable_dt.restype = C.c_double
        L.plo_finished.argtypes = [P]
        L.plo_step.argtypes = [P, C.c_double]
        L.plo_advance.argtypes = [P, C.c_double, C.POINTER(abi.Diagnostics)]
        L.plo_set_tilt_target.argtypes = [P, C.c_double, C.c_double]
        L.plo_diagnostics.argtypes = [P, C.POINTER(abi.Diagnostics)]
        L.plo_discharged_fractions.argtypes = [P, dp]
        L.plo_read_particles.argtypes = [P, dp, dp, dp, dp, dp, dp, u8p]
        L.plo_read_origin.argtypes = [P, u8p]
        L.plo_read_y0.argtypes = [P, C.POINTER(C.c_float)]
        L.plo_discharge_order.argtypes = [P, C.POINTER(C.c_int32), C.c_int32]
        L.plo_get_state.argtypes = [P, C.POINTER(abi.SimState)]
        L.plo_set_state.argtypes = [P, C.POINTER(abi.SimState), dp, dp, dp, dp, dp, dp, u8p]
        L.plo_get_field.argtypes = [P, C.c_int32, P, C.c_size_t]
        L.plo_pcg_solve.argtypes = [u8p, dp, dp, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32,
                                    C.POINTER(C.c_int32), dp]
        L.plo_get_affine.argtypes = [P, dp]
        L.plo_set_affine.argtypes = [P, dp]
        L.plo_poisson_solve.argtypes = [u8p, dp, dp, C.c_int32, C.c_double, C.c_int32, C.POINTER(C.c_int32), dp]
        L.plo_poisson_solve_box.argtypes = [u8p, dp, dp, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32,
                                            C.POINTER(C.c_int32), dp]
        L.plo_teapot_sdf.argtypes = [C.POINTER(abi.Teapot), C.c_double, C.c_double, C.c_double]
        L.plo_teapot_sdf.restype = C.c_double
        L.plo_in_cavity.argtypes = [C.POINTER(abi.Teapot), C.c_double, C.c_double, C.c_double]
        L.plo_rng.argtypes = [C.c_uint32, C.c_int32, dp]
        L.plo_js_hypot3.argtypes = [C.c_double, C.c_double, C.c_double]
        L.plo_js_hypot3.restype = C.c_double
        _lib = L
    return _lib


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(C.POINTER(t))


class OracleSim:
    """Simulation3D (solver3d.ts:62-824) on the CPU, FP64, one thread."""

    def __init__(self, cfg: abi.Config):
        L = lib()
        self._h = C.c_void_p()
        rc = L.plo_create(C.byref(cfg), C.byref(self._h))
        if rc != 0:
            raise ValueError(f"oracle create failed: {rc}")
        self.cfg = cfg
        s = abi.Sizes()
        L.plo_get_sizes(self._h, C.byref(s))
        self.sizes = s
        self.n, self.nx, self.ny, self.nz = s.n, s.nx, s.ny, s.nz
        self.h = s.h

    def close(self):
        if self._h:
            lib().plo_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nc(self):
        return self.nx * self.ny * self.nz

    @property
    def nfaces(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        return (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)

    def stable_dt(self) -> float:
        return lib().plo_stable_dt(self._h)

    @property
    def finished(self) -> bool:
        return bool(lib().plo_finished(self._h))

    def step(self, dt: float = -1.0):
        lib().plo_step(self._h, dt)

    def advance(self, duration: float) -> dict:
        d = abi.Diagnostics()
        lib().plo_advance(self._h, duration, C.byref(d))
        return d.as_dict()

    def set_tilt_target(self, angle_deg: float, time: float):
        lib().plo_set_tilt_target(self._h, angle_deg, time)

    def diagnostics(self) -> dict:
        d = abi.Diagnostics()
        lib().plo_diagnostics(self._h, C.byref(d))
        return d.as_dict()

    def discharged_fractions(self):
        out = np.zeros(3)
        rc = lib().plo_discharged_fractions(self._h, _ptr(out, C.c_double))
        return None if rc == abi.PL_NONE else out

    def particles(self) -> dict:
        n = self.n
        a = {k: np.zeros(n) for k in ("x", "y", "z", "vx", "vy", "vz")}
        st = np.zeros(n, np.uint8)
        lib().plo_read_particles(self._h, *[_ptr(a[k], C.c_double) for k in ("x", "y", "z", "vx", "vy", "vz")],
                                 _ptr(st, C.c_uint8))
        a["status"] = st
        return a

    def origin(self) -> np.ndarray:
        o = np.zeros(self.n, np.uint8)
        lib().plo_read_origin(self._h, _ptr(o, C.c_uint8))
        return o

    def y0(self) -> np.ndarray:
        o = np.zeros(self.n, np.float32)
        lib().plo_read_y0(self._h, _ptr(o, C.c_float))
        return o

    def discharge_order(self) -> np.ndarray:
        n = lib().plo_discharge_order(self._h, None, 0)
        o = np.zeros(max(n, 1), np.int32)
        lib().plo_discharge_order(self._h, _ptr(o, C.c_int32), n)
        return o[:n]

    def get_state(self) -> abi.SimState:
        st = abi.SimState()
        lib().plo_get_state(self._h, C.byref(st))
        return st

    def set_state(self, st: abi.SimState | None, parts: dict | None):
        ptrs = [None] * 7
        if parts is not None:
            keep = [np.ascontiguousarray(parts[k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz")]
            stat = np.ascontiguousarray(parts["status"], dtype=np.uint8)
            ptrs = [_ptr(k, C.c_double) for k in keep] + [_ptr(stat, C.c_uint8)]
        lib().plo_set_state(self._h, C.byref(st) if st is not None else None, *ptrs)

    def affine(self) -> np.ndarray:
        """APIC affine state, (n, 3, 3): gradient of component a along axis b."""
        out = np.zeros(self.n * 9)
        lib().plo_get_affine(self._h, _ptr(out, C.c_double))
        return out.reshape(self.n, 3, 3)

    def set_affine(self, c):
        """Set the APIC affine state from (n, 3, 3) or a (3, 3) matrix for every parcel."""
        c = np.asarray(c, np.float64)
        if c.shape == (3, 3):
            c = np.broadcast_to(c, (self.n, 3, 3))
        c = np.ascontiguousarray(c).reshape(-1)
        lib().plo_set_affine(self._h, _ptr(c, C.c_double))

    def field(self, which: int) -> np.ndarray:
        n = self.nfaces if which in abi.FACE_FIELDS else self.nc
        dtype = np.uint8 if which in abi.U8_FIELDS else np.float64
        out = np.zeros(n, dtype)
        rc = lib().plo_get_field(self._h, which, out.ctypes.data_as(C.c_void_p), n)
        if rc != 0:
            raise ValueError(f"field {which}: {rc}")
        return out


def pcg_solve(cell: np.ndarray, b: np.ndarray, nx: int, ny: int, nz: int, tol: float, max_iter: int):
    """Pcg3D.solve (solver3d.ts:858-937): returns (q, iterations, converged, residual)."""
    cell = np.ascontiguousarray(cell, np.uint8)
    b = np.ascontiguousarray(b, np.float64)
    q = np.zeros_like(b)
    conv = C.c_int32()
    res = C.c_double()
    it = lib().plo_pcg_solve(_ptr(cell, C.c_uint8), _ptr(b, C.c_double), _ptr(q, C.c_double), nx, ny, nz, tol,
                             max_iter, C.byref(conv), C.byref(res))
    return q, it, bool(conv.value), res.value


def poisson_solve(cell: np.ndarray, b: np.ndarray, n, tol: float = 1e-12, max_iter: int = 4000):
    """FP64 MIC(0)-PCG of one dense Poisson snapshot (cells may carry the pin flag 4); n is the cube's edge
    or (nx, ny, nz)."""
    L = lib()
    nx, ny, nz = (n, n, n) if isinstance(n, int) else tuple(n)
    cell = np.ascontiguousarray(cell, np.uint8)
    b = np.ascontiguousarray(b, np.float64)
    q = np.zeros(nx * ny * nz)
    conv = C.c_int32(0)
    res = C.c_double(0)
    it = L.plo_poisson_solve_box(_ptr(cell, C.c_uint8), _ptr(b, C.c_double), _ptr(q, C.c_double), nx, ny, nz, tol,
                                 max_iter, C.byref(conv), C.byref(res))
    return q, it, bool(conv.value), res.value


def teapot_sdf(x, y, z, teapot=None) -> float:
    t = teapot or abi.default_teapot()
    return lib().plo_teapot_sdf(C.byref(t), x, y, z)


def in_cavity(x, y, z, teapot=None) -> bool:
    t = teapot or abi.default_teapot()
    return bool(lib().plo_in_cavity(C.byref(t), x, y, z))


def rng(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    lib().plo_rng(seed, n, _ptr(out, C.c_double))
    return out


def js_hypot3(a, b, c) -> float:
    return lib().plo_js_hypot3(a, b, c)
