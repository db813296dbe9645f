"""Python host side of the B200 pour engine, mirroring the reference's solver surface.

`Simulation3D` here has the members of PourLab's `Simulation3D` (src/sim3d/solver3d.ts:62-824) and
`GpuSimulation3D` (src/gpu3d/solver.ts:89-490) that callers use: construct from a config, `step`,
`advance`, `stable_dt`, `finished`, `diagnostics`, `discharged_fractions`, `read_particles`,
`read_render_positions`, the controller's `set_target` (setTilt) and the state accessors the
verification harness needs. Every call goes through the C ABI of libpourlab_cuda.so
(include/pourlab.h); there is no CPU fallback, and a missing library is an ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpourlab_cuda.so")

_lib = None

EXPORTED = [
    "pl_default_teapot", "pl_default_motion", "pl_gentle_pour", "pl_create", "pl_destroy", "pl_last_error",
    "pl_get_sizes", "pl_stable_dt", "pl_finished", "pl_step", "pl_advance", "pl_sync", "pl_set_tilt_target",
    "pl_controller", "pl_get_diagnostics", "pl_discharged_fractions", "pl_read_particles",
    "pl_read_particles_f64", "pl_read_origin", "pl_read_render_positions", "pl_get_state", "pl_set_state",
    "pl_get_field", "pl_pcg_solve_device", "pl_enqueue_substeps", "pl_stream", "pl_enable_stage_timing",
    "pl_stage_times", "pl_plan", "pl_autotune_solver", "pl_pcg_solve_device_noalloc",
    "pl_get_affine", "pl_set_affine", "pl_unet_create", "pl_unet_num_params", "pl_unet_get_params",
    "pl_unet_set_params", "pl_unet_apply", "pl_unet_train_step", "pl_unet_gradient", "pl_unet_destroy",
    "pl_unet_set_loss", "pl_set_unet", "pl_unet_set_conv_kernel", "pl_unet_error", "pl_read_quantized_positions", "pl_ensemble_configs", "pl_ensemble_create", "pl_ensemble_size",
    "pl_ensemble_member", "pl_ensemble_advance", "pl_ensemble_enqueue", "pl_ensemble_destroy",
    "pl_inject_fault", "pl_set_wait_limit",
    "pl_poisson_generate", "pl_poisson_gauge_fix", "pl_poisson_create", "pl_poisson_create_box", "pl_poisson_set_unet", "pl_poisson_solve", "pl_poisson_device_bytes", "pl_poisson_history", "pl_poisson_destroy",
]
STAGES = ["bin", "p2g", "pressure", "extrap", "density", "correction", "advect"]


class EngineError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pourlab error {code}: {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Load libpourlab_cuda.so (built by __graft_entry__.build()); raise if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build the CUDA engine first (python -c "
                          f"'import __graft_entry__ as g; g.build()')")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    fp = C.POINTER(C.c_float)
    u8p = C.POINTER(C.c_uint8)
    L.pl_default_teapot.argtypes = [C.POINTER(abi.Teapot)]
    L.pl_default_teapot.restype = None
    L.pl_default_motion.argtypes = [C.POINTER(abi.Motion)]
    L.pl_default_motion.restype = None
    L.pl_gentle_pour.argtypes = [C.c_double, C.c_double, C.POINTER(abi.Config)]
    L.pl_gentle_pour.restype = None
    L.pl_create.argtypes = [C.POINTER(abi.Config), C.POINTER(P)]
    L.pl_destroy.argtypes = [P]
    L.pl_destroy.restype = None
    L.pl_last_error.argtypes = []
    L.pl_last_error.restype = C.c_char_p
    L.pl_get_sizes.argtypes = [P, C.POINTER(abi.Sizes)]
    L.pl_stable_dt.argtypes = [P, dp]
    L.pl_finished.argtypes = [P]
    L.pl_step.argtypes = [P, C.c_double]
    L.pl_advance.argtypes = [P, C.c_double, C.POINTER(abi.Diagnostics)]
    L.pl_sync.argtypes = [P]
    L.pl_set_tilt_target.argtypes = [P, C.c_double, C.c_double]
    L.pl_controller.argtypes = [P, dp, C.POINTER(C.c_int32)]
    L.pl_get_diagnostics.argtypes = [P, C.POINTER(abi.Diagnostics)]
    L.pl_discharged_fractions.argtypes = [P, dp]
    L.pl_read_particles.argtypes = [P, fp, fp, C.POINTER(C.c_uint32)]
    L.pl_read_particles_f64.argtypes = [P, dp, dp, dp, dp, dp, dp, u8p]
    L.pl_read_origin.argtypes = [P, u8p]
    L.pl_read_render_positions.argtypes = [P, fp]
    L.pl_get_state.argtypes = [P, C.POINTER(abi.SimState)]
    L.pl_set_state.argtypes = [P, C.POINTER(abi.SimState), dp, dp, dp, dp, dp, dp, u8p]
    L.pl_get_field.argtypes = [P, C.c_int32, P, C.c_size_t]
    L.pl_pcg_solve_device.argtypes = [P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32, C.c_int32,
                                      C.c_int32, P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), dp]
    L.pl_pcg_solve_device_noalloc.argtypes = [P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_int32, P,
                                              C.POINTER(C.c_int32), C.POINTER(C.c_int32), dp]
    L.pl_plan.argtypes = [C.POINTER(abi.Config), C.POINTER(abi.Sizes), dp, dp, dp, u8p]
    L.pl_autotune_solver.argtypes = [C.POINTER(abi.Config), C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_float)]
    L.pl_enqueue_substeps.argtypes = [P, C.c_int32]
    L.pl_stream.argtypes = [P]
    L.pl_stream.restype = C.c_void_p
    L.pl_enable_stage_timing.argtypes = [P, C.c_int32]
    L.pl_stage_times.argtypes = [P, fp]
    L.pl_inject_fault.argtypes = [C.c_int32, C.c_int32]
    L.pl_set_wait_limit.argtypes = [P, C.c_int32]
    L.pl_unet_create.argtypes = [C.c_uint32, C.POINTER(P)]
    L.pl_unet_num_params.argtypes = [P]
    L.pl_unet_num_params.restype = C.c_int32
    L.pl_unet_get_params.argtypes = [P, fp]
    L.pl_unet_set_params.argtypes = [P, fp]
    L.pl_unet_apply.argtypes = [P, P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P]
    L.pl_unet_train_step.argtypes = [P, P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float, fp, P]
    L.pl_unet_gradient.argtypes = [P, P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, fp, fp, P]
    L.pl_unet_destroy.argtypes = [P]
    L.pl_unet_destroy.restype = None
    L.pl_unet_set_loss.argtypes = [P, C.c_int32]
    L.pl_set_unet.argtypes = [P, P]
    L.pl_unet_set_conv_kernel.argtypes = [P, C.c_int32]
    L.pl_read_quantized_positions.argtypes = [P, C.c_int32, C.c_double, C.POINTER(C.c_uint16)]
    L.pl_unet_error.argtypes = [P]
    L.pl_ensemble_configs.argtypes = [C.c_uint32, C.c_int32, C.c_double, C.c_double, C.POINTER(abi.Config)]
    L.pl_ensemble_create.argtypes = [C.POINTER(abi.Config), C.c_int32, C.POINTER(P)]
    L.pl_ensemble_size.argtypes = [P]
    L.pl_ensemble_size.restype = C.c_int32
    L.pl_ensemble_member.argtypes = [P, C.c_int32]
    L.pl_ensemble_member.restype = P
    L.pl_ensemble_advance.argtypes = [P, C.c_double]
    L.pl_ensemble_enqueue.argtypes = [P, C.c_int32]
    L.pl_ensemble_destroy.argtypes = [P]
    L.pl_ensemble_destroy.restype = None
    L.pl_get_affine.argtypes = [P, fp]
    L.pl_set_affine.argtypes = [P, fp]
    L.pl_poisson_generate.argtypes = [C.c_int32, C.c_int32, C.c_int32, u8p, fp, C.c_int32]
    L.pl_poisson_gauge_fix.argtypes = [C.c_int32, C.c_int32, u8p, fp, C.POINTER(C.c_int32)]
    L.pl_poisson_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(P)]
    L.pl_poisson_create_box.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                        C.POINTER(P)]
    L.pl_poisson_solve.argtypes = [P, P, P, P, C.c_double, C.c_int32, P, C.POINTER(C.c_int32), dp,
                                   C.POINTER(C.c_int32)]
    L.pl_poisson_set_unet.argtypes = [P, P]
    L.pl_poisson_device_bytes.argtypes = [P]
    L.pl_poisson_device_bytes.restype = C.c_size_t
    L.pl_poisson_history.argtypes = [P, C.c_int32, dp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.pl_poisson_destroy.argtypes = [P]
    L.pl_poisson_destroy.restype = None
    _lib = L
    return L


def _check(rc: int) -> int:
    if rc < 0:
        raise EngineError(rc, lib().pl_last_error().decode())
    return rc


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(C.POINTER(t))


def gentle_pour(cell_mm: float, seconds: float, **over) -> abi.Config:
    """gentlePour3D(cellMm, seconds) (src/sim3d/presets3d.ts:9-26) with keyword overrides."""
    return abi.gentle_pour(cell_mm, seconds, **over)


def plan(cfg: abi.Config) -> dict:
    """Host part of the constructor without a device (pl_plan): sizes, seeded parcels, origins."""
    L = lib()
    s = abi.Sizes()
    _check(L.pl_plan(C.byref(cfg), C.byref(s), None, None, None, None))
    n = s.n
    x, y, z = np.zeros(n), np.zeros(n), np.zeros(n)
    o = np.zeros(n, np.uint8)
    _check(L.pl_plan(C.byref(cfg), C.byref(s), _ptr(x, C.c_double), _ptr(y, C.c_double), _ptr(z, C.c_double),
                     _ptr(o, C.c_uint8)))
    return {"sizes": s, "x": x, "y": y, "z": z, "origin": o}


def autotune_solver(cfg: abi.Config, substeps: int = 3) -> tuple[int, int, float]:
    """pl_autotune_solver: (cluster CTAs, threads per CTA, ms per substep) of the fastest shape."""
    c, t, ms = C.c_int32(), C.c_int32(), C.c_float()
    _check(lib().pl_autotune_solver(C.byref(cfg), substeps, C.byref(c), C.byref(t), C.byref(ms)))
    return c.value, t.value, ms.value


class Simulation3D:
    """The pour simulation on one B200 (the reference's Simulation3D / GpuSimulation3D surface)."""

    def __init__(self, cfg: abi.Config, _member=None):
        L = lib()
        self._h = C.c_void_p()
        self._owned = _member is None
        if _member is None:
            _check(L.pl_create(C.byref(cfg), C.byref(self._h)))
        else:  # a pour of an Ensemble, which owns it
            self._h = C.c_void_p(_member)
        self.cfg = cfg
        s = abi.Sizes()
        _check(L.pl_get_sizes(self._h, C.byref(s)))
        self.sizes = s
        self.n, self.nx, self.ny, self.nz = s.n, s.nx, s.ny, s.nz
        self.h = s.h
        self.parcel_volume = s.parcel_volume
        self.pivot_world = (s.pivot_world[0], s.pivot_world[1])
        self.fill_height = s.fill_height
        self.band_counts = [s.band_counts[0], s.band_counts[1], s.band_counts[2]]

    # ------------------------------------------------------------ lifetime
    def destroy(self):
        """GpuSimulation3D.destroy() (src/gpu3d/solver.ts:486-489)."""
        if self._h:
            if self._owned:
                lib().pl_destroy(self._h)
            self._h = C.c_void_p()

    close = destroy

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # ------------------------------------------------------------ sizes
    @property
    def nc(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def nfaces(self) -> int:
        nx, ny, nz = self.nx, self.ny, self.nz
        return (nx + 1) * ny * nz + nx * (ny + 1) * nz + nx * ny * (nz + 1)

    # ------------------------------------------------------------ stepping
    def stable_dt(self) -> float:
        """stableDt() (solver3d.ts:268-278)."""
        out = C.c_double()
        _check(lib().pl_stable_dt(self._h, C.byref(out)))
        return out.value

    @property
    def finished(self) -> bool:
        return bool(lib().pl_finished(self._h))

    def step(self, dt: float = -1.0):
        """step(dt) (solver3d.ts:288-309); dt <= 0 uses min(stableDt(), duration - time)."""
        _check(lib().pl_step(self._h, dt))

    def advance(self, duration: float) -> dict:
        """advance(duration) (solver3d.ts:281-286): whole stable substeps; returns diagnostics()."""
        d = abi.Diagnostics()
        _check(lib().pl_advance(self._h, duration, C.byref(d)))
        return d.as_dict()

    def sync(self):
        _check(lib().pl_sync(self._h))

    def enqueue(self, count: int = 1):
        """Queue `count` stable substeps without waiting (pl_enqueue_substeps)."""
        _check(lib().pl_enqueue_substeps(self._h, count))

    @property
    def stream(self) -> int:
        """cudaStream_t of this simulation (for ordering external work such as timing events)."""
        return lib().pl_stream(self._h) or 0

    def enable_stage_timing(self, on: bool = True):
        _check(lib().pl_enable_stage_timing(self._h, 1 if on else 0))

    def stage_times(self) -> dict:
        """Device milliseconds per stage of the last completed substep."""
        out = np.zeros(len(STAGES), np.float32)
        _check(lib().pl_stage_times(self._h, _ptr(out, C.c_float)))
        return dict(zip(STAGES, out.tolist()))

    def set_wait_limit(self, polls: int):
        """Polls before the bin scan's bounded look-back wait gives up (0: the default); for tests."""
        _check(lib().pl_set_wait_limit(self._h, int(polls)))

    # ------------------------------------------------------------ controller
    def set_target(self, angle_deg: float, time: float | None = None):
        """controller.setTarget(angleDeg, time) (src/sim/motion.ts:40-44): the setTilt of a manual pour."""
        t = self.diagnostics()["time"] if time is None else time
        _check(lib().pl_set_tilt_target(self._h, angle_deg, t))

    set_tilt = set_target

    def controller(self) -> tuple[float, str]:
        a = C.c_double()
        ph = C.c_int32()
        _check(lib().pl_controller(self._h, C.byref(a), C.byref(ph)))
        return a.value, abi.PHASES[ph.value]

    # ------------------------------------------------------------ results
    def diagnostics(self) -> dict:
        """diagnostics() (solver3d.ts:796-814)."""
        d = abi.Diagnostics()
        _check(lib().pl_get_diagnostics(self._h, C.byref(d)))
        return d.as_dict()

    def discharged_fractions(self):
        """dischargedFractions() (solver3d.ts:817-823): None before anything poured."""
        out = np.zeros(3)
        rc = _check(lib().pl_discharged_fractions(self._h, _ptr(out, C.c_double)))
        return None if rc == abi.PL_NONE else out

    def read_particles(self) -> dict:
        """readParticles() (src/gpu3d/solver.ts:409-428): pos/vel as float4 rows, status u32."""
        n = self.n
        pos = np.zeros((n, 4), np.float32)
        vel = np.zeros((n, 4), np.float32)
        st = np.zeros(n, np.uint32)
        _check(lib().pl_read_particles(self._h, _ptr(pos, C.c_float), _ptr(vel, C.c_float), _ptr(st, C.c_uint32)))
        return {"pos": pos, "vel": vel, "status": st}

    def particles(self) -> dict:
        """Parcel state as FP64 SoA in id order (the arrays Simulation3D exposes)."""
        n = self.n
        a = {k: np.zeros(n) for k in ("x", "y", "z", "vx", "vy", "vz")}
        st = np.zeros(n, np.uint8)
        _check(lib().pl_read_particles_f64(self._h, *[_ptr(a[k], C.c_double) for k in ("x", "y", "z", "vx", "vy", "vz")],
                                           _ptr(st, C.c_uint8)))
        a["status"] = st
        return a

    def origin(self) -> np.ndarray:
        o = np.zeros(self.n, np.uint8)
        _check(lib().pl_read_origin(self._h, _ptr(o, C.c_uint8)))
        return o

    def quantized_positions(self, stride: int = 3, quantum: float = 0.00025) -> np.ndarray:
        """A recording frame (pl_read_quantized_positions): every stride-th parcel's position as the
        recording format quantises it, 3 * ceil(n / stride) integers."""
        out = np.zeros(3 * ((self.n + stride - 1) // stride), np.uint16)
        _check(lib().pl_read_quantized_positions(self._h, stride, quantum, _ptr(out, C.c_uint16)))
        return out.astype(np.int64)

    def read_render_positions(self) -> np.ndarray:
        """readRenderPositions() (src/gpu3d/solver.ts:443-475): xyz of the half, then the mirror (full
        domain: the xyz of every parcel)."""
        out = np.zeros((3 if self.cfg.domain == abi.DOMAIN_FULL else 6) * self.n, np.float32)
        _check(lib().pl_read_render_positions(self._h, _ptr(out, C.c_float)))
        return out

    # ------------------------------------------------------------ state (parity harness)
    def get_state(self) -> abi.SimState:
        st = abi.SimState()
        _check(lib().pl_get_state(self._h, C.byref(st)))
        return st

    def set_state(self, st: abi.SimState | None, parts: dict | None):
        ptrs = [None] * 7
        if parts is not None:
            keep = [np.ascontiguousarray(parts[k], dtype=np.float64) for k in ("x", "y", "z", "vx", "vy", "vz")]
            stat = np.ascontiguousarray(parts["status"], dtype=np.uint8)
            ptrs = [_ptr(k, C.c_double) for k in keep] + [_ptr(stat, C.c_uint8)]
        _check(lib().pl_set_state(self._h, C.byref(st) if st is not None else None, *ptrs))

    def affine(self) -> np.ndarray:
        """APIC affine state (pl_get_affine), (n, 3, 3): gradient of component a along axis b."""
        out = np.zeros(self.n * 9, np.float32)
        _check(lib().pl_get_affine(self.handle, _ptr(out, C.c_float)))
        return out.reshape(self.n, 3, 3)

    def set_affine(self, c):
        """pl_set_affine from (n, 3, 3) or one (3, 3) matrix for every parcel."""
        c = np.asarray(c, np.float32)
        if c.shape == (3, 3):
            c = np.broadcast_to(c, (self.n, 3, 3))
        c = np.ascontiguousarray(c).reshape(-1)
        _check(lib().pl_set_affine(self.handle, _ptr(c, C.c_float)))

    def set_unet(self, net: "UNet"):
        """pl_set_unet: the network of a PRECOND_LEARNED simulation (kept alive by this object)."""
        _check(lib().pl_set_unet(self.handle, net._h))
        self._net = net

    def field(self, which: int) -> np.ndarray:
        n = self.nfaces if which in abi.FACE_FIELDS else self.nc
        dtype = np.uint8 if which in abi.U8_FIELDS else np.float64
        out = np.zeros(n, dtype)
        _check(lib().pl_get_field(self._h, which, out.ctypes.data_as(C.c_void_p), n))
        return out


FAULT_ALLOC = 1  # PL_FAULT_ALLOC


def inject_fault(kind: int, count: int = 1):
    """Host-side failure injection (pl_inject_fault): the next `count` device allocations of
    pl_create on this thread fail as an out-of-memory cudaMalloc would."""
    _check(lib().pl_inject_fault(int(kind), int(count)))


def pcg_solve_device(cell_ptr: int, b_ptr: int, q_ptr: int, nx: int, ny: int, nz: int, tol: float, max_iter: int,
                     preconditioner: int = abi.PRECOND_MIC0, precision: int = abi.SOLVE_F64, stream: int = 0):
    """Pcg3D.solve on device buffers (pl_pcg_solve_device): returns (iterations, converged, residual)."""
    it = C.c_int32()
    conv = C.c_int32()
    res = C.c_double()
    _check(lib().pl_pcg_solve_device(C.c_void_p(cell_ptr), C.c_void_p(b_ptr), C.c_void_p(q_ptr), nx, ny, nz, tol,
                                     max_iter, preconditioner, precision, C.c_void_p(stream), C.byref(it),
                                     C.byref(conv), C.byref(res)))
    return it.value, bool(conv.value), res.value


NOALLOC_MAX_CELLS = 262144  # PL_NOALLOC_MAX_CELLS


def pcg_solve_device_noalloc(cell_ptr: int, b_ptr: int, q_ptr: int, nx: int, ny: int, nz: int, tol: float,
                             max_iter: int, stream: int = 0):
    """pcg_solve_device (MIC(0), FP64) with the library's fixed static scratch: allocates no device memory.

    Grids above NOALLOC_MAX_CELLS cells raise EngineError; calls on one device must not overlap."""
    it = C.c_int32()
    conv = C.c_int32()
    res = C.c_double()
    _check(lib().pl_pcg_solve_device_noalloc(C.c_void_p(cell_ptr), C.c_void_p(b_ptr), C.c_void_p(q_ptr), nx, ny, nz,
                                             tol, max_iter, C.c_void_p(stream), C.byref(it), C.byref(conv),
                                             C.byref(res)))
    return it.value, bool(conv.value), res.value


# ------------------------------------------------------------------ Poisson batch

POISSON_MIC0 = 0
POISSON_MG = 1
POISSON_LEARNED = 2
POISSON_PIN = 4


def ensemble_configs(seed: int, count: int, cell_mm: float, seconds: float) -> list:
    """pl_ensemble_configs: seeded gentle pours (fill U[0.6, 1.0] L, peak tilt U[60, 110] deg, tilt-in ramp
    U[4, 12] s)."""
    arr = (abi.Config * count)()
    _check(lib().pl_ensemble_configs(seed, count, cell_mm, seconds, arr))
    return list(arr)


class Ensemble:
    """Many pours on one device (pl_ensemble_*): each pour on its own stream, substeps interleaved."""

    def __init__(self, cfgs: list):
        arr = (abi.Config * len(cfgs))(*cfgs)
        h = C.c_void_p()
        _check(lib().pl_ensemble_create(arr, len(cfgs), C.byref(h)))
        self._h = h
        self.members = [Simulation3D(cfgs[i], _member=lib().pl_ensemble_member(h, i)) for i in range(len(cfgs))]

    def __len__(self):
        return len(self.members)

    def advance(self, duration: float):
        _check(lib().pl_ensemble_advance(self._h, duration))

    def enqueue(self, substeps: int):
        _check(lib().pl_ensemble_enqueue(self._h, substeps))

    def destroy(self):
        if self._h:
            for m in self.members:
                m.destroy()
            lib().pl_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def poisson_generate(n: int, first: int, count: int, threads: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Synthetic snapshots first..first+count-1 (pl_poisson_generate): cells u8 and rhs f32, (count, n^3)."""
    cell = np.zeros((count, n * n * n), np.uint8)
    b = np.zeros((count, n * n * n), np.float32)
    _check(lib().pl_poisson_generate(n, first, count, _ptr(cell, C.c_uint8), _ptr(b, C.c_float), threads))
    return cell, b


def poisson_gauge_fix(n: int, cell: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Gauge fix in place on (count, n^3) cells and rhs (pl_poisson_gauge_fix); returns enclosed counts."""
    count = cell.shape[0]
    assert cell.dtype == np.uint8 and b.dtype == np.float32 and cell.flags.c_contiguous and b.flags.c_contiguous
    enc = np.zeros(count, np.int32)
    _check(lib().pl_poisson_gauge_fix(n, count, _ptr(cell, C.c_uint8), _ptr(b, C.c_float), _ptr(enc, C.c_int32)))
    return enc


class PoissonBatch:
    """Batched dense-grid pressure solver (pl_poisson_create / pl_poisson_solve) on device buffers."""

    def __init__(self, n, count: int, method: int, precision: int):
        """n: the cube's edge, or (nx, ny, nz) of a box (powers of two)."""
        nx, ny, nz = (n, n, n) if isinstance(n, int) else tuple(n)
        self.n, self.count, self.shape = nx, count, (nx, ny, nz)
        h = C.c_void_p()
        _check(lib().pl_poisson_create_box(nx, ny, nz, count, method, precision, C.byref(h)))
        self._h = h

    @property
    def device_bytes(self) -> int:
        return int(lib().pl_poisson_device_bytes(self._h))

    def solve(self, cell_ptr: int, b_ptr: int, x_ptr: int, tol: float, max_iter: int, stream: int = 0):
        """Solve on device pointers (cell u8, b f32, x f64); returns (iterations, residuals, converged)."""
        it = np.zeros(self.count, np.int32)
        res = np.zeros(self.count)
        conv = np.zeros(self.count, np.int32)
        _check(lib().pl_poisson_solve(self._h, C.c_void_p(cell_ptr), C.c_void_p(b_ptr), C.c_void_p(x_ptr), tol,
                                      max_iter, C.c_void_p(stream), _ptr(it, C.c_int32), _ptr(res, C.c_double),
                                      _ptr(conv, C.c_int32)))
        return it, res, conv.astype(bool)

    def history(self, snapshot: int):
        """(max|r| after each of the first 64 iterations of the last solve, iterations with the network)."""
        out = np.zeros(64)
        n, li = C.c_int32(), C.c_int32()
        _check(lib().pl_poisson_history(self._h, snapshot, _ptr(out, C.c_double), 64, C.byref(n), C.byref(li)))
        return out[:n.value].copy(), int(li.value)

    def destroy(self):
        if self._h:
            lib().pl_poisson_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


# ------------------------------------------------------------------ learned preconditioner

UNET_LAYERS = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16),
               (16, 16)]  # (input, output) channels of the 11 convolutions, padded to multiples of 16
UNET_LOSS_L2, UNET_LOSS_ENERGY = 0, 1
UNET_CONV_TCGEN05, UNET_CONV_MMA_SYNC = 0, 1


class UNet:
    """The learned preconditioner's network (pl_unet_*) on device pointers (cell u8, r/z/e f32)."""

    def __init__(self, seed: int = 1):
        h = C.c_void_p()
        _check(lib().pl_unet_create(seed, C.byref(h)))
        self._h = h
        self.nparams = int(lib().pl_unet_num_params(h))

    def set_conv_kernel(self, kind: int):
        """UNET_CONV_TCGEN05 (default) or UNET_CONV_MMA_SYNC (the warp-level tensor-core kernels)."""
        _check(lib().pl_unet_set_conv_kernel(self._h, kind))

    def error(self) -> int:
        """1 if a tensor-core convolution gave up a bounded wait (pl_unet_error)."""
        return int(lib().pl_unet_error(self._h))

    def set_loss(self, kind: int):
        """UNET_LOSS_L2 (relative squared error) or UNET_LOSS_ENERGY (relative error in the energy norm)."""
        _check(lib().pl_unet_set_loss(self._h, kind))

    def params(self) -> np.ndarray:
        out = np.zeros(self.nparams, np.float32)
        _check(lib().pl_unet_get_params(self._h, _ptr(out, C.c_float)))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams
        _check(lib().pl_unet_set_params(self._h, _ptr(p, C.c_float)))

    def apply(self, cell_ptr: int, r_ptr: int, z_ptr: int, nx: int, ny: int, nz: int, count: int, stream: int = 0):
        _check(lib().pl_unet_apply(self._h, C.c_void_p(cell_ptr), C.c_void_p(r_ptr), C.c_void_p(z_ptr), nx, ny, nz,
                                   count, C.c_void_p(stream)))

    def train_step(self, cell_ptr, r_ptr, e_ptr, nx, ny, nz, count, lr: float, stream: int = 0) -> float:
        loss = C.c_float(0)
        _check(lib().pl_unet_train_step(self._h, C.c_void_p(cell_ptr), C.c_void_p(r_ptr), C.c_void_p(e_ptr), nx, ny,
                                        nz, count, lr, C.byref(loss), C.c_void_p(stream)))
        return float(loss.value)

    def gradient(self, cell_ptr, r_ptr, e_ptr, nx, ny, nz, count, stream: int = 0) -> tuple[float, np.ndarray]:
        loss = C.c_float(0)
        g = np.zeros(self.nparams, np.float32)
        _check(lib().pl_unet_gradient(self._h, C.c_void_p(cell_ptr), C.c_void_p(r_ptr), C.c_void_p(e_ptr), nx, ny,
                                      nz, count, C.byref(loss), _ptr(g, C.c_float), C.c_void_p(stream)))
        return float(loss.value), g

    def destroy(self):
        if self._h:
            lib().pl_unet_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
