"""ctypes mirror of the plain-data types in include/pourlab.h.

The field order and types here must match the C header exactly; tests/test_abi.py checks the
struct sizes against the values the compiled library reports.
"""
from __future__ import annotations

import ctypes as C

PL_OK = 0
PL_E_ARG = -1
PL_E_CUDA = -2
PL_E_TIMEOUT = -3
PL_E_STATE = -4
PL_E_NOMEM = -5
PL_NONE = 1

AIR, FLUID, SOLID = 0, 1, 2
IN_POT, DISCHARGED, SPILLED, LOST = 0, 1, 2, 3

MOTION_STILL, MOTION_POUR, MOTION_TILT, MOTION_MANUAL = 0, 1, 2, 3
MOTION_KINDS = {"still": MOTION_STILL, "pour": MOTION_POUR, "tilt": MOTION_TILT, "manual": MOTION_MANUAL}
PHASES = ["wait", "tilt-in", "hold", "return", "rest", "done", "manual"]

PRECOND_MIC0, PRECOND_MG, PRECOND_CHEB, PRECOND_BOX_MG, PRECOND_LEARNED = 0, 1, 2, 3, 4
SOLVE_F64, SOLVE_MIXED = 0, 1
TRANSFER_FLIP, TRANSFER_APIC = 0, 1
DOMAIN_HALF, DOMAIN_FULL = 0, 1

FIELD_CELL = 0
FIELD_VELOCITY = 1
FIELD_VELOCITY_PREV = 2
FIELD_PRESSURE = 3
FIELD_CORRECTION = 4
FIELD_VALID = 5
FIELD_DENSITY = 6
FIELD_RHS = 7
U8_FIELDS = (FIELD_CELL, FIELD_VALID)
FACE_FIELDS = (FIELD_VELOCITY, FIELD_VELOCITY_PREV, FIELD_CORRECTION, FIELD_VALID)


class Teapot(C.Structure):
    _fields_ = [
        ("radius", C.c_double),
        ("height", C.c_double),
        ("wall", C.c_double),
        ("inlet_height", C.c_double),
        ("bore_radius", C.c_double),
        ("spout_angle_deg", C.c_double),
        ("spout_length", C.c_double),
    ]


class Motion(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("repeats", C.c_int32),
        ("start_delay", C.c_double),
        ("tilt_duration", C.c_double),
        ("hold_angle_deg", C.c_double),
        ("hold_tilt_rate", C.c_double),
        ("max_angle_deg", C.c_double),
        ("return_duration", C.c_double),
        ("max_hold", C.c_double),
        ("hold_time", C.c_double),
        ("target_volume", C.c_double),
        ("anticipation", C.c_double),
        ("repeat_gap", C.c_double),
        ("settle_time", C.c_double),
    ]


class Config(C.Structure):
    _fields_ = [
        ("teapot", Teapot),
        ("h", C.c_double),
        ("initial_volume", C.c_double),
        ("motion", Motion),
        ("pivot", C.c_double * 2),
        ("gravity", C.c_double),
        ("flip_ratio", C.c_double),
        ("density_correction", C.c_double),
        ("cfl", C.c_double),
        ("max_substep", C.c_double),
        ("pressure_tolerance", C.c_double),
        ("pressure_max_iterations", C.c_int32),
        ("seed", C.c_uint32),
        ("duration", C.c_double),
        ("preconditioner", C.c_int32),
        ("solve_precision", C.c_int32),
        ("device", C.c_int32),
        ("solve_cluster", C.c_int32),
        ("solve_threads", C.c_int32),
        ("transfer", C.c_int32),
        ("domain", C.c_int32),
        ("reserved", C.c_int32),
    ]


class Diagnostics(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("steps", C.c_int64),
        ("angle_deg", C.c_double),
        ("phase", C.c_int32),
        ("particles", C.c_int32),
        ("grid", C.c_int32 * 3),
        ("pressure_iterations", C.c_int32),
        ("pressure_failures", C.c_int32),
        ("correction_iterations", C.c_int32),
        ("discharged_ml", C.c_double),
        ("spilled_ml", C.c_double),
        ("lost_ml", C.c_double),
        ("in_pot_ml", C.c_double),
        ("max_divergence", C.c_double),
        ("interior_density", C.c_double),
        ("liquid_cells", C.c_int32),
        ("reserved", C.c_int32),
    ]

    def as_dict(self) -> dict:
        """Field names and meaning of Diagnostics3D (solver3d.ts:45-60)."""
        return {
            "time": self.time,
            "steps": int(self.steps),
            "angleDeg": self.angle_deg,
            "phase": PHASES[self.phase] if 0 <= self.phase < len(PHASES) else str(self.phase),
            "particles": self.particles,
            "grid": [self.grid[0], self.grid[1], self.grid[2]],
            "dischargedMl": self.discharged_ml,
            "spilledMl": self.spilled_ml,
            "lostMl": self.lost_ml,
            "inPotMl": self.in_pot_ml,
            "pressureIterations": self.pressure_iterations,
            "pressureFailures": self.pressure_failures,
            "correctionIterations": self.correction_iterations,
            "maxDivergence": self.max_divergence,
            "interiorDensity": self.interior_density,
            "liquidCells": self.liquid_cells,
        }


class Sizes(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("h", C.c_double),
        ("parcel_volume", C.c_double),
        ("pivot_world", C.c_double * 2),
        ("fill_height", C.c_double),
        ("band_counts", C.c_int32 * 3),
        ("step_copy_bytes", C.c_int32),
    ]


class ControllerState(C.Structure):
    _fields_ = [
        ("phase", C.c_int32),
        ("pour", C.c_int32),
        ("angle", C.c_double),
        ("phase_start", C.c_double),
        ("start_angle", C.c_double),
        ("start_rate", C.c_double),
        ("last_rate", C.c_double),
        ("flow_rate", C.c_double),
        ("last_discharged", C.c_double),
        ("target", C.c_double),
        ("manual_rate", C.c_double),
    ]


class SimState(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("steps", C.c_int64),
        ("phi", C.c_double),
        ("omega", C.c_double),
        ("counts", C.c_int32 * 4),
        ("discharged_by_origin", C.c_int32 * 3),
        ("last_iterations", C.c_int32),
        ("failures", C.c_int32),
        ("reserved", C.c_int32),
        ("max_div", C.c_double),
        ("interior", C.c_double),
        ("controller", ControllerState),
    ]


ML = 1e-6  # m^3 per millilitre (src/sim/config.ts:9)


def default_teapot() -> Teapot:
    """defaultTeapot3D() (src/sim3d/vessel3d.ts:22-32)."""
    return Teapot(0.065, 0.15, 0.008, 0.035, 0.01, 45.0, 0.14)


def default_motion() -> Motion:
    """defaultMotion() (src/sim/config.ts:168-186) with maxHold 20 (src/sim3d/presets3d.ts:17)."""
    m = Motion()
    m.kind = MOTION_POUR
    m.start_delay = 0.5
    m.tilt_duration = 2.0
    m.hold_angle_deg = 22.0
    m.hold_tilt_rate = 3.0
    m.max_angle_deg = 80.0
    m.return_duration = 1.2
    m.max_hold = 20.0
    m.hold_time = 1.5
    m.target_volume = 400 * ML
    m.anticipation = 0.254
    m.repeats = 1
    m.repeat_gap = 1.5
    m.settle_time = 2.0
    return m


def gentle_pour(cell_mm: float, seconds: float, **over) -> Config:
    """gentlePour3D(cellMm, seconds) (src/sim3d/presets3d.ts:9-26); keyword overrides by field name.

    `motion` may be given as a dict of Motion field overrides (`kind` as a name or number).
    """
    c = Config()
    c.teapot = default_teapot()
    c.h = cell_mm / 1000
    c.initial_volume = 1500 * ML
    c.motion = default_motion()
    c.pivot[0], c.pivot[1] = 0.0, 0.06
    c.gravity = 9.81
    c.flip_ratio = 0.95
    c.density_correction = 0.3
    c.cfl = 0.8
    c.max_substep = 1 / 200
    c.pressure_tolerance = 1e-6
    c.pressure_max_iterations = 400
    c.seed = 1
    c.duration = seconds
    c.preconditioner = PRECOND_MIC0
    c.solve_precision = SOLVE_F64
    c.device = -1
    for k, v in over.items():
        if k == "motion":
            for mk, mv in v.items():
                if mk == "kind" and isinstance(mv, str):
                    mv = MOTION_KINDS[mv]
                setattr(c.motion, mk, mv)
        elif k == "pivot":
            c.pivot[0], c.pivot[1] = v
        else:
            setattr(c, k, v)
    return c
