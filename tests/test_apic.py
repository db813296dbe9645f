"""APIC transfer: the 3D form of the 2D solver's affine particle-grid transfer (src/sim/solver.ts:543-590,
944-990). The 3D reference has no APIC, so parity is pinned by an invariant (an affine velocity field
survives the particle-to-grid transfer exactly) on the oracle, and by the engine agreeing with the oracle."""
import numpy as np
import pytest

from teapotfluidsimulation_b200 import abi


def face_positions(nx, ny, nz, h):
    out = []
    for comp, (sx, sy, sz) in enumerate([(nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1)]):
        k, j, i = np.meshgrid(np.arange(sz), np.arange(sy), np.arange(sx), indexing="ij")
        off = [0.5, 0.5, 0.5]
        off[comp] = 0.0
        out.append((comp, np.stack([(i + off[0]) * h, (j + off[1]) * h, (k + off[2]) * h], -1).reshape(-1, 3)))
    return out


G = np.array([[0.3, -0.2, 0.1], [0.05, 0.4, -0.1], [0.2, 0.0, -0.3]])
V0 = np.array([0.01, -0.02, 0.005])


def affine_p2g_error(sim, parts, field_prev):
    X = np.stack([parts["x"], parts["y"], parts["z"]], 1)
    V = V0 + X @ G.T
    sim.set_state(None, {"x": parts["x"], "y": parts["y"], "z": parts["z"], "vx": V[:, 0], "vy": V[:, 1],
                         "vz": V[:, 2], "status": parts["status"]})
    sim.set_affine(G)
    sim.step(1e-7)
    prev = field_prev()
    worst, base, touched = 0.0, 0, 0
    for comp, xf in face_positions(sim.nx, sim.ny, sim.nz, sim.h):
        nfc = len(xf)
        got = prev[base:base + nfc]
        base += nfc
        expect = V0[comp] + xf @ G[comp]
        m = got != 0
        touched += int(m.sum())
        worst = max(worst, float(np.abs(got[m] - expect[m]).max()))
    return worst, touched


def test_oracle_apic_p2g_is_exact_for_affine_fields(oracle_mod):
    cfg = abi.gentle_pour(10, 1.0, transfer=abi.TRANSFER_APIC)
    sim = oracle_mod.OracleSim(cfg)
    worst, touched = affine_p2g_error(sim, sim.particles(), lambda: sim.field(abi.FIELD_VELOCITY_PREV))
    assert touched > 1000 and worst < 1e-12


def test_oracle_flip_p2g_is_not(oracle_mod):
    # the same parcels without the affine term smear the field: the invariant is APIC's, not the stencil's
    cfg = abi.gentle_pour(10, 1.0)
    sim = oracle_mod.OracleSim(cfg)
    parts = sim.particles()
    X = np.stack([parts["x"], parts["y"], parts["z"]], 1)
    V = V0 + X @ G.T
    sim.set_state(None, {"x": parts["x"], "y": parts["y"], "z": parts["z"], "vx": V[:, 0], "vy": V[:, 1],
                         "vz": V[:, 2], "status": parts["status"]})
    sim.step(1e-7)
    prev = sim.field(abi.FIELD_VELOCITY_PREV)
    xf = face_positions(sim.nx, sim.ny, sim.nz, sim.h)[0][1]
    got = prev[:len(xf)]
    m = got != 0
    assert np.abs(got[m] - (V0[0] + xf[m] @ G[0])).max() > 1e-4


def test_oracle_apic_at_rest_settles_faster_than_flip(oracle_mod):
    # 5 mm (the 2 cm spout bore spans cells; at 10 mm it is one cell wide and the wall shear there makes
    # the affine terms large): a pot at rest keeps its liquid, and APIC dissipates more than FLIP/PIC
    ke = {}
    for tr in (abi.TRANSFER_FLIP, abi.TRANSFER_APIC):
        sim = oracle_mod.OracleSim(abi.gentle_pour(5, 0.3, transfer=tr, motion={"kind": "still"}))
        d = sim.advance(0.3)
        assert d["lostMl"] == 0 and d["spilledMl"] == 0 and d["pressureFailures"] == 0
        p = sim.particles()
        ke[tr] = 0.5 * float((p["vx"] ** 2 + p["vy"] ** 2 + p["vz"] ** 2).sum())
        if tr == abi.TRANSFER_APIC:
            assert np.abs(sim.affine()).max() > 0
    assert ke[abi.TRANSFER_APIC] < ke[abi.TRANSFER_FLIP]


@pytest.mark.gpu
def test_engine_apic_p2g_is_exact_for_affine_fields(engine):
    cfg = abi.gentle_pour(10, 1.0, transfer=abi.TRANSFER_APIC)
    sim = engine.Simulation3D(cfg)
    worst, touched = affine_p2g_error(sim, sim.particles(), lambda: sim.field(abi.FIELD_VELOCITY_PREV))
    sim.destroy()
    # FP32 parcels, FP32 affine vectors and FP32 node partials: exact to single precision
    assert touched > 1000 and worst < 2e-6


@pytest.mark.gpu
def test_engine_apic_follows_the_oracle(engine, oracle_mod):
    cfg = abi.gentle_pour(10, 1.0, transfer=abi.TRANSFER_APIC)
    gpu = engine.Simulation3D(cfg)
    cpu = oracle_mod.OracleSim(cfg)
    for _ in range(3):
        dt = cpu.stable_dt()
        cpu.step(dt)
        gpu.step(dt)
    for f in (abi.FIELD_VELOCITY, abi.FIELD_VELOCITY_PREV):
        a, b = gpu.field(f), cpu.field(f)
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), f
    pa, pb = gpu.particles(), cpu.particles()
    rms = np.sqrt(((pa["x"] - pb["x"]) ** 2 + (pa["y"] - pb["y"]) ** 2 + (pa["z"] - pb["z"]) ** 2).mean()) / gpu.h
    assert rms < 1e-4
    ca, cb = gpu.affine(), cpu.affine()
    assert np.linalg.norm(ca - cb) <= 1e-4 * np.linalg.norm(cb)
    gpu.destroy()
