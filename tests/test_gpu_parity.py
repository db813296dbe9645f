"""The CUDA engine against the CPU oracle, through the C ABI (needs a GPU).

Tolerances (the engine stores parcels and face velocities in FP32, the oracle is FP64):
  - cell classification, valid masks, origin tags, binning: bit-exact;
  - per-substep fields from an identical state (pressure, projected velocity, particle-to-grid
    velocity): relative L2 < 1e-5;
  - the reference's own GPU-vs-CPU step comparison (e2e/gpuSolver.spec.ts:31-41): 20 substeps at
    10 mm, RMS position < 1e-3 cells, max < 1e-2 cells, relative velocity RMS < 1e-3, no status
    mismatch, no pressure failure, nothing lost.
"""
import numpy as np
import pytest

from teapotfluidsimulation_b200 import abi

pytestmark = pytest.mark.gpu

REL_FIELD = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def lockstep(engine, oracle_mod, cfg, steps):
    gpu = engine.Simulation3D(cfg)
    cpu = oracle_mod.OracleSim(cfg)
    for _ in range(steps):
        if cpu.finished:
            break
        dt = min(cpu.stable_dt(), cfg.duration - cpu.diagnostics()["time"])
        cpu.step(dt)
        gpu.step(dt)
    return gpu, cpu


def compare_particles(gpu, cpu):
    """The reference's step comparison (src/gpu3d/verify.ts:38-67)."""
    a, b = gpu.particles(), cpu.particles()
    mism = int((a["status"] != b["status"]).sum())
    m = b["status"] == abi.IN_POT
    d = np.sqrt((a["x"] - b["x"]) ** 2 + (a["y"] - b["y"]) ** 2 + (a["z"] - b["z"]) ** 2)[m]
    dv2 = ((a["vx"] - b["vx"]) ** 2 + (a["vy"] - b["vy"]) ** 2 + (a["vz"] - b["vz"]) ** 2)[m].sum()
    v2 = (b["vx"] ** 2 + b["vy"] ** 2 + b["vz"] ** 2)[m].sum()
    c = max(1, int(m.sum()))
    return {"rms": float(np.sqrt((d**2).sum() / c) / gpu.h), "max": float(d.max(initial=0) / gpu.h),
            "vel": float(np.sqrt(dv2 / v2) if v2 > 0 else np.sqrt(dv2 / c)), "mismatch": mism}


def test_construction_matches_oracle(engine, oracle_mod):
    for mm in (10, 5):
        cfg = abi.gentle_pour(mm, 20)
        gpu, cpu = engine.Simulation3D(cfg), oracle_mod.OracleSim(cfg)
        assert (gpu.n, gpu.nx, gpu.ny, gpu.nz) == (cpu.n, cpu.nx, cpu.ny, cpu.nz)
        assert np.array_equal(gpu.origin(), cpu.origin())
        a, b = gpu.particles(), cpu.particles()
        for k in ("x", "y", "z"):
            assert np.array_equal(a[k], b[k].astype(np.float32).astype(np.float64))
        gpu.destroy()


@pytest.mark.parametrize("mm", [10, 5])
def test_first_substep_fields(engine, oracle_mod, mm):
    cfg = abi.gentle_pour(mm, 20)
    gpu, cpu = lockstep(engine, oracle_mod, cfg, 1)
    assert np.array_equal(gpu.field(abi.FIELD_CELL), cpu.field(abi.FIELD_CELL))
    assert np.array_equal(gpu.field(abi.FIELD_VALID), cpu.field(abi.FIELD_VALID))
    for f in (abi.FIELD_VELOCITY_PREV, abi.FIELD_PRESSURE, abi.FIELD_VELOCITY):
        assert rel_l2(gpu.field(f), cpu.field(f)) < REL_FIELD, f
    assert rel_l2(gpu.field(abi.FIELD_CORRECTION), cpu.field(abi.FIELD_CORRECTION)) < 1e-4
    dg, dc = gpu.diagnostics(), cpu.diagnostics()
    assert dg["pressureIterations"] == dc["pressureIterations"]  # identical MIC(0) preconditioner
    assert dg["liquidCells"] == int((cpu.field(abi.FIELD_CELL) == abi.FLUID).sum())
    assert abs(dg["interiorDensity"] - dc["interiorDensity"]) < 1e-7
    gpu.destroy()


def test_step_comparison_10mm(engine, oracle_mod):
    # e2e/gpuSolver.spec.ts:23-42: compare(10 mm, 20 steps)
    cfg = abi.gentle_pour(10, 20)
    gpu, cpu = lockstep(engine, oracle_mod, cfg, 20)
    r = compare_particles(gpu, cpu)
    assert r["rms"] < 1e-3 and r["max"] < 1e-2, r
    assert r["vel"] < 1e-3, r
    assert r["mismatch"] == 0
    d = gpu.diagnostics()
    assert d["steps"] == 20 and d["pressureFailures"] == 0 and d["pressureIterations"] > 0 and d["lostMl"] == 0
    gpu.destroy()


def test_fields_from_identical_midpour_state(engine, oracle_mod):
    # an 8 mm steep-tilt state with liquid in the spout, then one substep on both from that state
    cfg = abi.gentle_pour(8, 1.6, pressure_max_iterations=300,
                          motion={"start_delay": 0.0, "tilt_duration": 0.4, "hold_angle_deg": 60.0,
                                  "max_angle_deg": 60.0, "max_hold": 5.0})
    cpu = oracle_mod.OracleSim(cfg)
    cpu.advance(0.7)
    st, parts = cpu.get_state(), cpu.particles()
    assert st.counts[abi.DISCHARGED] > 0  # pouring
    # the engine stores FP32 parcels: give both the same rounded state
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        parts[k] = parts[k].astype(np.float32).astype(np.float64)
    cpu.set_state(st, parts)
    gpu = engine.Simulation3D(cfg)
    gpu.set_state(st, parts)
    dt = cpu.stable_dt()
    cpu.step(dt)
    gpu.step(dt)
    assert np.array_equal(gpu.field(abi.FIELD_CELL), cpu.field(abi.FIELD_CELL))
    for f in (abi.FIELD_VELOCITY_PREV, abi.FIELD_PRESSURE, abi.FIELD_VELOCITY):
        assert rel_l2(gpu.field(f), cpu.field(f)) < REL_FIELD, f
    r = compare_particles(gpu, cpu)
    assert r["rms"] < 1e-4 and r["mismatch"] == 0, r
    dg, dc = gpu.diagnostics(), cpu.diagnostics()
    assert dg["dischargedMl"] == dc["dischargedMl"]
    assert np.allclose(gpu.discharged_fractions(), cpu.discharged_fractions(), atol=0, rtol=0)
    gpu.destroy()


def test_rest_is_stable(engine):
    # sim3d.test.ts:84-94 on the engine
    cfg = abi.gentle_pour(8, 0.3, pressure_max_iterations=300, motion={"kind": "still", "target_volume": 0.0})
    sim = engine.Simulation3D(cfg)
    d = sim.advance(0.3)
    assert abs(d["inPotMl"] - 1500) < 1e-6
    assert d["dischargedMl"] + d["spilledMl"] + d["lostMl"] == 0 and d["pressureFailures"] == 0
    assert sim.discharged_fractions() is None
    assert (sim.particles()["z"] >= np.float32(sim.h) * (1 - 1e-6)).all()
    sim.destroy()


def test_tilt_pours_and_chunking_is_bit_identical(engine):
    # sim3d.test.ts:96-123 on the engine: chunking 0.4 s vs 0.8 s gives identical parcels
    def cfg():
        return abi.gentle_pour(8, 1.6, pressure_max_iterations=300,
                               motion={"start_delay": 0.0, "tilt_duration": 0.4, "hold_angle_deg": 60.0,
                                       "max_angle_deg": 60.0, "max_hold": 5.0})

    a, b = engine.Simulation3D(cfg()), engine.Simulation3D(cfg())
    while not a.finished:
        a.advance(0.4)
    while not b.finished:
        b.advance(0.8)
    d = a.diagnostics()
    assert d["dischargedMl"] > 20 and d["lostMl"] == 0
    assert abs(d["inPotMl"] + d["dischargedMl"] + d["spilledMl"] + d["lostMl"] - 1500) < 1e-6
    assert abs(a.discharged_fractions().sum() - 1) < 1e-12
    pa, pb = a.particles(), b.particles()
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(pa[k], pb[k]), k
    poured = pa["status"] == abi.DISCHARGED
    assert pa["y"][poured].min() < a.pivot_world[1]
    a.destroy()
    b.destroy()


def test_step_vs_advance_and_enqueue_agree(engine):
    cfg = abi.gentle_pour(10, 20)
    a, b, c = engine.Simulation3D(cfg), engine.Simulation3D(cfg), engine.Simulation3D(cfg)
    for _ in range(30):
        a.step(-1.0)
    c.enqueue(30)
    c.sync()
    d = a.diagnostics()
    b.advance(d["time"] - 1e-9)
    assert b.diagnostics()["steps"] == 30
    for s in (b, c):
        assert s.diagnostics()["time"] == d["time"]
        assert np.array_equal(s.particles()["x"], a.particles()["x"])
    for s in (a, b, c):
        s.destroy()


def test_render_positions(engine):
    # writePositions (src/gpu3d/shaders.ts:786-799)
    sim = engine.Simulation3D(abi.gentle_pour(10, 20))
    sim.advance(0.05)
    p = sim.particles()
    r = sim.read_render_positions().reshape(2, sim.n, 3)
    y = np.where(p["y"].astype(np.float32) < np.float32(0.0005), -100.0, p["y"].astype(np.float32))
    assert np.array_equal(r[0, :, 0], p["x"].astype(np.float32)) and np.array_equal(r[0, :, 1], y)
    assert np.array_equal(r[1, :, 2], (np.float32(2 * sim.h) - p["z"].astype(np.float32)))
    sim.destroy()


def test_manual_tilt_target(engine, oracle_mod):
    # controller.setTarget (src/sim/motion.ts:40-44, 82-93) in manual mode, engine vs oracle
    cfg = abi.gentle_pour(10, 2.0, motion={"kind": "manual"})
    gpu, cpu = engine.Simulation3D(cfg), oracle_mod.OracleSim(cfg)
    gpu.set_target(35.0, 0.0)
    cpu.set_tilt_target(35.0, 0.0)
    for _ in range(40):
        dt = cpu.stable_dt()
        cpu.step(dt)
        gpu.step(dt)
    ag, ph = gpu.controller()
    assert ph == "manual"
    assert abs(ag - cpu.diagnostics()["angleDeg"]) < 1e-9
    assert 5 < ag < 35
    gpu.destroy()


def test_standalone_pcg_matches_oracle(engine, oracle_mod):
    import torch

    n = 8
    cell = np.zeros(n**3, np.uint8)
    for k in range(n):
        for j in range(n):
            for i in range(n):
                c = i + n * (j + n * k)
                border = i in (0, n - 1) or j in (0, n - 1) or k in (0, n - 1)
                cell[c] = 2 if border else (1 if j < 5 else 0)
    b = np.where(cell == 1, np.sin(np.arange(n**3)), 0.0)
    q0, it0, conv0, res0 = oracle_mod.pcg_solve(cell, b, n, n, n, 1e-8, 200)
    dc = torch.tensor(cell, device="cuda")
    db = torch.tensor(b, device="cuda")
    dq = torch.zeros(n**3, dtype=torch.float64, device="cuda")
    it, conv, res = engine.pcg_solve_device(dc.data_ptr(), db.data_ptr(), dq.data_ptr(), n, n, n, 1e-8, 200)
    assert conv and it == it0
    assert rel_l2(dq.cpu().numpy(), q0) < 1e-12
    it, conv, _ = engine.pcg_solve_device(dc.data_ptr(), torch.zeros_like(db).data_ptr(), dq.data_ptr(), n, n, n,
                                          1e-8, 10)
    assert it == 0 and conv
    _, conv, _ = engine.pcg_solve_device(dc.data_ptr(), db.data_ptr(), dq.data_ptr(), n, n, n, 1e-14, 1)
    assert not conv


def test_standalone_pcg_odd_sized_grid(engine, oracle_mod):
    # an odd cell count (9 x 7 x 5) places the solver's FP64 scratch after an odd number of ints
    import torch

    nx, ny, nz = 9, 7, 5
    rng = np.random.default_rng(3)
    cell = np.full(nx * ny * nz, 2, np.uint8)
    for k in range(1, nz - 1):
        for j in range(1, ny - 1):
            for i in range(1, nx - 1):
                cell[i + nx * (j + ny * k)] = 1 if j < 4 else 0
    b = np.where(cell == 1, rng.standard_normal(cell.size), 0.0)
    q0, it0, conv0, _ = oracle_mod.pcg_solve(cell, b, nx, ny, nz, 1e-10, 200)
    dc, db = torch.tensor(cell, device="cuda"), torch.tensor(b, device="cuda")
    dq = torch.zeros(cell.size, dtype=torch.float64, device="cuda")
    it, conv, _ = engine.pcg_solve_device(dc.data_ptr(), db.data_ptr(), dq.data_ptr(), nx, ny, nz, 1e-10, 200)
    assert conv and conv0 and it == it0
    assert rel_l2(dq.cpu().numpy(), q0) < 1e-12


@pytest.mark.slow
def test_whole_pour_5mm_against_reference(engine, goldens):
    # benchmarks/run3d.json 5 mm: 406.78 mL, shares 27.71 / 51.94 / 20.35 %, nothing spilled or lost
    ref = {r["cellMm"]: r for r in goldens["run3d"]}[5]
    sim = engine.Simulation3D(abi.gentle_pour(5, 20))
    done_at = -1.0
    while not sim.finished:  # benchmarks/run3d.ts:14-23
        d = sim.advance(0.5)
        if d["phase"] == "done" and done_at < 0:
            done_at = d["time"]
        if done_at >= 0 and d["time"] > done_at + 1.5:
            break
    d = sim.diagnostics()
    sh = sim.discharged_fractions()
    assert abs(d["dischargedMl"] / ref["dischargedMl"] - 1) < 0.003, d["dischargedMl"]
    assert np.abs(sh - np.array(ref["dischargedFractions"])).max() < 0.013, sh
    assert d["spilledMl"] == 0 and d["lostMl"] == 0 and d["pressureFailures"] == 0
    sim.destroy()
