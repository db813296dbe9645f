"""Failure handling and checkpoint/resume through the C ABI (needs a GPU).

Every failure here is made on the host or by a bounded device wait running out; nothing faults,
traps or hangs the GPU:
  - a parcel whose position is NaN becomes LOST in the same substep and its volume is reported as
    lost, as the reference's advect does (solver3d.ts:761-764); the rest of the substep agrees with
    the oracle fed the same state;
  - an iteration cap the pressure solve cannot meet counts a pressure failure every substep while the
    run goes on (solver3d.ts:540);
  - a device allocation that fails (injected on the host) makes pl_create return PL_E_NOMEM and leaves
    nothing behind; a bad device ordinal returns PL_E_CUDA;
  - the binning scan's look-back wait, given a poll limit of 1, gives up: the call returns
    PL_E_TIMEOUT, the parcels keep their state, and the device stays usable;
  - a state saved mid-pour and restored into a fresh handle continues bit for bit like the
    uninterrupted run (the reference's determinism: results independent of chunking,
    solver3d.ts:280-286, tests/sim3d.test.ts:111-121).
"""
import numpy as np
import pytest

from teapotfluidsimulation_b200 import abi

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def midpour(engine, mm, seconds, **over):
    cfg = abi.gentle_pour(mm, 20, **over)
    cfg.preconditioner, cfg.solve_precision = abi.PRECOND_CHEB, abi.SOLVE_MIXED
    sim = engine.Simulation3D(cfg)
    sim.advance(seconds)
    return cfg, sim


def test_nan_parcel_becomes_lost(engine, oracle_mod):
    cfg, sim = midpour(engine, 8, 0.4)
    st, parts = sim.get_state(), sim.particles()
    sim.destroy()
    inpot = np.flatnonzero(parts["status"] == abi.IN_POT)
    bad = int(inpot[len(inpot) // 2])
    parts["x"][bad] = np.nan
    ocfg = abi.gentle_pour(8, 20)
    cpu = oracle_mod.OracleSim(ocfg)
    cpu.set_state(st, parts)
    gpu = engine.Simulation3D(ocfg)
    gpu.set_state(st, parts)
    dt = cpu.stable_dt()
    cpu.step(dt)
    gpu.step(dt)
    a, b = gpu.particles(), cpu.particles()
    assert a["status"][bad] == abi.LOST and b["status"][bad] == abi.LOST
    dg, dc = gpu.diagnostics(), cpu.diagnostics()
    assert dc["lostMl"] > 0 and abs(dg["lostMl"] / dc["lostMl"] - 1) < 1e-12
    assert abs(dg["lostMl"] / (gpu.sizes.parcel_volume * 2 * 1e6) - 1) < 1e-12  # one parcel
    assert np.array_equal(a["status"], b["status"])
    ok = np.arange(gpu.n) != bad
    assert np.isfinite(a["x"][ok]).all() and np.isfinite(a["vx"][ok]).all()
    assert np.array_equal(gpu.field(abi.FIELD_CELL), cpu.field(abi.FIELD_CELL))
    assert rel_l2(gpu.field(abi.FIELD_VELOCITY), cpu.field(abi.FIELD_VELOCITY)) < 1e-5
    # the run goes on with the parcel out of the liquid
    gpu.advance(0.1)
    d = gpu.diagnostics()
    assert d["lostMl"] == dg["lostMl"] and d["pressureFailures"] == 0
    gpu.destroy()


@pytest.mark.parametrize("precond,precision", [(abi.PRECOND_MIC0, abi.SOLVE_F64),
                                               (abi.PRECOND_CHEB, abi.SOLVE_MIXED)])
def test_iteration_cap_counts_failures_and_the_run_continues(engine, oracle_mod, precond, precision):
    cfg = abi.gentle_pour(10, 20, pressure_max_iterations=1)
    cpu = oracle_mod.OracleSim(cfg)
    cfg.preconditioner, cfg.solve_precision = precond, precision
    gpu = engine.Simulation3D(cfg)
    for _ in range(5):
        dt = cpu.stable_dt()
        cpu.step(dt)
        gpu.step(dt)
    dg, dc = gpu.diagnostics(), cpu.diagnostics()
    assert dc["pressureFailures"] == 5 and dg["pressureFailures"] == 5
    assert dg["steps"] == 5 and dg["time"] == dc["time"]
    assert np.isfinite(gpu.particles()["x"]).all()
    gpu.destroy()


def test_allocation_failure_returns_nomem(engine):
    cfg = abi.gentle_pour(10, 1)
    engine.engine.inject_fault(engine.engine.FAULT_ALLOC, 1)
    with pytest.raises(engine.EngineError) as e:
        engine.Simulation3D(cfg)
    assert e.value.code == -5 and "cudaMalloc" in str(e.value)  # PL_E_NOMEM
    sim = engine.Simulation3D(cfg)  # the injection is used up; creation works again
    sim.step(-1.0)
    assert sim.diagnostics()["steps"] == 1
    sim.destroy()
    bad = abi.gentle_pour(10, 1)
    bad.device = 4096
    with pytest.raises(engine.EngineError) as e:
        engine.Simulation3D(bad)
    assert e.value.code == -2  # PL_E_CUDA: invalid device ordinal


def test_scan_wait_gives_up_with_timeout(engine):
    cfg = abi.gentle_pour(4, 20)
    cfg.preconditioner, cfg.solve_precision = abi.PRECOND_CHEB, abi.SOLVE_MIXED
    sim = engine.Simulation3D(cfg)
    sim.step(-1.0)
    before = sim.particles()
    sim.set_wait_limit(1)
    code = None
    for _ in range(20):
        try:
            sim.step(-1.0)
            before = sim.particles()
        except engine.EngineError as e:
            code = e.code
            assert "bin scan wait gave up" in str(e)
            break
    assert code == -3  # PL_E_TIMEOUT
    after = sim.particles()  # a plain read of the parcel buffers (no scalar synchronisation)
    for k in ("x", "y", "z", "vx", "vy", "vz", "status"):
        assert np.array_equal(before[k], after[k]), k
    sim.destroy()
    probe = engine.Simulation3D(cfg)  # the device is still usable
    probe.step(-1.0)
    assert probe.diagnostics()["steps"] == 1 and np.isfinite(probe.particles()["x"]).all()
    probe.destroy()


@pytest.mark.parametrize("mm,over", [(5, {}), (8, {"transfer": abi.TRANSFER_APIC})])
def test_checkpoint_resume_is_bit_identical(engine, mm, over):
    cfg, a = midpour(engine, mm, 3.0, **over)
    st, parts = a.get_state(), a.particles()
    aff = a.affine() if over.get("transfer") == abi.TRANSFER_APIC else None
    a.advance(1.0)
    b = engine.Simulation3D(cfg)
    b.set_state(st, parts)
    if aff is not None:
        b.set_affine(aff)
    b.advance(1.0)
    da, db = a.diagnostics(), b.diagnostics()
    for k in ("time", "steps", "angleDeg", "phase", "dischargedMl", "spilledMl", "lostMl", "inPotMl",
              "pressureFailures"):
        assert da[k] == db[k], (k, da[k], db[k])
    pa, pb = a.particles(), b.particles()
    for k in ("x", "y", "z", "vx", "vy", "vz", "status"):
        assert np.array_equal(pa[k], pb[k]), k
    if aff is not None:
        assert np.array_equal(a.affine(), b.affine())
    fa, fb = a.discharged_fractions(), b.discharged_fractions()
    assert (fa is None and fb is None) or np.array_equal(fa, fb)
    a.destroy()
    b.destroy()
