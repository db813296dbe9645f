"""The grid-scale pressure solves of the pour engine (PRECOND_BOX_MG, PRECOND_LEARNED): the liquid system
embedded in a dense power-of-two box and solved by the Poisson batch's multigrid PCG / learned flexible CG,
each solve a while-loop node of the substep's CUDA graph.

Fields are compared with the oracle (the reference's MIC(0)-PCG) at a tight tolerance, whole pours with
the reference's committed results, and the large full-domain APIC configuration runs substeps with no
pressure failure."""
import numpy as np
import pytest

from teapotfluidsimulation_b200 import abi

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def stepped(engine, oracle_mod, mm, precision, tol, net=None, precond=abi.PRECOND_BOX_MG):
    cfg = abi.gentle_pour(mm, 20, pressure_tolerance=tol)
    cpu = oracle_mod.OracleSim(cfg)
    cfg.preconditioner = precond
    cfg.solve_precision = precision
    gpu = engine.Simulation3D(cfg)
    if net is not None:
        gpu.set_unet(net)
    for _ in range(2):
        dt = cpu.stable_dt()
        cpu.step(dt)
        gpu.step(dt)
    return gpu, cpu


@pytest.mark.parametrize("precision", [abi.SOLVE_F64, abi.SOLVE_MIXED])
@pytest.mark.parametrize("mm", [5, 4])
def test_fields_match_oracle(engine, oracle_mod, mm, precision):
    # the box operator is the liquid list's operator; the right-hand side enters the box in FP32, so
    # the pressure agrees to the rounding of b (about 1e-7) however tight the tolerance
    gpu, cpu = stepped(engine, oracle_mod, mm, precision, 1e-10)
    assert np.array_equal(gpu.field(abi.FIELD_CELL), cpu.field(abi.FIELD_CELL))
    for f in (abi.FIELD_PRESSURE, abi.FIELD_VELOCITY, abi.FIELD_VELOCITY_PREV):
        assert rel_l2(gpu.field(f), cpu.field(f)) < 1e-5, f
    d = gpu.diagnostics()
    assert d["pressureFailures"] == 0 and d["pressureIterations"] > 0
    assert d["pressureIterations"] < cpu.diagnostics()["pressureIterations"]
    gpu.destroy()


def test_learned_in_the_engine_with_an_untrained_network(engine, oracle_mod):
    # an untrained network stalls at once; the multigrid fall-back still ends every solve on the
    # reference's stopping rule, so the fields agree with the oracle within the solve tolerance
    net = engine.engine.UNet(seed=4)
    gpu, cpu = stepped(engine, oracle_mod, 10, abi.SOLVE_MIXED, 1e-6, net=net, precond=abi.PRECOND_LEARNED)
    assert rel_l2(gpu.field(abi.FIELD_PRESSURE), cpu.field(abi.FIELD_PRESSURE)) < 1e-4
    assert rel_l2(gpu.field(abi.FIELD_VELOCITY), cpu.field(abi.FIELD_VELOCITY)) < 1e-5
    assert gpu.diagnostics()["pressureFailures"] == 0
    gpu.destroy()


def test_learned_needs_a_network(engine):
    cfg = abi.gentle_pour(10, 20)
    cfg.preconditioner = abi.PRECOND_LEARNED
    cfg.solve_precision = abi.SOLVE_MIXED
    sim = engine.Simulation3D(cfg)
    with pytest.raises(engine.EngineError):
        sim.step(-1.0)
    sim.destroy()
    cfg.solve_precision = abi.SOLVE_F64
    with pytest.raises(engine.EngineError):
        engine.Simulation3D(cfg)


@pytest.mark.slow
def test_whole_pour_5mm_against_reference(engine, goldens):
    ref = {r["cellMm"]: r for r in goldens["run3d"]}[5]
    cfg = abi.gentle_pour(5, 20)
    cfg.preconditioner = abi.PRECOND_BOX_MG
    cfg.solve_precision = abi.SOLVE_MIXED
    sim = engine.Simulation3D(cfg)
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


def test_full_domain_apic_2_5mm_runs(engine):
    # the large configuration: both halves of the pot at 2.5 mm with APIC (about 126 x 126 x 64 cells and
    # 700k parcels), beyond the cluster solves; every pressure solve converges and the projected
    # velocity is divergence-free to the solve tolerance
    cfg = abi.gentle_pour(2.5, 20, domain=abi.DOMAIN_FULL, transfer=abi.TRANSFER_APIC)
    cfg.preconditioner = abi.PRECOND_BOX_MG
    cfg.solve_precision = abi.SOLVE_MIXED
    sim = engine.Simulation3D(cfg)
    assert sim.n > 600_000 and sim.nz >= 60
    for _ in range(20):
        sim.step(-1.0)
    d = sim.diagnostics()
    assert d["pressureFailures"] == 0 and d["pressureIterations"] > 0
    assert d["liquidCells"] > 65_536  # beyond what the 16-CTA cluster solves hold
    assert d["lostMl"] == 0 and d["spilledMl"] == 0
    assert 0 <= d["maxDivergence"] < 1e-2
    sim.destroy()
