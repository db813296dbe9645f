"""Full-domain mode: both halves of the pot instead of the reference's half pot behind the symmetry plane
(solver3d.ts:9-10, 157, 756-760). No reference counterpart: the seeded half is the reference's own
construction, the other half its mirror image, and parity is pinned by mirror symmetry and by the engine
agreeing with the oracle extended the same way."""
import numpy as np
import pytest

from teapotfluidsimulation_b200 import abi


def test_construction_is_the_seeded_half_plus_its_mirror(engine, oracle_mod):
    half = engine.engine.plan(abi.gentle_pour(10, 1.0))
    full = engine.engine.plan(abi.gentle_pour(10, 1.0, domain=abi.DOMAIN_FULL))
    n, N = half["sizes"].n, full["sizes"].n
    assert N == 2 * n and full["sizes"].nz == 2 * half["sizes"].nz - 2
    assert (full["sizes"].nx, full["sizes"].ny) == (half["sizes"].nx, half["sizes"].ny)
    h = half["sizes"].h
    zoff = (half["sizes"].nz - 1) * h
    assert np.array_equal(full["x"][:n], half["x"]) and np.array_equal(full["y"][:n], half["y"])
    assert np.allclose(full["z"][:n] - zoff, half["z"] - h, rtol=0, atol=1e-15)
    assert np.array_equal(full["x"][n:], full["x"][:n]) and np.array_equal(full["y"][n:], full["y"][:n])
    assert np.allclose(full["z"][n:] - zoff, -(full["z"][:n] - zoff), rtol=0, atol=1e-15)
    assert np.array_equal(full["origin"][:n], half["origin"]) and np.array_equal(full["origin"][n:], half["origin"])
    assert list(full["sizes"].band_counts) == [2 * b for b in half["sizes"].band_counts]
    assert full["sizes"].parcel_volume == half["sizes"].parcel_volume
    # the oracle builds the same parcels
    o = oracle_mod.OracleSim(abi.gentle_pour(10, 1.0, domain=abi.DOMAIN_FULL))
    po = o.particles()
    assert np.array_equal(po["x"], full["x"]) and np.array_equal(po["z"], full["z"])
    assert np.array_equal(o.origin(), full["origin"])


def test_oracle_full_domain_stays_mirror_symmetric(oracle_mod):
    # the discretisation is symmetric about the plane; the iterative solves are not (the MIC(0) factor
    # sweeps in index order), so they run to 1e-13 and without the 1e-4 density-correction solve
    cfg = abi.gentle_pour(10, 0.5, domain=abi.DOMAIN_FULL, pressure_tolerance=1e-13, pressure_max_iterations=2000,
                          density_correction=0.0)
    sim = oracle_mod.OracleSim(cfg)
    d = sim.advance(0.12)
    assert d["lostMl"] == 0 and abs(d["inPotMl"] - 1500) < 1e-6 * 1500  # both halves counted once
    p = sim.particles()
    n = sim.n // 2
    zoff = sim.sizes.nz // 2 * sim.h  # (nz_half - 1) h with nz = 2 nz_half - 2
    assert np.abs(p["x"][n:] - p["x"][:n]).max() < 1e-12
    assert np.abs((p["z"][n:] - zoff) + (p["z"][:n] - zoff)).max() < 1e-12
    assert np.abs(p["vz"][n:] + p["vz"][:n]).max() < 1e-10


@pytest.mark.gpu
def test_engine_full_domain_follows_the_oracle(engine, oracle_mod):
    cfg = abi.gentle_pour(10, 1.0, domain=abi.DOMAIN_FULL)
    gpu = engine.Simulation3D(cfg)
    cpu = oracle_mod.OracleSim(cfg)
    for _ in range(2):
        dt = cpu.stable_dt()
        cpu.step(dt)
        gpu.step(dt)
    assert np.array_equal(gpu.field(abi.FIELD_CELL), cpu.field(abi.FIELD_CELL))
    for f in (abi.FIELD_VELOCITY, abi.FIELD_PRESSURE):
        a, b = gpu.field(f), cpu.field(f)
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), f
    pa, pb = gpu.particles(), cpu.particles()
    rms = np.sqrt(((pa["x"] - pb["x"]) ** 2 + (pa["y"] - pb["y"]) ** 2 + (pa["z"] - pb["z"]) ** 2).mean()) / gpu.h
    assert rms < 1e-4
    gd, cd = gpu.diagnostics(), cpu.diagnostics()
    assert abs(gd["inPotMl"] - cd["inPotMl"]) < 1e-9
    r = gpu.read_render_positions()
    assert r.size == 3 * gpu.n
    gpu.destroy()
