"""The CPU oracle against the reference's own goldens and unit tests (no GPU).

Pins: benchmarks/run3d.json (parcel counts, grids), public/data/pour3d.bin.gz (pivotWorld, domain,
origin tags, the first 1.9 s of positions), benchmarks/gpu3d.json (the CPU state after 200
substeps), and the known answers of tests/sim3d.test.ts.
"""
import math

import numpy as np
import pytest

from teapotfluidsimulation_b200 import abi
from conftest import quantize


def test_rng_mulberry32(oracle_mod):
    # rng.ts:5-14: values are k / 2^32 in [0, 1), deterministic per seed
    a = oracle_mod.rng(1, 1000)
    b = oracle_mod.rng(1, 1000)
    assert np.array_equal(a, b)
    assert (a >= 0).all() and (a < 1).all()
    assert np.array_equal(a * 2**32, np.floor(a * 2**32))
    assert not np.array_equal(a, oracle_mod.rng(2, 1000))


def test_js_hypot():
    from oracle import oracle as O

    assert O.js_hypot3(3.0, 4.0, 0.0) == 5.0
    assert O.js_hypot3(0.0, 0.0, 0.0) == 0.0
    for v in [(1e-3, 2e-3, 3e-3), (0.1, 0.2, 0.3), (66.0, 66.0, 0.0)]:
        assert abs(O.js_hypot3(*v) - math.hypot(*v)) <= 2e-16 * math.hypot(*v)


def test_geometry_signs(oracle_mod):
    # sim3d.test.ts:28-58
    t = abi.default_teapot()
    sdf, cav = oracle_mod.teapot_sdf, oracle_mod.in_cavity
    assert sdf(0, 0.05, 0) > 0.03
    assert sdf(-(t.radius + t.wall / 2), 0.08, 0) < 0
    assert sdf(0, -t.wall / 2, 0) < 0
    assert sdf(0, t.height + 0.02, 0) > 0
    assert cav(0, 0.05, 0) and not cav(0, -0.01, 0)
    a = math.radians(t.spout_angle_deg)
    ax, ay, dx, dy = t.radius - t.wall, t.inlet_height, math.cos(a), math.sin(a)
    s = 0.0
    while s < t.spout_length - 0.005:
        assert sdf(ax + s * dx, ay + s * dy, 0) > 0
        assert cav(ax + s * dx, ay + s * dy, 0)
        s += 0.01
    s, off = 0.08, t.bore_radius + t.wall / 2
    assert sdf(ax + s * dx - dy * off, ay + s * dy + dx * off, 0) < 0
    assert sdf(t.radius + t.wall / 2, 0.11, 0) < 0
    tip_y = ay + dy * t.spout_length
    assert tip_y - t.bore_radius > 1.5e-3 / (math.pi * t.radius**2)


def column(n=8):
    cell = np.zeros(n * n * n, np.uint8)
    for k in range(n):
        for j in range(n):
            for i in range(n):
                c = i + n * (j + n * k)
                border = i == 0 or j == 0 or k == 0 or i == n - 1 or j == n - 1 or k == n - 1
                cell[c] = 2 if border else (1 if j < 5 else 0)
    b = np.where(cell == 1, np.sin(np.arange(n**3)), 0.0)
    return cell, b


def test_pcg_column(oracle_mod):
    # sim3d.test.ts:60-81
    n = 8
    cell, b = column(n)
    q, it, conv, res = oracle_mod.pcg_solve(cell, b, n, n, n, 1e-8, 200)
    assert conv and it < 40
    _, it0, conv0, _ = oracle_mod.pcg_solve(cell, np.zeros(n**3), n, n, n, 1e-8, 10)
    assert it0 == 0 and conv0
    _, _, conv1, _ = oracle_mod.pcg_solve(cell, b, n, n, n, 1e-14, 1)
    assert not conv1


def test_construction_goldens(oracle_mod, goldens, recording):
    # run3d.json:7-12, 27-33 and the recording header (scripts/record3d.ts:212-229)
    rows = {r["cellMm"]: r for r in goldens["run3d"]}
    for mm in (5, 4):
        s = oracle_mod.OracleSim(abi.gentle_pour(mm, 20))
        assert s.n == rows[mm]["parcelsHalfPot"]
        assert [s.nx, s.ny, s.nz] == rows[mm]["grid"]
        bc = list(s.sizes.band_counts)
        assert max(bc) - min(bc) <= 1  # sim3d.test.ts:87
        if mm == 5:
            rec = goldens["recording"]
            assert list(s.sizes.pivot_world) == rec["pivotWorld"]  # bit-exact
            assert [s.nx * s.h, s.ny * s.h, s.nz * s.h] == rec["domain"]
            keep = np.arange(0, s.n, 3)
            assert np.array_equal(s.origin()[keep], recording["origin"])  # origin tags bit-exact
            p = s.particles()
            assert np.array_equal(quantize(p["x"], p["y"], p["z"], keep), recording["frames"][0])


@pytest.mark.slow
def test_state_after_200_substeps(oracle_mod, goldens):
    # benchmarks/gpu3d.json stepComparison.cpu: the CPU solver after 200 substeps at 5 mm
    g = goldens["state200"]
    s = oracle_mod.OracleSim(abi.gentle_pour(5, 20))
    for _ in range(200):
        s.step(-1.0)
    d = s.diagnostics()
    assert d["steps"] == g["steps"]
    assert d["time"] == g["time"]
    assert d["angleDeg"] == g["angleDeg"]
    assert d["pressureIterations"] == g["pressureIterations"]
    assert d["maxDivergence"] == g["maxDivergence"]
    assert d["interiorDensity"] == g["interiorDensity"]
    assert d["inPotMl"] == g["inPotMl"] and d["dischargedMl"] == 0


@pytest.mark.slow
def test_recorded_trajectory_first_seconds(oracle_mod, goldens, recording):
    # The recording's positions (10 fps, every 3rd parcel) are reproduced exactly over the first
    # 1.9 s, as are the controller angles; later frames diverge chaotically from a last-bit
    # difference between the JavaScript and C cos().
    s = oracle_mod.OracleSim(abi.gentle_pour(5, 14))
    keep = np.arange(0, s.n, 3)
    angles = goldens["recording_angles"]
    for k in range(1, 20):
        s.advance(0.1)
        d = s.diagnostics()
        if k < 10:  # exact until the first last-bit cos() difference (t = 1.0 s)
            assert d["angleDeg"] == angles[k]
        else:
            assert abs(d["angleDeg"] - angles[k]) <= 1e-8 * abs(angles[k])
        if k in recording["frames"]:
            p = s.particles()
            assert np.array_equal(quantize(p["x"], p["y"], p["z"], keep), recording["frames"][k]), f"frame {k}"


@pytest.mark.slow
def test_rest_and_layers(oracle_mod):
    # sim3d.test.ts:84-94 at 8 mm, 0.3 s, still pot
    cfg = abi.gentle_pour(8, 0.3, pressure_max_iterations=300, motion={"kind": "still", "target_volume": 0.0})
    s = oracle_mod.OracleSim(cfg)
    d = s.advance(0.3)
    assert abs(d["inPotMl"] - 1500) < 1e-6
    assert d["dischargedMl"] + d["spilledMl"] + d["lostMl"] == 0
    assert d["pressureFailures"] == 0
    assert s.discharged_fractions() is None
    assert (s.particles()["z"] >= s.h).all()


def tilt_cfg():
    return abi.gentle_pour(8, 1.6, pressure_max_iterations=300,
                           motion={"start_delay": 0.0, "tilt_duration": 0.4, "hold_angle_deg": 60.0,
                                   "max_angle_deg": 60.0, "max_hold": 5.0})


@pytest.mark.slow
def test_tilt_pours_deterministically(oracle_mod):
    # sim3d.test.ts:96-123
    a = oracle_mod.OracleSim(tilt_cfg())
    b = oracle_mod.OracleSim(tilt_cfg())
    while not a.finished:
        a.advance(0.4)
    while not b.finished:
        b.advance(0.8)
    d = a.diagnostics()
    assert d["dischargedMl"] > 20 and d["lostMl"] == 0
    assert abs(d["inPotMl"] + d["dischargedMl"] + d["spilledMl"] + d["lostMl"] - 1500) < 1e-6
    assert abs(a.discharged_fractions().sum() - 1) < 1e-12
    pa = a.particles()
    order = a.discharge_order()
    assert (pa["status"][order] == abi.DISCHARGED).all()
    assert pa["y"][order].min() < a.sizes.pivot_world[1]
    assert np.array_equal(pa["x"], b.particles()["x"])
    assert (pa["status"] == abi.IN_POT).any()
