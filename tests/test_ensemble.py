"""Ensembles of pours: the seeded configurations (host only) and, on the GPU, that pours run together on
their own streams give exactly what each gives alone."""
import numpy as np
import pytest

from teapotfluidsimulation_b200 import abi
from teapotfluidsimulation_b200 import engine as E


def test_configs_are_seeded_and_in_range():
    a = E.ensemble_configs(7, 16, 5.0, 20.0)
    b = E.ensemble_configs(7, 16, 5.0, 20.0)
    c = E.ensemble_configs(8, 16, 5.0, 20.0)
    fills = np.array([x.initial_volume for x in a]) / abi.ML / 1000
    peaks = np.array([x.motion.max_angle_deg for x in a])
    ramps = np.array([x.motion.tilt_duration for x in a])
    assert np.all((fills >= 0.6) & (fills < 1.0)) and np.all((peaks >= 60) & (peaks < 110))
    assert np.all((ramps >= 4) & (ramps < 12))
    assert [x.initial_volume for x in a] == [x.initial_volume for x in b]
    assert [x.initial_volume for x in a] != [x.initial_volume for x in c]
    assert len({x.seed for x in a}) == 16
    ref = abi.gentle_pour(5.0, 20.0)
    assert all(x.h == ref.h and x.motion.hold_angle_deg == ref.motion.hold_angle_deg for x in a)


def test_ensemble_grids_are_uneven():
    # the constructor's domain sweep follows each pour's fill and peak tilt (solver3d.ts:125-157)
    grids = set()
    for c in E.ensemble_configs(3, 8, 5.0, 20.0):
        s = E.plan(c)["sizes"]
        grids.add((s.nx, s.ny, s.nz))
    assert len(grids) > 1


@pytest.mark.gpu
def test_ensemble_members_match_single_runs(engine):
    cfgs = E.ensemble_configs(11, 4, 10.0, 20.0)
    for c in cfgs:
        c.preconditioner = abi.PRECOND_CHEB
    ens = E.Ensemble(cfgs)
    ens.advance(0.4)
    ens.enqueue(20)
    for i, c in enumerate(cfgs):
        alone = engine.Simulation3D(c)
        alone.advance(0.4)
        alone.enqueue(20)
        alone.sync()
        pa, pb = ens.members[i].particles(), alone.particles()
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.array_equal(pa[k], pb[k]), (i, k)
        assert ens.members[i].diagnostics()["time"] == alone.diagnostics()["time"]
        alone.destroy()
    ens.destroy()
