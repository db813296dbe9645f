import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the engine's kernels)")
    config.addinivalue_line("markers", "slow: takes longer than a few seconds")


@pytest.fixture(scope="session")
def goldens():
    with open(os.path.join(GOLDEN, "reference_goldens.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def recording():
    """Early frames of the reference's 5 mm recording (every 3rd parcel, quantum 0.25 mm)."""
    d = np.load(os.path.join(GOLDEN, "pour3d_early.npz"))
    f0 = d["frame0"].astype(np.int64)
    frames = {0: f0}
    for k, idx in enumerate(d["frame_index"][1:]):
        frames[int(idx)] = f0 + d["deltas"][k].astype(np.int64)
    return {"origin": d["origin"], "frames": frames}


def quantize(x, y, z, keep, quantum=0.00025):
    """format.ts:64 on Float32 positions: max(0, min(65535, round(f / q)))."""
    q = np.stack([x[keep], y[keep], z[keep]], 1).reshape(-1).astype(np.float32).astype(np.float64)
    return np.clip(np.floor(q / quantum + 0.5), 0, 65535).astype(np.int64)


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def engine():
    import teapotfluidsimulation_b200 as pkg

    pkg.lib()
    return pkg
