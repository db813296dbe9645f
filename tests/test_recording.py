"""The recording writer: the reference's playback format (src/view3d/format.ts) byte for byte, pinned
against the first 202,526 bytes of the reference's own 5 mm recording (public/data/pour3d.bin.gz:
header, origin tags, frame 0 and the frame-1 deltas), and on the GPU a short engine recording whose
device-quantised frames equal the host quantisation of the same parcels."""
import hashlib
import json
import os

import numpy as np
import pytest

from teapotfluidsimulation_b200 import recording as R

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_js_numbers():
    # ECMAScript Number::toString cases the header holds (and its edges)
    cases = {0.0: "0", -0.0: "0", 5.0: "5", 0.06: "0.06", 0.00025: "0.00025", 7.503631454386371e-05:
             "0.00007503631454386371", 1e-7: "1e-7", 1.5e-7: "1.5e-7", 123456789012345680000.0:
             "123456789012345680000", 1e21: "1e+21", 2.5e22: "2.5e+22", -0.14185: "-0.14185",
             0.11475045349225214: "0.11475045349225214", 44958: "44958", 1e-6: "0.000001"}
    for x, want in cases.items():
        assert R.js_number(x) == want, (x, R.js_number(x), want)
    assert R.js_stringify({"a": [1.0, 0.5], "b": "x\"y", "c": None, "d": True}) == '{"a":[1,0.5],"b":"x\\"y","c":null,"d":true}'


def test_header_serialises_as_the_reference_wrote_it():
    pin = json.load(open(os.path.join(GOLDEN, "recording_pin.json")))
    header = json.loads(pin["header_json"])
    assert R.js_stringify(header) == pin["header_json"]


def test_writer_reproduces_the_reference_recording_prefix(recording):
    pin = json.load(open(os.path.join(GOLDEN, "recording_pin.json")))
    header = json.loads(pin["header_json"])
    d = np.load(os.path.join(GOLDEN, "pour3d_early.npz"))
    f0 = d["frame0"].astype(np.int64)
    f1 = f0 + d["frame1_delta"].astype(np.int64)
    q = header["quantum"]
    # through Float32 metres, as the reference's frames are: the quantisation gives back the integers
    frames = [(f0 * q).astype(np.float32), (f1 * q).astype(np.float32)]
    raw = R.encode_recording(header, d["origin"], frames)
    assert len(raw) == pin["prefix_bytes"]
    assert hashlib.sha256(raw).hexdigest() == pin["prefix_sha256"]


def test_round_trip_and_delta_clamp():
    rng = np.random.default_rng(3)
    P = 50
    base = rng.uniform(1, 15, 3 * P)
    f = [(base + rng.normal(0, 0.01, 3 * P) * k).astype(np.float32) for k in range(4)]
    f[1][0] = 0.0
    f[2][0] = 15.9  # a jump from 0 larger than an int16 delta (63,600 quanta)
    h = {"version": 1, "frames": 4, "parcels": P, "fps": 10, "quantum": 0.00025}
    hd, origin, pos = R.decode_recording(R.encode_recording(h, np.arange(P) % 3, f))
    assert hd == h and np.array_equal(origin, np.arange(P) % 3)
    for k in range(4):
        got, want = R.quantize(pos[k], 0.00025), R.quantize(f[k], 0.00025)
        assert np.array_equal(got[1:], want[1:]), k
    # the clamped delta is what the decoder reconstructs: the jump is cut to +32767 quanta, and the
    # next delta starts from there
    assert R.quantize(pos[2], 0.00025)[0] == 32767
    assert R.quantize(pos[3], 0.00025)[0] == R.quantize(f[3], 0.00025)[0]
    # Math.round halves go up; out-of-range positions clamp
    assert list(R.quantize(np.array([0.000125, -1.0, 20.0], np.float32), 0.00025)) == [1, 0, 65535]


@pytest.mark.gpu
def test_engine_recording_matches_host_quantisation(engine):
    from teapotfluidsimulation_b200 import abi

    cfg = abi.gentle_pour(10, 20)
    cfg.preconditioner = abi.PRECOND_CHEB
    sim = engine.Simulation3D(cfg)
    sim.advance(0.3)
    dev = sim.quantized_positions(3, 0.00025)
    p = sim.particles()
    host = np.stack([p["x"], p["y"], p["z"]], 1)[::3].reshape(-1)
    assert np.array_equal(dev, R.quantize(host, 0.00025))
    raw = R.record_pour(sim, stride=3, fps=10, max_seconds=0.5)
    h, origin, pos = R.decode_recording(raw)
    assert h["frames"] == 6 and h["parcels"] == (sim.n + 2) // 3 and h["simulatedParcels"] == sim.n
    assert np.array_equal(origin, sim.origin()[::3])
    p = sim.particles()
    last = np.stack([p["x"], p["y"], p["z"]], 1)[::3].reshape(-1)
    assert np.array_equal(R.quantize(pos[-1], 0.00025), R.quantize(last, 0.00025))
    assert len(h["angles"]) == 6 and len(h["poured"]) == 6
    sim.destroy()
