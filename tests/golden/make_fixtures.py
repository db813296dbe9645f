"""Extract the golden vectors the tests pin the oracle and the engine against.

Usage: python tests/golden/make_fixtures.py <reference checkout>

Reads the reference's committed results from the given checkout:
  benchmarks/run3d.json      whole-pour results of the CPU solver at 5 and 4 mm
  benchmarks/gpu3d.json      the CPU state after 200 substeps at 5 mm (stepComparison.cpu)
  public/data/pour3d.bin.gz  the 5 mm recording (format: src/view3d/format.ts:4-8): origin tags
                             of every 3rd parcel and 10 fps frames of their positions
and writes tests/golden/reference_goldens.json, tests/golden/pour3d_early.npz and
tests/golden/recording_pin.json.
"""
import gzip
import json
import os
import struct
import sys

import numpy as np

OUT = os.path.dirname(os.path.abspath(__file__))
FRAMES = [0, 2, 5, 9, 14, 19]  # within the first 1.9 s (the recording is 10 fps)


def main():
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: make_fixtures.py <path of the reference checkout>")
    ref = sys.argv[1]
    run3d = json.load(open(os.path.join(ref, "benchmarks/run3d.json")))
    gpu3d = json.load(open(os.path.join(ref, "benchmarks/gpu3d.json")))
    raw = gzip.open(os.path.join(ref, "public/data/pour3d.bin.gz")).read()
    hl = struct.unpack("<I", raw[:4])[0]
    head = json.loads(raw[4:4 + hl])
    P = head["parcels"]
    o = 4 + hl
    origin = np.frombuffer(raw[o:o + P], np.uint8).copy()
    o += P
    cur = np.frombuffer(raw[o:o + 6 * P], "<u2").astype(np.int64)
    o += 6 * P
    frames = [cur.copy()]
    for _ in range(1, head["frames"]):
        d = np.frombuffer(raw[o:o + 6 * P], "<i2").astype(np.int64)
        o += 6 * P
        cur = cur + d
        frames.append(cur.copy())
    f0 = frames[0].astype(np.uint16)
    # the first bytes of the file exactly (header, origin tags, frame 0, the frame 1 deltas): pins the
    # recording writer byte for byte; frame 1 itself goes into the npz
    import hashlib

    pre = 4 + hl + P + 2 * 6 * P
    pin = {"header_json": raw[4:4 + hl].decode("utf-8"), "prefix_bytes": pre,
           "prefix_sha256": hashlib.sha256(raw[:pre]).hexdigest()}
    with open(os.path.join(OUT, "recording_pin.json"), "w") as f:
        json.dump(pin, f, indent=1)
    deltas = np.stack([frames[k] - frames[0] for k in FRAMES[1:]]).astype(np.int16)
    np.savez_compressed(os.path.join(OUT, "pour3d_early.npz"), origin=origin, frame0=f0, deltas=deltas,
                        frame_index=np.array(FRAMES), frame1_delta=(frames[1] - frames[0]).astype(np.int16))
    gold = {
        "source": "marcelpetrick/teapotFluidSimulation benchmarks/run3d.json, benchmarks/gpu3d.json, "
                  "public/data/pour3d.bin.gz",
        "run3d": run3d["rows"],
        "state200": gpu3d["stepComparison"]["cpu"],
        "gpu_rows": [{k: r[k] for k in ("cellMm", "simulatedSeconds", "steps", "dischargedMl", "dischargedFractions",
                                         "maxPressureIterations", "wallSeconds", "realTimeFactor")}
                     for r in gpu3d["rows"]],
        "step_comparison_gpu": {k: gpu3d["stepComparison"][k] for k in
                                ("steps", "rmsPositionCells", "maxPositionCells", "relativeVelocityRms",
                                 "statusMismatches")},
        "recording": {k: head[k] for k in ("frames", "parcels", "fps", "quantum", "cellMm", "simulatedParcels",
                                            "pivot", "pivotWorld", "zOffset", "domain", "finalShares")},
        "recording_angles": head["angles"],
        "recording_poured": head["poured"],
    }
    with open(os.path.join(OUT, "reference_goldens.json"), "w") as f:
        json.dump(gold, f, indent=1)


if __name__ == "__main__":
    main()
