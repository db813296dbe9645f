"""Recordings of a pour in the reference's playback format (`pour3d.bin.gz`), written from the engine.

Format (src/view3d/format.ts:4-8, little endian): u32 header length | header JSON (UTF-8) |
u8 origin[P] | u16 frame0[3P] | i16 delta[F-1][3P]. Positions are quantised to `quantum` metres and
stored as deltas to the previous frame, clamped to int16 with the decoder kept in step
(format.ts:47-77). The header is serialised as JavaScript's `JSON.stringify` does it
(shortest round-trip numbers in ECMAScript's notation, no spaces), so a recording made here is byte
for byte what `encodeRecording` makes of the same frames, and the reference's browser viewer plays it.

`record_pour` follows scripts/record3d.ts: every `stride`-th parcel in id order, `fps` frames per
simulated second, until 1.5 s after the controller is done. The positions are quantised on the device
(`pl_read_quantized_positions`), so a frame crosses PCIe as 6 bytes per kept parcel.
"""
from __future__ import annotations

import decimal
import gzip
import json
import math
import struct

import numpy as np

MAX_U16 = 65535


# ------------------------------------------------------------------ JSON as JavaScript writes it

def js_number(x: float) -> str:
    """ECMAScript Number::toString(10) of a finite double, as JSON.stringify writes it (NaN and the
    infinities become null)."""
    if isinstance(x, bool):
        return "true" if x else "false"
    x = float(x)
    if math.isnan(x) or math.isinf(x):
        return "null"
    if x == 0:
        return "0"
    sign = "-" if x < 0 else ""
    d = decimal.Decimal(repr(abs(x))).normalize()  # repr: the shortest digits that round-trip
    t = d.as_tuple()
    digits = "".join(str(v) for v in t.digits)
    k = len(digits)
    n = t.exponent + k  # x = 0.digits * 10^n
    if k <= n <= 21:
        body = digits + "0" * (n - k)
    elif 0 < n <= 21:
        body = digits[:n] + "." + digits[n:]
    elif -6 < n <= 0:
        body = "0." + "0" * (-n) + digits
    else:
        e = n - 1
        es = ("+" if e >= 0 else "-") + str(abs(e))
        body = (digits if k == 1 else digits[0] + "." + digits[1:]) + "e" + es
    return sign + body


def js_stringify(v) -> str:
    """JSON.stringify(v) for dicts (insertion order), lists/tuples, strings, numbers, booleans, None."""
    if v is None:
        return "null"
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, (int, float, np.integer, np.floating)):
        return js_number(float(v))
    if isinstance(v, str):
        return json.dumps(v, ensure_ascii=False)
    if isinstance(v, dict):
        return "{" + ",".join(json.dumps(str(k), ensure_ascii=False) + ":" + js_stringify(x) for k, x in v.items()) + "}"
    if isinstance(v, (list, tuple, np.ndarray)):
        return "[" + ",".join(js_stringify(x) for x in v) + "]"
    raise TypeError(f"cannot serialise {type(v).__name__}")


# ------------------------------------------------------------------ quantisation and the binary format

def js_round(x: np.ndarray) -> np.ndarray:
    """Math.round: to the nearest integer, halves toward +infinity."""
    f = np.floor(x)
    return f + (x - f >= 0.5)


def quantize(positions: np.ndarray, quantum: float) -> np.ndarray:
    """format.ts:60: max(0, min(65535, round(f / q))) of Float32 positions (3P values)."""
    f = np.asarray(positions, np.float32).astype(np.float64)
    return np.clip(js_round(f / quantum), 0, MAX_U16).astype(np.int64)


def encode_quantized(header: dict, origin: np.ndarray, frames_q) -> bytes:
    """encodeRecording (format.ts:47-77) of frames already quantised (integers 0..65535, 3P each)."""
    head = js_stringify(header).encode("utf-8")
    P = int(header["parcels"])
    out = [struct.pack("<I", len(head)), head, np.asarray(origin, np.uint8).tobytes()]
    prev = None
    for k, cur in enumerate(frames_q):
        cur = np.asarray(cur, np.int64)
        assert cur.size == 3 * P
        if k == 0:
            out.append(cur.astype("<u2").tobytes())
        else:
            d = np.clip(cur - prev, -32768, 32767)
            out.append(d.astype("<i2").tobytes())
            cur = prev + d  # what the decoder will reconstruct
        prev = cur
    return b"".join(out)


def encode_recording(header: dict, origin: np.ndarray, frames) -> bytes:
    """encodeRecording of Float32 position frames (metres, 3P values each)."""
    q = float(header["quantum"])
    return encode_quantized(header, origin, [quantize(f, q) for f in frames])


def decode_recording(buf: bytes):
    """decodeRecording (format.ts:79-100): (header dict, origin u8[P], positions float32[F][3P])."""
    hl = struct.unpack_from("<I", buf, 0)[0]
    header = json.loads(buf[4:4 + hl].decode("utf-8"))
    if header.get("version") != 1:
        raise ValueError(f"Unsupported recording version {header.get('version')}")
    P = header["parcels"]
    o = 4 + hl
    origin = np.frombuffer(buf, np.uint8, P, o).copy()
    o += P
    cur = None
    positions = []
    for k in range(header["frames"]):
        if k == 0:
            cur = np.frombuffer(buf, "<u2", 3 * P, o).astype(np.int64)
        else:
            cur = cur + np.frombuffer(buf, "<i2", 3 * P, o).astype(np.int64)
        o += 6 * P
        positions.append((cur * header["quantum"]).astype(np.float32))
    return header, origin, positions


# ------------------------------------------------------------------ recording a pour on the engine

def record_pour(sim, stride: int = 3, fps: int = 10, quantum: float = 0.00025, label: str | None = None,
                max_seconds: float | None = None) -> bytes:
    """scripts/record3d.ts on an engine simulation: capture, then advance(1 / fps) and capture until the
    pour is finished or 1.5 s after the controller is done. Returns the raw (uncompressed) recording."""
    from . import abi

    P = (sim.n + stride - 1) // stride
    frames, angles, poured = [], [], []

    def capture():
        frames.append(sim.quantized_positions(stride, quantum))
        deg, _ = sim.controller()
        angles.append(deg)
        d = sim.diagnostics()
        fr = sim.discharged_fractions()
        poured.append([0.0, 0.0, 0.0] if fr is None else [float(f * d["dischargedMl"]) for f in fr])

    done_at = -1.0
    capture()
    t0 = sim.diagnostics()["time"]
    while not sim.finished:
        sim.advance(1.0 / fps)
        capture()
        d = sim.diagnostics()
        if d["phase"] == "done" and done_at < 0:
            done_at = d["time"]
        if done_at >= 0 and d["time"] > done_at + 1.5:
            break
        if max_seconds is not None and d["time"] - t0 >= max_seconds - 1e-9:
            break
    shares = sim.discharged_fractions()
    cfg = sim.cfg
    t = cfg.teapot
    cell_mm = cfg.h * 1000
    header = {
        "version": 1,
        "frames": len(frames),
        "parcels": P,
        "fps": fps,
        "quantum": quantum,
        "cellMm": cell_mm,
        "simulatedParcels": sim.n,
        "teapot": {"radius": t.radius, "height": t.height, "wall": t.wall, "inletHeight": t.inlet_height,
                   "boreRadius": t.bore_radius, "spoutAngleDeg": t.spout_angle_deg, "spoutLength": t.spout_length},
        "pivot": [cfg.pivot[0], cfg.pivot[1]],
        "pivotWorld": [sim.pivot_world[0], sim.pivot_world[1]],
        "zOffset": sim.h if cfg.domain == abi.DOMAIN_HALF else (sim.nz // 2) * sim.h,
        "domain": [sim.nx * sim.h, sim.ny * sim.h, sim.nz * sim.h],
        "angles": angles,
        "poured": poured,
        "finalShares": [0.0, 0.0, 0.0] if shares is None else [float(s) for s in shares],
        "label": label or (f"Recorded 3D simulation on the B200 engine ({js_number(cell_mm)} mm cells, {sim.n} "
                           f"parcels); every {stride}th parcel shown."),
    }
    origin = sim.origin()[::stride]
    return encode_quantized(header, origin, frames)


def write_gzip(path: str, raw: bytes) -> None:
    """gzip level 9, as scripts/record3d.ts writes the file."""
    with open(path, "wb") as f:
        f.write(gzip.compress(raw, compresslevel=9))
