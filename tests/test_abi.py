"""The C ABI (no GPU): exports, struct layouts, and the engine's host-side construction.

The engine's host construction (pl_plan) must reproduce the reference constructor bit for bit: the
same grid, pivot, seeded positions and origin layers as the oracle and the reference's goldens.
"""
import ctypes as C
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT
from teapotfluidsimulation_b200 import abi

HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(pl_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_function(engine):
    names = declared_functions()
    assert len(names) >= 25
    L = engine.lib()
    for n in names:
        assert hasattr(L, n), n
    assert set(engine.engine.EXPORTED) == set(names)


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "pourlab.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(pl_teapot), sizeof(pl_motion),"
        " sizeof(pl_config), sizeof(pl_diagnostics), sizeof(pl_sizes), sizeof(pl_controller_state),"
        " sizeof(pl_sim_state), offsetof(pl_config, duration), offsetof(pl_diagnostics, discharged_ml),"
        " offsetof(pl_sim_state, controller));return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(abi.Teapot), C.sizeof(abi.Motion), C.sizeof(abi.Config), C.sizeof(abi.Diagnostics),
            C.sizeof(abi.Sizes), C.sizeof(abi.ControllerState), C.sizeof(abi.SimState),
            abi.Config.duration.offset, abi.Diagnostics.discharged_ml.offset, abi.SimState.controller.offset]
    assert got == want


def test_presets_match_python_mirror(engine):
    L = engine.lib()
    c = abi.Config()
    L.pl_gentle_pour(4.0, 20.0, C.byref(c))
    py = abi.gentle_pour(4, 20)
    assert bytes(c) == bytes(py)


@pytest.mark.parametrize("mm", [10, 5, 4])
def test_host_construction_is_bit_exact(engine, oracle_mod, mm):
    cfg = abi.gentle_pour(mm, 20)
    p = engine.engine.plan(cfg)
    s = oracle_mod.OracleSim(cfg)
    o = s.particles()
    assert (p["sizes"].n, p["sizes"].nx, p["sizes"].ny, p["sizes"].nz) == (s.n, s.nx, s.ny, s.nz)
    assert list(p["sizes"].pivot_world) == list(s.sizes.pivot_world)
    assert p["sizes"].parcel_volume == s.sizes.parcel_volume
    assert list(p["sizes"].band_counts) == list(s.sizes.band_counts)
    for k in ("x", "y", "z"):
        assert np.array_equal(p[k], o[k])
    assert np.array_equal(p["origin"], s.origin())


def test_host_construction_matches_reference_goldens(engine, goldens, recording):
    rows = {r["cellMm"]: r for r in goldens["run3d"]}
    for mm in (5, 4):
        p = engine.engine.plan(abi.gentle_pour(mm, 20))
        assert p["sizes"].n == rows[mm]["parcelsHalfPot"]
        assert [p["sizes"].nx, p["sizes"].ny, p["sizes"].nz] == rows[mm]["grid"]
    p = engine.engine.plan(abi.gentle_pour(5, 14))
    assert list(p["sizes"].pivot_world) == goldens["recording"]["pivotWorld"]
    assert np.array_equal(p["origin"][::3], recording["origin"])


def test_bad_config_is_rejected(engine):
    cfg = abi.gentle_pour(5, 20)
    cfg.h = -1.0
    with pytest.raises(engine.EngineError, match="invalid config"):
        engine.engine.plan(cfg)
    cfg = abi.gentle_pour(0.05, 20)  # far too many cells
    with pytest.raises(engine.EngineError, match="out of range"):
        engine.engine.plan(cfg)


def test_missing_library_fails_loudly(tmp_path):
    code = ("import sys; sys.path.insert(0, %r)\n"
            "import teapotfluidsimulation_b200.engine as e\n"
            "e.LIB_PATH = %r\n"
            "try:\n    e.lib()\nexcept ImportError as x:\n    print('raised', 'missing' in str(x))\n") % (
        ROOT, str(tmp_path / "nope.so"))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout
    assert "raised True" in out


def test_noalloc_limit_matches_header(engine):
    text = open(os.path.join(ROOT, "include", "pourlab.h")).read()
    m = re.search(r"#define PL_NOALLOC_MAX_CELLS (\d+)", text)
    assert m and int(m.group(1)) == engine.engine.NOALLOC_MAX_CELLS
