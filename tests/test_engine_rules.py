"""The engine's own host rules against vyges-gpl's unit-test vectors (tests/golden/
reference_rules.json), through the library's test-only `gpl_rules_*` exports: the same checks
as tests/test_oracle_rules.py, run on the engine's code instead of the oracle's, so a slip that
both restatements shared would still fail here (no GPU needed: host code only)."""
import ctypes as C

import numpy as np
import pytest

import oracle
import tests.test_oracle_rules as R

SHARED = ["test_boost_normal_draws_bit_for_bit", "test_boost_engine_position_after_1000_draws", "test_mt19937_reference_output",
          "test_boost_uniform_int", "test_min_max_idx", "test_snap_outward", "test_extend_size_by_scale", "test_orientations",
          "test_top_averages", "test_formats", "test_control_rules", "test_numeric_rules", "test_wavenumbers"]


class EngineRules:
    """The engine library seen under the oracle's names: oracle_X is gpl_rules_X, with the
    oracle's argument and result types."""

    def __init__(self):
        from gpl_b200 import build
        self.lib = C.CDLL(build.build())
        self.ref = oracle.lib()

    def __getattr__(self, name):
        assert name.startswith("oracle_"), name
        f = getattr(self.lib, "gpl_rules_" + name[len("oracle_"):])
        o = getattr(self.ref, name)
        f.restype = o.restype
        if o.argtypes is not None:
            f.argtypes = o.argtypes
        return f


@pytest.fixture(scope="module")
def engine_rules():
    return EngineRules()


@pytest.mark.parametrize("name", SHARED)
def test_engine_rule(engine_rules, name, monkeypatch):
    monkeypatch.setattr(R, "L", engine_rules)
    getattr(R, name)()


def test_engine_rudy_grid_blockage_and_congestion(engine_rules):
    """RUDY's host half (wire width, tile grid, blockage, congestion: src/route_base.rs:712-756);
    the demand itself is the device kernel's, checked by the GPU tests."""
    g = R.G["rudy"]
    L = engine_rules.lib
    L.gpl_rules_rudy_grid.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int] + [C.c_void_p] * 7

    def run(cap_red, pitches, demand):
        ww = C.c_int32()
        rects = (C.c_int32 * 16)()
        blk, cong = (C.c_float * 4)(), (C.c_float * 4)()
        cr = (C.c_uint8 * 8)(*[v for p in cap_red for v in p])
        L.gpl_rules_rudy_grid(R.i32p(g["die"]), g["grid"][0], g["grid"][1], g["tile"], len(pitches), R.i32p(pitches or [0]), cr,
                              (C.c_float * 4)(*demand), C.byref(ww), rects, blk, cong)
        return ww.value, [list(rects[4 * i:4 * i + 4]) for i in range(4)], list(blk), list(cong)

    ww, rects, _, _ = run(g["deposit_cap_red"], g["pitches"], [0, 0, 0, 0])
    assert ww == g["wire_width"] and rects == g["rects"]
    assert run(g["deposit_cap_red"], [], [0, 0, 0, 0])[0] == g["no_pitch_wire_width"]
    _, _, blk, cong = run(g["blockage_cap_red"], g["pitches"], [0, 0, 0, 0])
    assert blk == g["blockage"]
    assert np.isinf(cong[1])


@pytest.mark.gpu
def test_engine_parse_key_args():
    """The command's argument rules (src/run.rs:443-455) on the engine: unknown flags and
    positional arguments are errors with the reference's lines; prefixes are accepted."""
    from gpl_b200 import engine, synth
    d = synth.generate("cfg1")
    g = R.G["parse_key_args"]
    for arg, line in (g["bad_flag"], g["positional"]):
        r = engine.global_placement(d, [arg])
        assert r["status"] == "error" and r["lines"][-1] == line
    r = engine.global_placement(d, ["-bin", "16", "-skip_nesterov"])
    assert r["status"] == "placed" and r["outcome"] == "initially_placed"
    r = engine.global_placement(d, ["-bin", "16", "-overflow", "0.9"])
    assert any(l.endswith("Bin count (X, Y):          16 ,     16") for l in r["lines"])
