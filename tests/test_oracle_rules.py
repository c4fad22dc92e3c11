"""The oracle against vyges-gpl's own unit-test vectors (tests/golden/reference_rules.json).

Each check restates one reference test; a failure means the oracle no longer follows the
reference rule it cites.
"""
import ctypes as C
import json
import math
import os
import struct

import numpy as np
import pytest

import oracle

G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_rules.json")))
L = oracle.lib()


def f32(x):
    return struct.unpack("f", struct.pack("f", x))[0]


def i32p(vals):
    return (C.c_int32 * len(vals))(*vals)


def test_boost_normal_draws_bit_for_bit():
    g = G["boost_normal_seed1"]
    out = np.zeros(16)
    L.oracle_normal_draws(1, g["sigma"], 16, out.ctypes.data)
    got = [struct.pack(">d", v).hex() for v in out]
    assert got == g["bits"]


def test_boost_engine_position_after_1000_draws():
    g = G["boost_engine_after_1000_draws"]
    assert L.oracle_normal_draws(g["seed"], G["boost_normal_seed1"]["sigma"], g["draws"], None) == g["next_word"]


def test_mt19937_reference_output():
    g = G["mt19937_10000th"]
    assert L.oracle_mt19937_nth(g["seed"], g["n"]) == g["value"]


def test_boost_uniform_int():
    g = G["boost_uniform_int_seed42"]
    out = (C.c_int32 * 20)()
    L.oracle_uniform_int_draws(42, 4, i32p(g["ranges"]), 5, out)
    assert [list(out[r * 5:(r + 1) * 5]) for r in range(4)] == g["draws"]


def test_min_max_idx():
    for args, want in G["min_max_idx"]["cases"]:
        out = (C.c_int32 * 2)()
        L.oracle_min_max_idx(*args, out)
        assert list(out) == want


def test_snap_outward():
    g = G["snap_outward"]
    b = i32p(g["box"])
    L.oracle_snap_outward(b, *g["grid"])
    assert list(b) == g["expect"]


def test_extend_size_by_scale():
    g = G["extend_size_by_scale"]
    b = i32p(g["box"])
    assert L.oracle_extend_size_by_scale(b, g["scale"]) == g["delta"]
    assert list(b) == g["expect"]


def test_orientations():
    names = ["R0", "R90", "R180", "R270", "MY", "MYR90", "MX", "MXR90"]
    for o, x, y, ex, ey in G["orient_point"]["cases"]:
        out = (C.c_int32 * 2)()
        L.oracle_orient_point(names.index(o), x, y, out)
        assert list(out) == [ex, ey]


def _rudy(cap_red, nets, pitches=None):
    g = G["rudy"]
    pitches = g["pitches"] if pitches is None else pitches
    ww = C.c_int32()
    rects = (C.c_int32 * 16)()
    dem, blk, cong = (C.c_float * 4)(), (C.c_float * 4)(), (C.c_float * 4)()
    cr = (C.c_uint8 * 8)(*[v for p in cap_red for v in p])
    flat = [v for n in nets for v in n]
    L.oracle_rudy(i32p(g["die"]), g["grid"][0], g["grid"][1], g["tile"], len(pitches), i32p(pitches or [0]), cr,
                  len(nets), i32p(flat or [0]), C.byref(ww), rects, dem, blk, cong)
    return ww.value, [list(rects[4 * i:4 * i + 4]) for i in range(4)], list(dem), list(blk), list(cong)


def test_rudy_wire_width_and_grid():
    g = G["rudy"]
    ww, rects, *_ = _rudy(g["deposit_cap_red"], [])
    assert ww == g["wire_width"]
    assert rects == g["rects"]
    assert _rudy(g["deposit_cap_red"], [], pitches=[])[0] == g["no_pitch_wire_width"]


def test_rudy_strict_overlap_deposit():
    g = G["rudy"]
    _, _, dem, _, _ = _rudy(g["deposit_cap_red"], g["deposit_nets"])
    assert dem[0] == f32(f32(f32(1.86) * 0.5) * 100.0)
    assert dem[1:] == [0.0, 0.0, 0.0]


def test_rudy_blockage_and_congestion():
    g = G["rudy"]
    _, _, _, blk, cong = _rudy(g["blockage_cap_red"], [])
    assert blk == g["blockage"]
    assert math.isinf(cong[1])


def test_top_averages():
    g = G["rudy"]
    out = (C.c_double * 4)()
    v = np.array([10 - i for i in range(10)], float)
    L.oracle_top_averages(10, v.ctypes.data, out)
    assert list(out) == g["top10"]
    v = np.array([100 - i for i in range(100)], float)
    L.oracle_top_averages(100, v.ctypes.data, out)
    assert list(out) == g["top100"]


def _fmt(which, v, a=0, b=0):
    buf = C.create_string_buffer(128)
    L.oracle_fmt(which.encode(), v, a, b, buf, 128)
    return buf.value.decode()


def test_formats():
    g = G["fmt"]
    for v, p, want in g["fmt_g_prec"]:
        assert _fmt("fmt_g_prec", v, p) == want
    for v, p, w, want in g["fmt_e"]:
        assert _fmt("fmt_e", v, p, w) == want
    for v, want in g["fmt_g"]:
        assert _fmt("fmt_g", v) == want
    for v, want in g["log_f64"]:
        assert _fmt("log_f64", v) == want
    for v, want in g["log_f32"]:
        assert _fmt("log_f32", v) == want
    for v, d, want in g["log_e"]:
        assert _fmt("log_e", v, d) == want


def test_control_rules():
    for saved, reverts, disable, want in G["diverge_fallback"]["cases"]:
        assert L.oracle_diverge_fallback(saved, reverts, disable) == want
    for rs, att, saved, rev, need, want in G["routability_recovery_attempt"]["cases"]:
        assert L.oracle_routability_recovery_attempt(rs, att, saved, rev, need) == want
    for it, dis, saved, rev, sh, so, ov, h, want in G["max_iter_takes_min_hpwl_snapshot"]["cases"]:
        assert L.oracle_max_iter_takes_snapshot(it, 100, dis, saved, rev, sh, so, ov, h) == want
    for start, it, act, st, ws, we, wx in G["settle_wait_step"]["cases"]:
        out = (C.c_int * 3)()
        L.oracle_settle_wait_step(start, it, act, st, out)
        assert out[0] == ws and out[1] == we and (we != 2 or out[2] == wx)


def test_numeric_rules():
    assert L.oracle_fast_exp(0.0) == 1.0
    e = np.float32(1.0) - np.float32(1.0) / np.float32(1024.0)
    for _ in range(10):
        e = np.float32(e * e)
    assert L.oracle_fast_exp(-1.0) == e
    assert L.oracle_fast_exp(-1.0) != np.float32(math.exp(-1.0))
    for x, want in G["round_down_to_power_of_two"]["cases"]:
        assert L.oracle_round_down_pow2(x) == want
    for rects, want in G["union_area"]["cases"]:
        flat = [v for r in rects for v in r] or [0]
        assert L.oracle_union_area(len(rects), i32p(flat)) == want
    a = np.array(G["distance"]["a"], np.float32).ravel()
    b = np.array(G["distance"]["b"], np.float32).ravel()
    assert L.oracle_distance(2, a.ctypes.data, b.ctypes.data) == np.float32(math.sqrt(25.0 / 4.0))
    for user, h, want in G["derived_reference_hpwl"]["cases"]:
        assert L.oracle_derived_reference_hpwl(user, h) == np.float32(want)
    big = L.oracle_derived_reference_hpwl(0.0, 100_000_000_000)
    assert big == np.float32(np.float32(0.01) * np.float32(100_000_000_000))
    b4 = i32p(G["set_size"]["box"])
    L.oracle_set_size(b4, *G["set_size"]["size"])
    assert list(b4) == G["set_size"]["expect"]


def test_wavenumbers():
    assert L.oracle_wavenumber_x(0, 64) == 0.0
    assert L.oracle_wavenumber_x(32, 64) == np.float32(math.pi / 2)
    assert L.oracle_wavenumber_y(32, 64, 3.0, 3.0) == L.oracle_wavenumber_x(32, 64)
    assert L.oracle_wavenumber_y(32, 64, 1.0, 2.0) == np.float32(math.pi)
    assert L.oracle_wavenumber_y(32, 64, 2.0, 1.0) == np.float32(math.pi / 4)


def test_eigen_packet_sum():
    v = np.array(G["eigen_sum"]["v"], np.float32)
    p0 = [f32(1e8 + 1.0), f32(1.0 + 1.0), f32(f32(-1e8) + 1.0), f32(1.0 + 1.0)]
    expect = f32(f32(f32(f32(f32(p0[0] + p0[2]) + f32(p0[1] + p0[3])) + 1.0) + 1.0) + 1.0)
    assert L.oracle_eigen_sum(len(v), v.ctypes.data) == np.float32(expect)
    assert L.oracle_eigen_sum(3, v.ctypes.data) == np.float32(f32(f32(1e8 + 1.0) - 1e8))


def _csr(n, trip):
    rows = np.array([t[0] for t in trip], np.int64)
    cols = np.array([t[1] for t in trip], np.int64)
    vals = np.array([t[2] for t in trip], np.float32)
    starts = np.zeros(n + 1, np.int64)
    oc = np.zeros(len(trip), np.int32)
    ov = np.zeros(len(trip), np.float32)
    nnz = L.oracle_csr_from_triplets(n, len(trip), rows.ctypes.data, cols.ctypes.data, vals.ctypes.data,
                                     starts.ctypes.data, oc.ctypes.data, ov.ctypes.data)
    return starts, oc[:nnz], ov[:nnz]


def test_triplets_collapse_in_order():
    g = G["triplets"]
    starts, cols, vals = _csr(2, g["triplets"])
    assert list(starts) == g["starts"]
    assert list(cols) == g["cols"]
    assert list(vals) == [2.0, 3.0, np.float32(np.float32(np.float32(1e8) + np.float32(1.0)) - np.float32(1e8))]


def test_bicgstab_small_system():
    g = G["bicgstab_2x2"]
    starts, cols, vals = _csr(2, g["triplets"])
    x = np.zeros(2, np.float32)
    rhs = np.array(g["rhs"], np.float32)
    err, conv = C.c_float(), C.c_int()
    L.oracle_bicgstab(2, starts.ctypes.data, cols.ctypes.data, vals.ctypes.data, rhs.ctypes.data, x.ctypes.data,
                      100, C.byref(err), C.byref(conv))
    assert conv.value
    assert abs(x[0] - g["x"][0]) < 1e-6 and abs(x[1] - g["x"][1]) < 1e-6


def test_parse_key_args():
    from gpl_b200 import synth
    d = synth.generate("cfg1")
    g = G["parse_key_args"]
    for arg, line in (g["bad_flag"], g["positional"]):
        r = oracle.global_placement(d, [arg])
        assert r["status"] == "error" and r["lines"][-1] == line
    r = oracle.global_placement(d, ["-bin", "16", "-skip_nesterov"])
    assert r["status"] == "placed" and r["outcome"] == "initially_placed"
    r = oracle.global_placement(d, ["-bin", "16", "-overflow", "0.9"])
    assert any(l.endswith("Bin count (X, Y):          16 ,     16") for l in r["lines"])


def _direct(n, kind, x):
    j = np.arange(n)
    if kind == 0:
        return np.array([np.sum(x * np.cos(np.pi * k * (j + 0.5) / n)) for k in range(n)])
    if kind == 1:
        return np.array([np.sum(x * np.cos(np.pi * j * (k + 0.5) / n)) for k in range(n)])
    A = np.r_[x[1:], x[0]]  # A[1..n], A[n] = a[0]
    kk = np.arange(1, n + 1)
    return np.array([np.sum(A * np.sin(np.pi * kk * (k + 0.5) / n)) for k in range(n)])


@pytest.mark.parametrize("n", [1, 2, 4, 8, 64, 12])
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_transforms_match_their_definitions(n, kind):
    rng = np.random.default_rng(n * 7 + kind)
    x = rng.standard_normal(n)
    out = np.zeros(n)
    L.oracle_dct1(n, kind, x.ctypes.data, out.ctypes.data)
    np.testing.assert_allclose(out, _direct(n, kind, x), rtol=1e-10, atol=1e-10)


def test_forward_then_inverse_is_the_identity():
    # src/ooura.rs:3187-3207: ddct2d(-1), halve row 0 and column 0, scale 4/(n1 n2), ddct2d(+1)
    n1, n2 = 16, 32
    x = np.random.default_rng(3).random((n1, n2)).astype(np.float32)
    a = x.copy()
    L.oracle_transform2(n1, n2, -1, 0, 0, a.ctypes.data)
    a[0, :] *= 0.5
    a[:, 0] *= 0.5
    a *= 4.0 / (n1 * n2)
    L.oracle_transform2(n1, n2, 1, 0, 0, a.ctypes.data)
    assert np.max(np.abs(a - x)) < 1e-5
