"""Device kernels against the oracle on the same inputs (bit-exact where the reference's own
order is kept; a stated tolerance where a sum is reordered or the precision differs)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from tests.gpu_util import dev, ptr, stream, sync

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    from gpl_b200 import engine
    return engine.lib()


def grid(nx, ny, w, h, lx=0, ly=0):
    sx, sy = w / nx, h / ny
    bx = np.array([lx + int(np.floor(i * sx + 0.5)) for i in range(nx + 1)], np.int32)
    by = np.array([ly + int(np.floor(j * sy + 0.5)) for j in range(ny + 1)], np.int32)
    return bx, by, sx, sy


def random_cells(rng, n, bx, by, macro_frac=0.02, filler_frac=0.2):
    lx, ux, ly, uy = bx[0], bx[-1], by[0], by[-1]
    hx = rng.integers(100, 3000, n).astype(np.int32)
    hy = rng.integers(100, 3000, n).astype(np.int32)
    cx = rng.integers(lx - 2000, ux + 2000, n).astype(np.int32)
    cy = rng.integers(ly - 2000, uy + 2000, n).astype(np.int32)
    scale = rng.uniform(0.2, 1.0, n).astype(np.float32)
    u = rng.random(n)
    kind = np.where(u < macro_frac, 1, np.where(u < macro_frac + filler_frac, 2, 0)).astype(np.uint8)
    return cx, cy, hx, hy, scale, kind


# (8, 8): bins so large that the scatter's shared tile sums in 64 bits
@pytest.mark.parametrize("form", ["tiles", "global", "pooled"])
@pytest.mark.parametrize("nx,ny,aligned", [(64, 64, False), (96, 40, False), (64, 64, True), (40, 80, True), (8, 8, False)])
def test_density_scatter_bit_exact(L, nx, ny, aligned, form, monkeypatch):
    """The scatter's three forms (shared tiles, the default; every addend straight to HBM with
    GPL_SCATTER=global; straight to HBM pooled by bin within a warp with GPL_SCATTER=pooled)
    against the oracle's int64 bin sums."""
    monkeypatch.setenv("GPL_SCATTER", form)
    rng = np.random.default_rng(nx * 1000 + ny + aligned)
    if aligned:
        # bins 1000 x 1250 DBU wide and cell edges on multiples of 250: many spans end exactly
        # on a bin edge, where the bin index is decided by the division itself
        bx, by, sx, sy = grid(nx, ny, nx * 1000.0, ny * 1250.0, lx=1000, ly=-500)
        cx, cy, hx, hy, sc, kind = random_cells(rng, 20000, bx, by)
        cx, cy, hx, hy = ((a // 250) * 250 for a in (cx, cy, hx, hy))
        hx, hy = np.maximum(hx, 250).astype(np.int32), np.maximum(hy, 250).astype(np.int32)
        cx, cy = cx.astype(np.int32), cy.astype(np.int32)
    else:
        bx, by, sx, sy = grid(nx, ny, 123457.0, 76543.0, lx=1000, ly=-500)
        cx, cy, hx, hy, sc, kind = random_cells(rng, 20000, bx, by)
    td = np.float32(0.7)
    want_i = np.zeros(nx * ny, np.int64)
    want_f = np.zeros(nx * ny, np.int64)
    O = oracle.lib()
    O.oracle_density_scatter(C.c_int64(len(cx)), *[a.ctypes.data_as(C.c_void_p) for a in (cx, cy, hx, hy, sc, kind)],
                             nx, ny, int(bx[0]), int(by[0]), bx.ctypes.data_as(C.c_void_p), by.ctypes.data_as(C.c_void_p),
                             C.c_double(sx), C.c_double(sy), C.c_float(td), want_i.ctypes.data_as(C.c_void_p), want_f.ctypes.data_as(C.c_void_p))
    d = [dev(a) for a in (cx, cy, hx, hy, sc, kind, bx, by)]
    gi = dev(np.zeros(nx * ny, np.int64))
    gf = dev(np.zeros(nx * ny, np.int64))
    rc = L.gpl_kernel_density_scatter(len(cx), *[ptr(t) for t in d[:6]], nx, ny, int(bx[0]), int(by[0]), ptr(d[6]), ptr(d[7]),
                                      sx, sy, td, ptr(gi), ptr(gf), stream())
    sync()
    assert rc == 0
    np.testing.assert_array_equal(gi.cpu().numpy(), want_i)
    np.testing.assert_array_equal(gf.cpu().numpy(), want_f)


def random_nets(rng, n_nets, span=200000):
    deg = np.where(rng.random(n_nets) < 0.9, rng.integers(2, 6, n_nets), rng.integers(6, 65, n_nets))
    # nets without pins and with one pin, and nets larger than one WA tile (512 pins)
    deg[rng.integers(0, n_nets, 40)] = 0
    deg[rng.integers(0, n_nets, 40)] = 1
    deg[rng.integers(0, n_nets, 5)] = rng.integers(513, 3000, 5)
    deg[-1] = 700
    start = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    npins = int(start[-1])
    xy = rng.integers(0, span, (npins, 2)).astype(np.int32)
    # tight nets too: every pin of some nets within a few hundred DBU
    tight = rng.random(n_nets) < 0.3
    for k in np.flatnonzero(tight)[:2000]:
        xy[start[k]:start[k + 1]] = xy[start[k]] + rng.integers(0, 300, (deg[k], 2))
    w = rng.uniform(1.0, 2.0, n_nets).astype(np.float32)
    return start, xy, w


@pytest.mark.parametrize("coef", [2.1e-4, 1.7e-3])
def test_wa_bit_exact(L, coef):
    rng = np.random.default_rng(7)
    start, xy, w = random_nets(rng, 30000)
    want = np.zeros(2 * len(xy), np.float32)
    oracle.lib().oracle_wa(C.c_int64(len(start) - 1), start.ctypes.data_as(C.c_void_p), xy.ctypes.data_as(C.c_void_p),
                           w.ctypes.data_as(C.c_void_p), C.c_float(coef), C.c_float(coef * 1.25), want.ctypes.data_as(C.c_void_p))
    ds, dxy, dw = dev(start), dev(xy), dev(w)
    g = dev(np.zeros(2 * len(xy), np.float32))
    rc = L.gpl_kernel_wa(len(start) - 1, ptr(ds), ptr(dxy), ptr(dw), coef, coef * 1.25, ptr(g), stream())
    sync()
    assert rc == 0
    np.testing.assert_array_equal(g.cpu().numpy(), want)


@pytest.mark.parametrize("coef,offset", [(1e-5, 0), (3e-4, -100000), (4e-3, 0), (2e-2, -7000000)])
def test_wa_quotients_bit_exact_at_scale(L, coef, offset):
    """The forces' double quotients at scale: 100k nets, about 2M quotients per case, against
    the oracle's IEEE division, bit for bit (signed zeros included); coordinates shifted
    negative in two cases (negative numerators)."""
    rng = np.random.default_rng(17 + int(coef * 1e6))
    start, xy, w = random_nets(rng, 100000, span=4000000)
    xy = (xy.astype(np.int64) + offset).astype(np.int32)
    want = np.zeros(2 * len(xy), np.float32)
    oracle.lib().oracle_wa(C.c_int64(len(start) - 1), start.ctypes.data_as(C.c_void_p), xy.ctypes.data_as(C.c_void_p),
                           w.ctypes.data_as(C.c_void_p), C.c_float(coef), C.c_float(coef * 0.8), want.ctypes.data_as(C.c_void_p))
    ds, dxy, dw = dev(start), dev(xy), dev(w)
    g = dev(np.zeros(2 * len(xy), np.float32))
    assert L.gpl_kernel_wa(len(start) - 1, ptr(ds), ptr(dxy), ptr(dw), coef, coef * 0.8, ptr(g), stream()) == 0
    sync()
    np.testing.assert_array_equal(g.cpu().numpy().view(np.uint32), want.view(np.uint32))


def _poisson_oracle(nx, ny, bin_x, bin_y, dens):
    O = oracle.lib()
    phi, fx, fy = (np.zeros(nx * ny, np.float32) for _ in range(3))
    wx, wy = np.zeros(nx, np.float32), np.zeros(ny, np.float32)
    O.oracle_poisson(nx, ny, C.c_float(bin_x), C.c_float(bin_y), dens.ctypes.data, phi.ctypes.data, fx.ctypes.data, fy.ctypes.data, wx.ctypes.data, wy.ctypes.data)
    return fx, fy, wx, wy


@pytest.mark.parametrize("nx,ny,mode", [(64, 64, 0), (128, 256, 0), (256, 256, 1), (1024, 1024, 1)])
def test_poisson(L, nx, ny, mode):
    rng = np.random.default_rng(nx + ny)
    dens = (rng.random(nx * ny) * 1.5).astype(np.float32)
    fx, fy, wx, wy = _poisson_oracle(nx, ny, 900.0, 1400.0, dens)
    d = dev(dens)
    gx = dev(np.zeros(nx * ny, np.float32))
    gy = dev(np.zeros(nx * ny, np.float32))
    rc = L.gpl_kernel_poisson(nx, ny, wx.ctypes.data, wy.ctypes.data, ptr(d), ptr(gx), ptr(gy), mode, stream())
    sync()
    if mode == 1 and rc == 801:  # cudaErrorNotSupported: the tensor-core path is not built in
        pytest.fail("the split-BF16 tensor-core solver is not available")
    assert rc == 0
    ex, ey = gx.cpu().numpy(), gy.cpu().numpy()
    # FP32 GEMMs: relative to the field's scale, 1e-4; split-BF16 (3 products, 16-bit
    # mantissas, FP32 accumulate): 5e-4
    tol = 1e-4 if mode == 0 else 5e-4
    assert np.max(np.abs(ex - fx)) <= tol * np.max(np.abs(fx))
    assert np.max(np.abs(ey - fy)) <= tol * np.max(np.abs(fy))


@pytest.mark.parametrize("form", [0, 1, 2])
def test_spmv_forms_match_the_reference_order(L, form):
    """`Csr::mul` (src/bicgstab.rs:72-82) bit for bit: each row's products summed in float in
    column order, then 0 + 1 * sum. Rows 512-767 hold 40 entries each (10240 in one block of
    256 rows), past the tiled form's shared-memory tile, so its fallback runs too; the sliced
    form's last slice is partial (5000 rows), empty rows sit beside long ones, and rows 1000-
    1009 run past 64 entries (its warp-per-row part), two of them past 1024 (the top length
    class) and some with a partial last chunk of 32."""
    rng = np.random.default_rng(21)
    n = 5000
    lens = rng.integers(0, 31, n)
    lens[512:768] = 40
    lens[1000:1010] = [65, 96, 100, 129, 200, 300, 997, 1030, 1500, 2047]
    starts = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    cols = np.concatenate([np.sort(rng.choice(n, int(k), replace=False)) for k in lens]).astype(np.int32)
    vals = rng.uniform(-2, 2, int(starts[-1])).astype(np.float32)
    x = rng.uniform(-1e3, 1e3, n).astype(np.float32)
    prod = (vals * x[cols]).astype(np.float32)
    tmp = np.zeros(n, np.float32)
    for j in range(int(lens.max())):
        rows = np.flatnonzero(lens > j)
        tmp[rows] = (tmp[rows] + prod[starts[rows] + j]).astype(np.float32)
    ref = (np.float32(0.0) + np.float32(1.0) * tmp).astype(np.float32)
    d = [dev(starts), dev(cols), dev(vals), dev(x)]  # held across the call
    y = dev(np.full(n, np.nan, np.float32))
    L.gpl_kernel_spmv.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    assert L.gpl_kernel_spmv(n, ptr(d[0]), ptr(d[1]), ptr(d[2]), ptr(d[3]), ptr(y), form, stream()) == 0
    sync()
    assert np.array_equal(y.cpu().numpy().view(np.uint32), ref.view(np.uint32))


def test_csr_from_triplets_matches_the_oracle_at_every_row_length(L):
    """`Csr::from_triplets` (src/bicgstab.rs:501-541) bit for bit: the same row starts, columns
    and summed values. Row lengths reach every tier of the device collapse: up to 64 keys (a
    warp, registers), 256 (a warp, eight per lane), 8192 (a block, shared memory) and beyond (a
    thread); narrow column ranges force many duplicates, summed in triplet order."""
    rng = np.random.default_rng(23)
    n = 4000
    lens = rng.integers(0, 40, n)
    lens[rng.choice(n, 60, replace=False)] = rng.integers(65, 257, 60)
    lens[rng.choice(n, 12, replace=False)] = rng.integers(300, 8193, 12)
    lens[rng.choice(n, 2, replace=False)] = [9000, 20000]
    rows = np.repeat(np.arange(n), lens)
    span = np.where(rng.random(n) < 0.5, 8, n)  # half the rows draw from 8 columns only
    cols = (rng.integers(0, 1 << 30, len(rows)) % np.repeat(span, lens)).astype(np.int64)
    order = rng.permutation(len(rows))  # triplets in no particular order
    rows, cols = rows[order].astype(np.int64), cols[order]
    vals = rng.uniform(-1, 1, len(rows)).astype(np.float32)
    O = oracle.lib()
    ws = np.zeros(n + 1, np.int64)
    wc = np.zeros(len(rows), np.int32)
    wv = np.zeros(len(rows), np.float32)
    nnz = O.oracle_csr_from_triplets(n, len(rows), rows.ctypes.data, cols.ctypes.data, vals.ctypes.data, ws.ctypes.data, wc.ctypes.data, wv.ctypes.data)
    d = [dev(rows.astype(np.int32)), dev(cols.astype(np.int32)), dev(vals)]  # held across the call
    gs = dev(np.zeros(n + 1, np.int64))
    gc = dev(np.zeros(len(rows), np.int32))
    gv = dev(np.zeros(len(rows), np.float32))
    gn = C.c_int64()
    L.gpl_kernel_csr_from_triplets.argtypes = [C.c_int64, C.c_int64] + [C.c_void_p] * 6 + [C.POINTER(C.c_int64), C.c_void_p]
    assert L.gpl_kernel_csr_from_triplets(n, len(rows), ptr(d[0]), ptr(d[1]), ptr(d[2]), ptr(gs), ptr(gc), ptr(gv), C.byref(gn), stream()) == 0
    sync()
    assert gn.value == nnz
    np.testing.assert_array_equal(gs.cpu().numpy(), ws)
    np.testing.assert_array_equal(gc.cpu().numpy()[:nnz], wc[:nnz])
    np.testing.assert_array_equal(gv.cpu().numpy()[:nnz].view(np.uint32), wv[:nnz].view(np.uint32))


def test_bicgstab_matches_the_oracle(L):
    rng = np.random.default_rng(3)
    n = 3000
    rows, cols, vals = [], [], []
    diag = np.zeros(n, np.float32)
    for _ in range(12000):
        a, b = rng.integers(0, n, 2)
        if a == b:
            continue
        w = np.float32(rng.uniform(0.01, 0.5))
        rows += [a, b]
        cols += [b, a]
        vals += [-w, -w]
        diag[a] += w
        diag[b] += w
    for i in range(n):
        rows.append(i)
        cols.append(i)
        vals.append(diag[i] + np.float32(rng.uniform(0.05, 0.2)))
    O = oracle.lib()
    starts = np.zeros(n + 1, np.int64)
    oc = np.zeros(len(rows), np.int32)
    ov = np.zeros(len(rows), np.float32)
    r_ = np.array(rows, np.int64)
    c_ = np.array(cols, np.int64)
    v_ = np.array(vals, np.float32)
    nnz = O.oracle_csr_from_triplets(n, len(rows), r_.ctypes.data, c_.ctypes.data, v_.ctypes.data, starts.ctypes.data, oc.ctypes.data, ov.ctypes.data)
    oc, ov = oc[:nnz], ov[:nnz]
    rhs = rng.uniform(-1e5, 1e5, n).astype(np.float32)
    x0 = rng.uniform(0, 1e4, n).astype(np.float32)
    xo = x0.copy()
    err, conv = C.c_float(), C.c_int()
    O.oracle_bicgstab(n, starts.ctypes.data, oc.ctypes.data, ov.ctypes.data, rhs.ctypes.data, xo.ctypes.data, 100, C.byref(err), C.byref(conv))
    ds, dc, dv, db, dx = dev(starts), dev(oc), dev(ov), dev(rhs), dev(x0)
    it, gerr = C.c_int32(), C.c_float()
    rc = L.gpl_kernel_bicgstab(n, ptr(ds), ptr(dc), ptr(dv), ptr(db), ptr(dx), 100, C.byref(it), C.byref(gerr), stream())
    assert rc == 0
    xg = dx.cpu().numpy()
    assert gerr.value < 1e-5
    np.testing.assert_allclose(xg, xo, rtol=1e-4, atol=1e-3 * np.max(np.abs(xo)))


def test_rudy_matches_the_oracle(L):
    rng = np.random.default_rng(11)
    die = np.array([0, 0, 251234, 199876], np.int32)
    tile, cx, cy = 1000, 251, 199
    n = 20000
    lo = rng.integers(0, 240000, (n, 2))
    size = rng.integers(0, 12000, (n, 2))
    boxes = np.concatenate([lo, lo + size], 1).astype(np.int32)
    boxes[:50] = [2147483647, 2147483647, -2147483648, -2147483648]
    cap_red = np.tile(np.array([10, 0], np.uint8), cx * cy)
    ww = C.c_int32()
    rects = np.zeros(4 * cx * cy, np.int32)
    dem, blk, cong = (np.zeros(cx * cy, np.float32) for _ in range(3))
    pitches = np.array([380, 380, 380], np.int32)
    oracle.lib().oracle_rudy(die.ctypes.data, cx, cy, tile, 3, pitches.ctypes.data, cap_red.ctypes.data, n, boxes.ctypes.data,
                             C.byref(ww), rects.ctypes.data, dem.ctypes.data, blk.ctypes.data, cong.ctypes.data)
    db = dev(boxes)
    gd = dev(np.zeros(cx * cy, np.float32))
    from gpl_b200 import engine
    rc = engine.lib().gpl_kernel_rudy(n, ptr(db), *[int(v) for v in die], cx, cy, tile, ww.value, ptr(gd), stream())
    sync()
    assert rc == 0
    np.testing.assert_allclose(gd.cpu().numpy(), dem, rtol=1e-5, atol=1e-3)


@pytest.mark.parametrize("nx,ny", [(128, 256), (512, 512)])
def test_poisson_errors_against_the_fp64_solve(L, nx, ny):
    """The FP64 device solve is the yardstick: the oracle (an f64 FFT rounded to f32) sits
    within 1e-6 of it, the FP32 GEMM form within 1e-4 and the split-BF16 form within 5e-4 of
    the field's maximum."""
    L.gpl_kernel_poisson_fp64.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(nx * 7 + ny)
    dens = (rng.random(nx * ny) * 1.5).astype(np.float32)
    fx, fy, wx, wy = _poisson_oracle(nx, ny, 900.0, 1400.0, dens)
    d = dev(dens)
    ex64, ey64 = dev(np.zeros(nx * ny)), dev(np.zeros(nx * ny))
    assert L.gpl_kernel_poisson_fp64(nx, ny, wx.ctypes.data, wy.ctypes.data, ptr(d), ptr(ex64), ptr(ey64), stream()) == 0
    sync()
    ex64, ey64 = ex64.cpu().numpy(), ey64.cpu().numpy()
    err = lambda a, b: np.max(np.abs(a - b)) / np.max(np.abs(b))
    assert err(fx, ex64) <= 1e-6 and err(fy, ey64) <= 1e-6
    for mode, tol in ((0, 1e-4), (1, 5e-4)):
        gx, gy = dev(np.zeros(nx * ny, np.float32)), dev(np.zeros(nx * ny, np.float32))
        assert L.gpl_kernel_poisson(nx, ny, wx.ctypes.data, wy.ctypes.data, ptr(d), ptr(gx), ptr(gy), mode, stream()) == 0
        sync()
        assert err(gx.cpu().numpy(), ex64) <= tol and err(gy.cpu().numpy(), ey64) <= tol, mode


@pytest.mark.parametrize("form", ["lean", "pins", "nets"])
def test_wa_small_net_forms_bit_exact(L, form, monkeypatch):
    """The degree-2..4 nets' three kernels (a thread per net forming the exp terms twice, the
    default; a lane per pin with GPL_WA_SMALL=pins; a thread per net keeping them with
    GPL_WA_SMALL=nets) against the oracle, bit for bit: most nets of a netlist are of these
    degrees."""
    monkeypatch.setenv("GPL_WA_SMALL", form)
    rng = np.random.default_rng(71)
    n_nets = 60000
    deg = rng.integers(2, 5, n_nets)
    start = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    xy = rng.integers(0, 400000, (int(start[-1]), 2)).astype(np.int32)
    for k in np.flatnonzero(rng.random(n_nets) < 0.4):
        xy[start[k]:start[k + 1]] = xy[start[k]] + rng.integers(0, 2000, (deg[k], 2))
    w = rng.uniform(1.0, 2.0, n_nets).astype(np.float32)
    want = np.zeros(2 * len(xy), np.float32)
    coef = 3.1e-4
    oracle.lib().oracle_wa(C.c_int64(n_nets), start.ctypes.data_as(C.c_void_p), xy.ctypes.data_as(C.c_void_p),
                           w.ctypes.data_as(C.c_void_p), C.c_float(coef), C.c_float(coef * 1.3), want.ctypes.data_as(C.c_void_p))
    ds, dxy, dw = dev(start), dev(xy), dev(w)
    g = dev(np.zeros(2 * len(xy), np.float32))
    assert L.gpl_kernel_wa(n_nets, ptr(ds), ptr(dxy), ptr(dw), coef, coef * 1.3, ptr(g), stream()) == 0
    sync()
    np.testing.assert_array_equal(g.cpu().numpy().view(np.uint32), want.view(np.uint32))
    got = C.c_int64()
    assert L.gpl_kernel_hpwl(n_nets, ptr(ds), ptr(dxy), 0, C.byref(got), stream()) == 0
    assert got.value == oracle.lib().oracle_hpwl(n_nets, start.ctypes.data_as(C.c_void_p), xy.ctypes.data_as(C.c_void_p))


@pytest.mark.parametrize("nx,ny", [(64, 64), (256, 128)])
def test_poisson_fp64_form_against_the_fp64_solve(L, nx, ny):
    """The engine's FP64 solve form (mode 2, the yardstick its placements are compared with):
    the FP32 form's transforms in double, against the separate double solve
    gpl_kernel_poisson_fp64; the fields agree to float rounding (1e-6 of the largest)."""
    rng = np.random.default_rng(nx * 3 + ny)
    dens = (rng.random(nx * ny) * 1.5).astype(np.float32)
    _, _, wx, wy = _poisson_oracle(nx, ny, 900.0, 1400.0, dens)
    d = dev(dens)
    gx, gy = dev(np.zeros(nx * ny, np.float32)), dev(np.zeros(nx * ny, np.float32))
    assert L.gpl_kernel_poisson(nx, ny, wx.ctypes.data, wy.ctypes.data, ptr(d), ptr(gx), ptr(gy), 2, stream()) == 0
    L.gpl_kernel_poisson_fp64.argtypes = [C.c_int32, C.c_int32] + [C.c_void_p] * 6
    hx, hy = dev(np.zeros(nx * ny, np.float64)), dev(np.zeros(nx * ny, np.float64))
    assert L.gpl_kernel_poisson_fp64(nx, ny, wx.ctypes.data, wy.ctypes.data, ptr(d), ptr(hx), ptr(hy), stream()) == 0
    sync()
    for got, want in ((gx, hx), (gy, hy)):
        g, w = got.cpu().numpy().astype(np.float64), want.cpu().numpy()
        assert np.max(np.abs(g - w)) <= 1e-6 * np.max(np.abs(w))


def test_rudy_on_a_1024_grid_matches_the_oracle(L):
    """RUDY's difference-array form on a 1024 x 1024 tile grid with large boxes (up to a fifth
    of the die a side, as the locality window's nets span), against the reference's per-tile
    visit on the oracle."""
    rng = np.random.default_rng(12)
    die = np.array([0, 0, 1024 * 700 + 321, 1024 * 650 + 77], np.int32)
    tile, cx, cy = 650, 1024, 1024
    n = 4000
    lo = rng.integers(0, 500000, (n, 2))
    size = rng.integers(0, 140000, (n, 2))
    boxes = np.concatenate([lo, lo + size], 1).astype(np.int32)
    cap_red = np.tile(np.array([10, 0], np.uint8), cx * cy)
    ww = C.c_int32()
    rects = np.zeros(4 * cx * cy, np.int32)
    dem, blk, cong = (np.zeros(cx * cy, np.float32) for _ in range(3))
    pitches = np.array([380, 380, 380], np.int32)
    oracle.lib().oracle_rudy(die.ctypes.data, cx, cy, tile, 3, pitches.ctypes.data, cap_red.ctypes.data, n, boxes.ctypes.data,
                             C.byref(ww), rects.ctypes.data, dem.ctypes.data, blk.ctypes.data, cong.ctypes.data)
    db = dev(boxes)
    gd = dev(np.zeros(cx * cy, np.float32))
    from gpl_b200 import engine
    rc = engine.lib().gpl_kernel_rudy(n, ptr(db), *[int(v) for v in die], cx, cy, tile, ww.value, ptr(gd), stream())
    sync()
    assert rc == 0
    np.testing.assert_allclose(gd.cpu().numpy(), dem, rtol=1e-5, atol=1e-3 * float(np.max(dem)) * 1e-2)
