"""The trial's per-cell stages through their C-ABI seams, bit for bit against the oracle on the
same inputs: the Nesterov step with the density centres and the scatter
(`nesterov_update_coordinates`, src/nesterov.rs:2718-2746, :2139-2153, :2218-2250), the
gradient update (`update_gradients`, :2455-2507, over the WA force of :2325-2430 and the density
force of :2434-2449) and the HPWL (`get_hpwl`, :2297-2304). Sizes of the 100k-cell design
(512 x 512 bins) and of the 1M-cell design (1.1M cells with fillers, 1024 x 1024 bins)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from tests.gpu_util import dev, ptr, stream, sync

pytestmark = pytest.mark.gpu

# (cells, bins per side, nets, grid origin): the two designs' sizes; one origin below zero so
# the centres' truncation toward zero meets negative coordinates
SIZES = {"100k": (120_000, 512, 105_000, (-3_000_000, 2000)), "1M": (1_100_000, 1024, 1_050_000, (1000, -500))}


@pytest.fixture(scope="module")
def L():
    from gpl_b200 import engine
    return engine.lib()


def vp(a):
    return a.ctypes.data_as(C.c_void_p)


def grid(nx, ny, lx, ly):
    # bins 1234.5 x 1530.25 DBU: edges rounded, so the bins are not all alike
    sx, sy = 1234.5, 1530.25
    bx = np.array([lx + int(np.floor(i * sx + 0.5)) for i in range(nx + 1)], np.int32)
    by = np.array([ly + int(np.floor(j * sy + 0.5)) for j in range(ny + 1)], np.int32)
    return bx, by, sx, sy


def cells(rng, n, bx, by, sx, sy):
    """Density boxes as the loop holds them: most cells widened to about sqrt(2) bins, a few
    macros of many bins, fillers; kinds 0 std, 1 macro, 2 filler."""
    u = rng.random(n)
    kind = np.where(u < 0.001, 1, np.where(u < 0.15, 2, 0)).astype(np.uint8)
    hx = rng.integers(int(0.71 * sx), int(1.6 * sx), n)
    hy = rng.integers(int(0.71 * sy), int(1.6 * sy), n)
    big = kind == 1
    hx[big] = rng.integers(int(4 * sx), int(30 * sx), big.sum())
    hy[big] = rng.integers(int(4 * sy), int(30 * sy), big.sum())
    scale = np.where(big, 1.0, rng.uniform(0.3, 1.0, n)).astype(np.float32)
    return hx.astype(np.int32), hy.astype(np.int32), scale, kind


@pytest.mark.parametrize("size", list(SIZES))
def test_nesterov_step_bit_exact(L, size):
    n, nb, _, (lx, ly) = SIZES[size]
    rng = np.random.default_rng(11 + nb)
    bx, by, sx, sy = grid(nb, nb, lx, ly)
    hx, hy, scale, kind = cells(rng, n, bx, by, sx, sy)
    W, H = float(bx[-1] - bx[0]), float(by[-1] - by[0])
    # coordinates over the grid and a margin beyond it (the clamp), gradients of both signs
    cur_slp = np.stack([rng.uniform(bx[0] - 0.05 * W, bx[-1] + 0.05 * W, n), rng.uniform(by[0] - 0.05 * H, by[-1] + 0.05 * H, n)], 1).astype(np.float32)
    cur = (cur_slp + rng.normal(0, 2000, (n, 2))).astype(np.float32)
    grad = rng.normal(0, 3.0, (n, 2)).astype(np.float32)
    locked = (rng.random(n) < 0.05).astype(np.uint8)
    step, coeff = np.float32(731.25), np.float32(0.8713)
    td = np.float32(0.7)
    want = [np.zeros(2 * n, np.float32), np.zeros(2 * n, np.float32), np.zeros(2 * n, np.int32), np.zeros(nb * nb, np.int64), np.zeros(nb * nb, np.int64)]
    oracle.lib().oracle_nesterov_step(n, vp(cur_slp), vp(grad), vp(cur), vp(hx), vp(hy), vp(scale), vp(kind), vp(locked), nb, nb, int(bx[0]), int(by[0]),
                                      vp(bx), vp(by), sx, sy, td, step, coeff, *[vp(a) for a in want])
    d = [dev(a) for a in (cur_slp, grad, cur, hx, hy, scale, kind, locked, bx, by)]
    out = [dev(np.zeros_like(a)) for a in want]
    rc = L.gpl_kernel_nesterov_step(n, *[ptr(t) for t in d[:8]], nb, nb, int(bx[0]), int(by[0]), ptr(d[8]), ptr(d[9]), sx, sy, td, step, coeff,
                                    *[ptr(t) for t in out], stream())
    sync()
    assert rc == 0
    names = ["next", "next_slp", "centre", "inst", "filler"]
    for name, g, w in zip(names, out, want):
        got = g.cpu().numpy()
        assert np.array_equal(got.view(np.uint32) if got.dtype == np.float32 else got, w.view(np.uint32) if w.dtype == np.float32 else w), name
    # the locked cells stayed, the others moved, and some of them were clamped
    nxt = out[0].cpu().numpy().reshape(-1, 2)
    assert np.array_equal(nxt[locked == 1], cur[locked == 1])
    assert np.any(nxt[:, 0] == np.float32(bx[0]) + hx.astype(np.float32))


def netlist(rng, n_cells, n_nets, centre, hx, hy):
    """Nets over cells (pins at cell centre + an offset inside the cell), a few pins without a
    cell; degree mix as the synthetic designs, a few nets larger than a WA tile."""
    deg = np.select([rng.random(n_nets) < p for p in (0.55, 0.75, 0.85)], [2, 3, 4], rng.integers(5, 17, n_nets))
    deg[rng.integers(0, n_nets, 50)] = rng.integers(17, 65, 50)
    deg[rng.integers(0, n_nets, 3)] = rng.integers(513, 900, 3)
    deg[rng.integers(0, n_nets, 20)] = 1
    start = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    npins = int(start[-1])
    # a net's cells near its first cell in the cells' order (the centres are spread over the grid)
    first = np.repeat(rng.integers(0, n_cells, n_nets), deg)
    pin_cell = np.clip(first + rng.integers(-400, 401, npins), 0, n_cells - 1)
    pin_cell[rng.random(npins) < 0.002] = -1
    c = np.where(pin_cell[:, None] >= 0, centre[np.maximum(pin_cell, 0)], 0)
    off = np.stack([rng.integers(-1, 2, npins) * (hx[np.maximum(pin_cell, 0)] // 2), rng.integers(-1, 2, npins) * (hy[np.maximum(pin_cell, 0)] // 2)], 1)
    xy = (c + off).astype(np.int32)
    fixed = pin_cell < 0
    xy[fixed] = rng.integers(0, 1_000_000, (fixed.sum(), 2))
    return start, pin_cell.astype(np.int32), xy


@pytest.mark.parametrize("size", list(SIZES))
def test_gradients_bit_exact(L, size):
    n, nb, n_nets, (lx, ly) = SIZES[size]
    rng = np.random.default_rng(23 + nb)
    bx, by, sx, sy = grid(nb, nb, lx, ly)
    hx, hy, scale, _ = cells(rng, n, bx, by, sx, sy)
    centre = np.stack([rng.integers(bx[0], bx[-1], n), rng.integers(by[0], by[-1], n)], 1).astype(np.int32)
    # cells numbered along strips 50 bins wide, so a net of nearby numbers is a local net
    centre = centre[np.lexsort((centre[:, 1], (centre[:, 0] - bx[0]) // int(50 * sx)))]
    dxc = np.maximum(2 * hx - rng.integers(0, 400, n), 1).astype(np.int32)  # the cell's own box
    dyc = np.maximum(2 * hy - rng.integers(0, 400, n), 1).astype(np.int32)
    area = (dxc.astype(np.float32) * dyc.astype(np.float32)).astype(np.float32)
    start, pin_cell, xy = netlist(rng, n, n_nets, centre, hx, hy)
    w = rng.uniform(1.0, 1.5, n_nets).astype(np.float32)
    # each cell's pins in an order of its own (not pin order)
    has = pin_cell >= 0
    pins = np.flatnonzero(has)
    order = np.lexsort((rng.random(len(pins)), pin_cell[pins]))
    cell_pins = pins[order].astype(np.int32)
    cps = np.concatenate([[0], np.cumsum(np.bincount(pin_cell[has], minlength=n))]).astype(np.int64)
    fx = rng.normal(0, 1e-3, nb * nb).astype(np.float32)
    fy = rng.normal(0, 1e-3, nb * nb).astype(np.float32)
    cx_, cy_ = np.float32(2.3e-4), np.float32(1.9e-4)
    penalty = np.float32(3.7e-5)
    want_sum, want_wl, want_den = (np.zeros(2 * n, np.float32) for _ in range(3))
    want_sums = np.zeros(2, np.float32)
    oracle.lib().oracle_gradients(n, vp(np.ascontiguousarray(centre[:, 0])), vp(np.ascontiguousarray(centre[:, 1])), vp(hx), vp(hy), vp(scale), vp(dxc), vp(dyc),
                                  vp(cps), vp(cell_pins), len(start) - 1, vp(start), vp(xy), vp(w), cx_, cy_, nb, nb, int(bx[0]), int(by[0]), vp(bx), vp(by),
                                  sx, sy, vp(fx), vp(fy), penalty, vp(want_sum), vp(want_wl), vp(want_den), vp(want_sums))
    # the device: the WA forces (pin order) through its seam, gathered cell-major, then the
    # gradient kernel
    ds, dxy, dw = dev(start), dev(xy), dev(w)
    force = dev(np.zeros(2 * len(xy), np.float32))
    assert L.gpl_kernel_wa(len(start) - 1, ptr(ds), ptr(dxy), ptr(dw), cx_, cy_, ptr(force), stream()) == 0
    sync()
    import torch
    pf = force.view(-1, 2)[torch.from_numpy(cell_pins.astype(np.int64)).cuda()].contiguous()
    a1 = rng.normal(0, 500, (n, 2)).astype(np.float32)
    b1 = rng.normal(0, 500, (n, 2)).astype(np.float32)
    b2 = rng.normal(0, 1e-2, (n, 2)).astype(np.float32)
    d = [dev(a) for a in (centre, hx, hy, scale, area, cps)]
    dbx, dby, dfx, dfy = dev(bx), dev(by), dev(fx), dev(fy)
    out = dev(np.zeros(2 * n, np.float32))
    da1, db1, db2 = dev(a1), dev(b1), dev(b2)
    sums = np.zeros(4, np.float64)
    rc = L.gpl_kernel_gradients(n, *[ptr(t) for t in d], ptr(pf), nb, nb, int(bx[0]), int(by[0]), ptr(dbx), ptr(dby), sx, sy, ptr(dfx), ptr(dfy), penalty,
                                ptr(out), ptr(da1), ptr(db1), ptr(db2), vp(sums), stream())
    sync()
    assert rc == 0
    got = out.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want_sum.view(np.uint32))
    # the four sums are taken in double on the device: against the exact sums of the same
    # float terms (the oracle's per-cell forces, the float differences squared)
    sq = lambda a, b: np.square((a - b).astype(np.float32)).astype(np.float32)
    exact = [np.abs(want_wl).astype(np.float64).sum(), np.abs(want_den).astype(np.float64).sum(),
             sq(a1, b1).astype(np.float64).sum(), sq(got.reshape(-1, 2), b2).astype(np.float64).sum()]
    np.testing.assert_allclose(sums, exact, rtol=1e-9)
    # and the reference's own float sums of |wl| and |density|, within float rounding
    np.testing.assert_allclose(sums[:2], want_sums.astype(np.float64), rtol=2e-3)


@pytest.mark.parametrize("size", list(SIZES))
@pytest.mark.parametrize("fused", [0, 1])
def test_hpwl_exact(L, size, fused):
    n, _, n_nets, _ = SIZES[size]
    rng = np.random.default_rng(31 + fused)
    centre = rng.integers(-2_000_000, 2_000_000, (n, 2)).astype(np.int32)
    hx = rng.integers(500, 3000, n).astype(np.int32)
    start, _, xy = netlist(rng, n, n_nets, centre, hx, hx)
    # nets without pins too
    deg = np.diff(start)
    deg[rng.integers(0, len(deg), 30)] = 0
    start = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    xy = xy[:start[-1]]
    want = oracle.lib().oracle_hpwl(len(start) - 1, vp(start), vp(np.ascontiguousarray(xy)))
    got = C.c_int64(-1)
    ds, dxy = dev(start), dev(xy)
    assert L.gpl_kernel_hpwl(len(start) - 1, ptr(ds), ptr(dxy), fused, C.byref(got), stream()) == 0
    assert got.value == want
