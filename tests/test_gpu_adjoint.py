"""The objectives' adjoints (gpl_fn_*) against central finite differences of their own forward
values, and against the reference's forces (the oracle's WA and density gradients).

Finite differences: step 1e-3 site (0.19 DBU), central, on continuous (untruncated) positions;
the adjoint must agree within 1e-4 relative (to the larger of the gradient's magnitude and a
floor of 1e-3 of the largest gradient). The density energy is piecewise quadratic in a cell's
position (its overlaps are piecewise linear), so cells with an edge within two steps of a bin
edge are left out of its check. Against the reference's forces: the reference differentiates
with (1 + e/1024)^1024 for e^e and takes the field at bin centres, so the agreement is stated
as a cosine similarity."""
import ctypes as C

import numpy as np
import pytest

import oracle
from tests.gpu_util import dev, ptr, stream, sync

pytestmark = pytest.mark.gpu

H = 0.19  # 1e-3 site (the site is 190 DBU)


@pytest.fixture(scope="module")
def L():
    from gpl_b200 import engine
    L = engine.lib()
    L.gpl_fn_wa_forward.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_double), C.c_void_p]
    L.gpl_fn_wa_backward.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    dens = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double]
    L.gpl_fn_density_forward.argtypes = dens + [C.POINTER(C.c_double), C.c_void_p]
    L.gpl_fn_density_backward.argtypes = dens + [C.c_double, C.c_void_p, C.c_void_p]
    return L


def _nets(rng, n_nets, span):
    deg = np.where(rng.random(n_nets) < 0.85, rng.integers(2, 6, n_nets), rng.integers(6, 33, n_nets))
    start = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    centre = rng.uniform(0, span, (n_nets, 2))
    xy = np.repeat(centre, deg, axis=0) + rng.uniform(-3000, 3000, (int(start[-1]), 2))
    w = rng.uniform(1.0, 2.0, n_nets).astype(np.float32)
    return start, xy, w


def _check(fd, g):
    floor = 1e-3 * np.max(np.abs(g))
    err = np.abs(fd - g) / np.maximum(np.abs(g), floor)
    assert np.max(err) <= 1e-4, (np.max(err), np.argmax(err))


def test_wa_adjoint_matches_finite_differences(L):
    rng = np.random.default_rng(11)
    start, xy, w = _nets(rng, 3000, 200000.0)
    cx, cy = 7.5e-4, 9e-4
    d_start, d_w = dev(start), dev(w)

    def value(pos):
        v = C.c_double()
        d_pos = dev(np.ascontiguousarray(pos))  # held across the call
        assert L.gpl_fn_wa_forward(len(start) - 1, ptr(d_start), ptr(d_pos), ptr(d_w), cx, cy, C.byref(v), stream()) == 0
        return v.value

    g = dev(np.zeros(xy.size))
    d_xy = dev(xy)
    assert L.gpl_fn_wa_backward(len(start) - 1, ptr(d_start), ptr(d_xy), ptr(d_w), cx, cy, 1.0, ptr(g), stream()) == 0
    sync()
    g = g.cpu().numpy().reshape(-1, 2)
    picks = rng.choice(len(xy), 150, replace=False)
    fd, ga = [], []
    for p in picks:
        for a in range(2):
            plus, minus = xy.copy(), xy.copy()
            plus[p, a] += H
            minus[p, a] -= H
            fd.append((value(plus) - value(minus)) / (2 * H))
            ga.append(g[p, a])
    _check(np.array(fd), np.array(ga))


def test_wa_adjoint_follows_the_reference_force(L):
    """The reference's WA force (gmin - gmax, fast exponentials) is minus this gradient."""
    rng = np.random.default_rng(12)
    start, xy, w = _nets(rng, 3000, 200000.0)
    xy = np.round(xy)
    cx, cy = 7.5e-4, 9e-4
    g = dev(np.zeros(xy.size))
    d = [dev(start), dev(xy), dev(w)]  # held across the call
    assert L.gpl_fn_wa_backward(len(start) - 1, ptr(d[0]), ptr(d[1]), ptr(d[2]), cx, cy, 1.0, ptr(g), stream()) == 0
    sync()
    g = g.cpu().numpy()
    ref = np.zeros(xy.size, np.float32)
    xi = xy.astype(np.int32)
    oracle.lib().oracle_wa(C.c_int64(len(start) - 1), start.ctypes.data_as(C.c_void_p), xi.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.c_void_p),
                           C.c_float(cx), C.c_float(cy), ref.ctypes.data_as(C.c_void_p))
    cos = np.dot(-g, ref) / (np.linalg.norm(g) * np.linalg.norm(ref))
    assert cos > 0.999, cos


def _cells(rng, n, nx, ny, bw, bh):
    xy = np.stack([rng.uniform(0, nx * bw, n), rng.uniform(0, ny * bh, n)], 1)
    half = np.stack([rng.uniform(300, 2500, n), rng.uniform(300, 2500, n)], 1)
    scale = rng.uniform(0.5, 1.0, n)
    return xy, half, scale


def test_density_adjoint_matches_finite_differences(L):
    rng = np.random.default_rng(13)
    nx, ny, bw, bh = 64, 64, 1000.0, 1250.0
    xy, half, scale = _cells(rng, 6000, nx, ny, bw, bh)
    d_half, d_scale = dev(half), dev(scale)

    def energy(pos):
        e = C.c_double()
        d_pos = dev(np.ascontiguousarray(pos))  # held across the call
        assert L.gpl_fn_density_forward(len(pos), ptr(d_pos), ptr(d_half), ptr(d_scale), nx, ny, 0.0, 0.0, bw, bh, C.byref(e), stream()) == 0
        return e.value

    g = dev(np.zeros(xy.size))
    d_xy = dev(xy)
    assert L.gpl_fn_density_backward(len(xy), ptr(d_xy), ptr(d_half), ptr(d_scale), nx, ny, 0.0, 0.0, bw, bh, 1.0, ptr(g), stream()) == 0
    sync()
    g = g.cpu().numpy().reshape(-1, 2)

    def clear(i, a):
        size = bw if a == 0 else bh
        for edge in (xy[i, a] - half[i, a], xy[i, a] + half[i, a]):
            f = edge / size
            if abs(f - round(f)) * size < 2 * H:
                return False
        return True

    picks = [i for i in rng.permutation(len(xy))[:400] if clear(i, 0) and clear(i, 1)][:120]
    fd, ga = [], []
    for i in picks:
        for a in range(2):
            plus, minus = xy.copy(), xy.copy()
            plus[i, a] += H
            minus[i, a] -= H
            fd.append((energy(plus) - energy(minus)) / (2 * H))
            ga.append(g[i, a])
    _check(np.array(fd), np.array(ga))


def test_density_adjoint_follows_the_reference_force(L):
    """The reference's density force (the overlap-weighted spectral field) points along minus
    this gradient: the same solve, the field integrated over the cell against the potential
    differenced across its edges. Cells lie inside the grid, as the placer keeps them (a cell
    hanging over the grid's edge moves only its inside edge's charge, which the field-based
    force does not model)."""
    rng = np.random.default_rng(14)
    nx, ny, bw, bh = 256, 256, 250, 250
    _, _, scale = _cells(rng, 6000, nx, ny, bw, bh)
    half = np.round(rng.uniform(1000, 2500, (6000, 2)))
    xy = np.round(rng.uniform(half, [nx * bw, ny * bh] - half))
    scale = scale.astype(np.float32)
    g = dev(np.zeros(xy.size))
    d = [dev(xy), dev(half), dev(scale.astype(np.float64))]  # held across the call
    assert L.gpl_fn_density_backward(len(xy), ptr(d[0]), ptr(d[1]), ptr(d[2]), nx, ny, 0.0, 0.0, float(bw), float(bh), 1.0, ptr(g), stream()) == 0
    sync()
    g = g.cpu().numpy()
    # the reference: scatter, density, solve, field-weighted overlaps (all on the oracle)
    O = oracle.lib()
    cx, cy = xy[:, 0].astype(np.int32), xy[:, 1].astype(np.int32)
    hx, hy = half[:, 0].astype(np.int32), half[:, 1].astype(np.int32)
    kind = np.zeros(len(xy), np.uint8)
    bx = (np.arange(nx + 1) * bw).astype(np.int32)
    by = (np.arange(ny + 1) * bh).astype(np.int32)
    inst = np.zeros(nx * ny, np.int64)
    fill = np.zeros(nx * ny, np.int64)
    a = lambda v: v.ctypes.data_as(C.c_void_p)
    O.oracle_density_scatter(C.c_int64(len(xy)), a(cx), a(cy), a(hx), a(hy), a(scale), a(kind), nx, ny, 0, 0, a(bx), a(by),
                             C.c_double(bw), C.c_double(bh), C.c_float(1.0), a(inst), a(fill))
    dens = (inst.astype(np.float32) / np.float32(bw * bh)).astype(np.float32)
    phi, fx, fy = (np.zeros(nx * ny, np.float32) for _ in range(3))
    wx, wy = np.zeros(nx, np.float32), np.zeros(ny, np.float32)
    O.oracle_poisson(nx, ny, C.c_float(bw), C.c_float(bh), dens.ctypes.data, phi.ctypes.data, fx.ctypes.data, fy.ctypes.data, wx.ctypes.data, wy.ctypes.data)
    ref = np.zeros(2 * len(xy), np.float32)
    O.oracle_density_gradient(C.c_int64(len(xy)), a(cx), a(cy), a(hx), a(hy), a(scale), nx, ny, 0, 0, a(bx), a(by),
                              C.c_double(bw), C.c_double(bh), a(fx), a(fy), a(ref))
    cos = np.dot(-g, ref) / (np.linalg.norm(g) * np.linalg.norm(ref))
    assert cos > 0.99, cos


def test_autograd_functions_give_the_adjoints(L):
    """The objectives as torch.autograd functions (gpl_b200.functions): their values are the
    forward entry points' and a backward through a weighted sum gives the adjoint entry
    points' gradients, scaled (the WA's bit for bit; the energy's to the last bits its
    double-precision bin sums leave to the order of their atomic adds)."""
    import torch
    from gpl_b200 import functions as F
    rng = np.random.default_rng(15)
    start, xy, w = _nets(rng, 2000, 100000.0)
    cx, cy = 7.5e-4, 9e-4
    t_start, t_w = dev(start), dev(w)
    pxy = torch.tensor(xy, dtype=torch.float64, device="cuda", requires_grad=True)
    W = F.wirelength(pxy, t_start, t_w, cx, cy)
    nx, ny, bw, bh = 64, 64, 1000.0, 1250.0
    cxy_h, half_h, scale_h = _cells(rng, 3000, nx, ny, bw, bh)
    cxy = torch.tensor(cxy_h, dtype=torch.float64, device="cuda", requires_grad=True)
    fn = F.DensityEnergy(nx, ny, 0.0, 0.0, bw, bh)
    t_half, t_scale = dev(half_h), dev(scale_h)
    E = fn(cxy, t_half, t_scale)
    (2.0 * W + 3.0 * E).backward()
    v = C.c_double()
    d_xy = dev(xy)
    assert L.gpl_fn_wa_forward(len(start) - 1, ptr(t_start), ptr(d_xy), ptr(t_w), cx, cy, C.byref(v), stream()) == 0
    assert W.item() == v.value
    gw = dev(np.zeros(xy.size))
    assert L.gpl_fn_wa_backward(len(start) - 1, ptr(t_start), ptr(d_xy), ptr(t_w), cx, cy, 2.0, ptr(gw), stream()) == 0
    e = C.c_double()
    d_cxy = dev(cxy_h)
    assert L.gpl_fn_density_forward(len(cxy_h), ptr(d_cxy), ptr(t_half), ptr(t_scale), nx, ny, 0.0, 0.0, bw, bh, C.byref(e), stream()) == 0
    # the density's bins add in double with atomics, so its last bits vary from call to call
    assert abs(E.item() - e.value) <= 1e-12 * abs(e.value)
    ge = dev(np.zeros(cxy_h.size))
    assert L.gpl_fn_density_backward(len(cxy_h), ptr(d_cxy), ptr(t_half), ptr(t_scale), nx, ny, 0.0, 0.0, bw, bh, 3.0, ptr(ge), stream()) == 0
    sync()
    assert torch.equal(pxy.grad.reshape(-1), gw)
    assert torch.allclose(cxy.grad.reshape(-1), ge, rtol=1e-9, atol=1e-12 * float(ge.abs().max()))
    fn.close()


def test_adjoints_match_finite_differences_at_2m_cells(L):
    """The 2M-cell design (about 2.1M nets and 8.4M pins, its cells at the generator's spread
    placement) on a 2048 x 2048 grid over its core: both adjoints over the whole design
    against central differences on 1000 seeded cells, within 1e-4 (relative to the larger of
    the gradient and 1e-3 of the largest); the WA's step 1e-3 site, the energy's one site
    (exact for its piecewise quadratic, below). The WA coefficient is the one
    the reference's schedule gives at overflow 0.5 (`update_wirelength_coef`,
    src/nesterov.rs:2532-2542, base 0.25 over the mean bin side, :2576); a cell's WA difference is
    taken over its own nets (no other net's term moves with it), the energy's over the whole
    grid. Pins are the cells' (the IO ports' and the macros' are left out of the objective);
    the cells checked have at least one pin."""
    import torch
    from gpl_b200 import functions as F, synth
    d = synth.generate("cfg5", placed=True)
    m = d.meta["cells"]
    box = d.inst_box[:m].astype(np.float64)
    cxy_h = np.stack([(box[:, 0] + box[:, 2]) / 2, (box[:, 1] + box[:, 3]) / 2], 1)
    half_h = np.stack([(box[:, 2] - box[:, 0]) / 2, (box[:, 3] - box[:, 1]) / 2], 1)
    # the cells' pins, net by net (each pin at its cell's corner plus its shape's centre)
    ist = d.net_iterm_start
    inst = d.iterm_inst.astype(np.int64)
    keep = inst < m
    net_of = np.repeat(np.arange(len(ist) - 1), np.diff(ist))[keep]
    pin_cell = inst[keep]
    shp = d.iterm_shape[keep].astype(np.float64)
    off = np.stack([(shp[:, 0] + shp[:, 2]) / 2, (shp[:, 1] + shp[:, 3]) / 2], 1)
    start = np.concatenate([[0], np.cumsum(np.bincount(net_of, minlength=len(ist) - 1))]).astype(np.int64)
    pxy_h = box[pin_cell, :2] + off
    w = np.ones(len(start) - 1, np.float32)
    core_w, core_h = d.core[2] - d.core[0], d.core[3] - d.core[1]
    n = 2048
    bw, bh = core_w / n, core_h / n
    base = 0.25 / ((bw + bh) * 0.5)
    coef = base / 10.0 ** ((0.5 - 0.1) * 20.0 / 9.0 - 1.0)
    t_start, t_w = dev(start), dev(w)
    # the adjoints over the whole design
    g_pin = dev(np.zeros(pxy_h.size))
    d_pxy = dev(pxy_h)
    assert L.gpl_fn_wa_backward(len(start) - 1, ptr(t_start), ptr(d_pxy), ptr(t_w), coef, coef, 1.0, ptr(g_pin), stream()) == 0
    fn = F.DensityEnergy(n, n, float(d.core[0]), float(d.core[1]), bw, bh)
    cxy = torch.tensor(cxy_h, dtype=torch.float64, device="cuda")
    t_half, t_scale = dev(half_h), dev(np.ones(m))
    g_den = torch.zeros_like(cxy)
    assert L.gpl_fn_density_eval(C.c_void_p(fn._f), m, ptr(cxy), ptr(t_half), ptr(t_scale), None, 1.0, ptr(g_den)) == 0
    sync()
    g_pin = g_pin.cpu().numpy().reshape(-1, 2)
    g_wa = np.zeros((m, 2))
    np.add.at(g_wa, pin_cell, g_pin)
    g_den = g_den.cpu().numpy()
    rng = np.random.default_rng(16)

    # the energy's step: one site. E is quadratic in a cell's position while no edge of the
    # cell crosses a bin edge, so a central difference is exact for any step that crosses
    # none; at 2M cells a difference over 1e-3 site would sit below the double sums' rounding
    # (E about 1e10 times the change), so the cells checked keep every edge more than a step
    # from a bin edge and take a one-site step
    HD = 190.0

    def clear(i):
        for a, size, lo in ((0, bw, d.core[0]), (1, bh, d.core[1])):
            for edge in (cxy_h[i, a] - half_h[i, a], cxy_h[i, a] + half_h[i, a]):
                f = (edge - lo) / size
                if abs(f - round(f)) * size < HD + 10.0:
                    return False
        return True

    has_pins = np.bincount(pin_cell, minlength=m) > 0
    cells = [int(i) for i in rng.permutation(m)[:8000] if has_pins[i] and clear(i)][:1000]
    assert len(cells) == 1000
    # the cells' nets and pins, for the local WA differences
    order = np.argsort(pin_cell, kind="stable")
    cstart = np.searchsorted(pin_cell[order], np.arange(m + 1))
    e = C.c_double()
    fd_wa, fd_den, a_wa, a_den = [], [], [], []
    for i in cells:
        pins = order[cstart[i]:cstart[i + 1]]
        nets = np.unique(net_of[pins])
        sub = np.concatenate([np.arange(start[k], start[k + 1]) for k in nets])
        s_start = np.concatenate([[0], np.cumsum(start[nets + 1] - start[nets])]).astype(np.int64)
        mine = np.isin(sub, pins)
        d_s, d_w = dev(s_start), dev(np.ones(len(nets), np.float32))
        for a in range(2):
            vals = []
            for sgn in (1.0, -1.0):
                p = pxy_h[sub].copy()
                p[mine, a] += sgn * H
                d_p = dev(p)
                v = C.c_double()
                assert L.gpl_fn_wa_forward(len(nets), ptr(d_s), ptr(d_p), ptr(d_w), coef, coef, C.byref(v), stream()) == 0
                vals.append(v.value)
            fd_wa.append((vals[0] - vals[1]) / (2 * H))
            a_wa.append(g_wa[i, a])
            vals = []
            for sgn in (1.0, -1.0):
                cxy[i, a] += sgn * HD
                assert L.gpl_fn_density_eval(C.c_void_p(fn._f), m, ptr(cxy), ptr(t_half), ptr(t_scale), C.byref(e), 0.0, None) == 0
                cxy[i, a] = float(cxy_h[i, a])
                vals.append(e.value)
            fd_den.append((vals[0] - vals[1]) / (2 * HD))
            a_den.append(g_den[i, a])
    fn.close()
    print("2M-cell adjoints: WA max rel err", np.max(np.abs(np.array(fd_wa) - a_wa) / np.maximum(np.abs(a_wa), 1e-3 * np.max(np.abs(a_wa)))),
          "density max rel err", np.max(np.abs(np.array(fd_den) - a_den) / np.maximum(np.abs(a_den), 1e-3 * np.max(np.abs(a_den)))))
    _check(np.array(fd_wa), np.array(a_wa))
    _check(np.array(fd_den), np.array(a_den))
