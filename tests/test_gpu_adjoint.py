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
