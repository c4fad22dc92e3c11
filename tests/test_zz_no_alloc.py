"""The allocation-free BiCGSTAB entry point (gpl_kernel_bicgstab_noalloc) against the allocating
one (gpl_kernel_bicgstab), through the C ABI.

Some callers of this library cannot allocate device memory while they call it: a host that
hands out device memory only from a pool sized in advance, a plug-in host that does not let a
library grow the device heap, or code sharing the GPU with latency-critical streams, where
cudaMalloc and cudaFree may wait for the whole device. The no-allocation variant keeps its
scratch in one fixed device array of the library instead. This file is named so that pytest
collects it last; it passes alone in a fresh process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ROWS = 131072  # GPL_BICGSTAB_NOALLOC_MAX_ROWS in include/gpl.h
TOO_LARGE = -2     # GPL_NOALLOC_TOO_LARGE


def _system(n, seed):
    """A diagonally dominant sparse system in CSR (rows sorted by column, duplicates summed)."""
    rng = np.random.default_rng(seed)
    a = rng.integers(0, n, 4 * n)
    b = rng.integers(0, n, 4 * n)
    keep = a != b
    a, b = a[keep], b[keep]
    w = rng.uniform(0.01, 0.5, len(a)).astype(np.float32)
    rows = np.concatenate([a, b, np.arange(n)])
    cols = np.concatenate([b, a, np.arange(n)])
    diag = np.zeros(n, np.float64)
    np.add.at(diag, a, w)
    np.add.at(diag, b, w)
    vals = np.concatenate([-w, -w, (diag + rng.uniform(0.05, 0.2, n)).astype(np.float32)]).astype(np.float32)
    key = rows.astype(np.int64) * n + cols
    order = np.argsort(key, kind="stable")
    key, vals = key[order], vals[order]
    uniq, start = np.unique(key, return_index=True)
    summed = np.add.reduceat(vals.astype(np.float64), start).astype(np.float32)
    r, c = uniq // n, (uniq % n).astype(np.int32)
    row_start = np.zeros(n + 1, np.int64)
    np.add.at(row_start, r + 1, 1)
    row_start = np.cumsum(row_start).astype(np.int64)
    rhs = rng.uniform(-1e5, 1e5, n).astype(np.float32)
    x0 = rng.uniform(0, 1e4, n).astype(np.float32)
    return row_start, c, summed, rhs, x0


def test_no_alloc_solve_matches_the_allocating_solve_twice_in_a_row():
    import torch
    from gpl_b200 import engine
    L = engine.lib()
    L.gpl_kernel_bicgstab_noalloc.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    n = 3000
    rs, cols, vals, rhs, x0 = _system(n, 21)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_rs, d_cols, d_vals, d_rhs = dev(rs), dev(cols), dev(vals), dev(rhs)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())

    x_ref = dev(x0)
    it_ref, err_ref = C.c_int32(), C.c_float()
    assert L.gpl_kernel_bicgstab(n, p(d_rs), p(d_cols), p(d_vals), p(d_rhs), p(x_ref), 100, C.byref(it_ref), C.byref(err_ref), stream) == 0
    want = x_ref.cpu().numpy()
    assert err_ref.value < 1e-5

    for _ in range(2):  # the shared scratch keeps the last call's contents: a second call must not care
        x = dev(x0)
        it, err = C.c_int32(), C.c_float()
        rc = L.gpl_kernel_bicgstab_noalloc(n, p(d_rs), p(d_cols), p(d_vals), p(d_rhs), p(x), 100, C.byref(it), C.byref(err), stream)
        assert rc == 0
        got = x.cpu().numpy()
        # the tolerance of the BiCGSTAB parity test (tests/test_gpu_kernels.py)
        np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-3 * np.max(np.abs(want)))
        assert err.value < 1e-5
        assert it.value == it_ref.value


def test_no_alloc_rejects_a_system_beyond_its_scratch():
    from gpl_b200 import engine
    L = engine.lib()
    L.gpl_kernel_bicgstab_noalloc.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    it, err = C.c_int32(-7), C.c_float()
    # the size check comes first: nothing else is read or launched for an oversized system
    rc = L.gpl_kernel_bicgstab_noalloc(MAX_ROWS + 1, None, None, None, None, None, 100, C.byref(it), C.byref(err), None)
    assert rc == TOO_LARGE
    assert it.value == -7


def test_no_alloc_solves_a_system_of_exactly_its_maximum_size():
    """At n = GPL_BICGSTAB_NOALLOC_MAX_ROWS the solve's scratch fills the fixed array exactly."""
    import torch
    from gpl_b200 import engine
    L = engine.lib()
    L.gpl_kernel_bicgstab_noalloc.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    n = MAX_ROWS
    rs, cols, vals, rhs, x0 = _system(n, 5)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d_rs, d_cols, d_vals, d_rhs = dev(rs), dev(cols), dev(vals), dev(rhs)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())
    x_ref, x = dev(x0), dev(x0)
    it_ref, err_ref, it, err = C.c_int32(), C.c_float(), C.c_int32(), C.c_float()
    assert L.gpl_kernel_bicgstab(n, p(d_rs), p(d_cols), p(d_vals), p(d_rhs), p(x_ref), 100, C.byref(it_ref), C.byref(err_ref), stream) == 0
    assert L.gpl_kernel_bicgstab_noalloc(n, p(d_rs), p(d_cols), p(d_vals), p(d_rhs), p(x), 100, C.byref(it), C.byref(err), stream) == 0
    want, got = x_ref.cpu().numpy(), x.cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-3 * np.max(np.abs(want)))
    assert it.value == it_ref.value and err.value < 1e-5


def test_no_alloc_rejects_a_negative_size():
    from gpl_b200 import engine
    L = engine.lib()
    L.gpl_kernel_bicgstab_noalloc.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    it, err = C.c_int32(-7), C.c_float()
    rc = L.gpl_kernel_bicgstab_noalloc(-1, None, None, None, None, None, 100, C.byref(it), C.byref(err), None)
    assert rc == 1  # cudaErrorInvalidValue
    assert it.value == -7
