"""ctypes binding of the oracle library (oracle/_build/liboracle.so)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from gpl_b200.design import gpl_result_t, result_to_dict

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build(force=False):
    """Compile the oracle with its Makefile (g++ -O2 -ffp-contract=off)."""
    srcs = [os.path.join(HERE, f) for f in ("oracle_place.cpp", "oracle_nesterov.cpp", "oracle.h")]
    if force or not os.path.exists(SO) or any(os.path.getmtime(s) > os.path.getmtime(SO) for s in srcs):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            build()
        _lib = C.CDLL(SO)
        _lib.oracle_global_placement.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_char_p), C.c_void_p, C.c_int, C.POINTER(gpl_result_t)]
        _lib.oracle_result_free.argtypes = [C.POINTER(gpl_result_t)]
        _lib.oracle_fast_exp.restype = C.c_float
        _lib.oracle_fast_exp.argtypes = [C.c_float]
        _lib.oracle_wavenumber_x.restype = C.c_float
        _lib.oracle_wavenumber_x.argtypes = [C.c_int, C.c_int]
        _lib.oracle_wavenumber_y.restype = C.c_float
        _lib.oracle_wavenumber_y.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float]
        _lib.oracle_round_down_pow2.restype = C.c_uint32
        _lib.oracle_union_area.restype = C.c_int64
        _lib.oracle_distance.restype = C.c_float
        _lib.oracle_derived_reference_hpwl.restype = C.c_float
        _lib.oracle_derived_reference_hpwl.argtypes = [C.c_float, C.c_int64]
        _lib.oracle_fmt.argtypes = [C.c_char_p, C.c_double, C.c_int, C.c_int, C.c_char_p, C.c_int]
        _lib.oracle_extend_size_by_scale.restype = C.c_int64
        _lib.oracle_extend_size_by_scale.argtypes = [C.c_void_p, C.c_double]
        _lib.oracle_eigen_sum.restype = C.c_float
        _lib.oracle_eigen_sum.argtypes = [C.c_int64, C.c_void_p]
        _lib.oracle_csr_from_triplets.restype = C.c_int64
        _lib.oracle_csr_from_triplets.argtypes = [C.c_int64, C.c_int64] + [C.c_void_p] * 6
        _lib.oracle_bicgstab.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int, C.c_void_p, C.c_void_p]
        _lib.oracle_mt19937_nth.restype = C.c_uint32
        _lib.oracle_mt19937_nth.argtypes = [C.c_uint32, C.c_int64]
        _lib.oracle_normal_draws.restype = C.c_uint32
        _lib.oracle_normal_draws.argtypes = [C.c_uint32, C.c_double, C.c_int, C.c_void_p]
        _lib.oracle_max_iter_takes_snapshot.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_float, C.c_float, C.c_int64]
        _lib.oracle_poisson.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float] + [C.c_void_p] * 6
        _lib.oracle_dct1.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        _lib.oracle_transform2.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        _lib.oracle_rudy.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p] + [C.c_void_p] * 5
        _lib.oracle_top_averages.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        _lib.oracle_density_scatter.argtypes = [C.c_int64] + [C.c_void_p] * 6 + [C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_float, C.c_void_p, C.c_void_p]
        _lib.oracle_density_gradient.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_wa.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_void_p]
        _lib.oracle_nesterov_step.argtypes = [C.c_int64] + [C.c_void_p] * 8 + [C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_float, C.c_float, C.c_float] + [C.c_void_p] * 5
        _lib.oracle_gradients.argtypes = [C.c_int64] + [C.c_void_p] * 9 + [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_hpwl.restype = C.c_int64
        _lib.oracle_hpwl.argtypes = [C.c_int64, C.c_void_p, C.c_void_p]
        _lib.oracle_uniform_int_draws.argtypes = [C.c_uint32, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
        _lib.oracle_min_max_idx.argtypes = [C.c_int32] * 6 + [C.c_void_p]
        _lib.oracle_snap_outward.argtypes = [C.c_void_p] + [C.c_int32] * 4
        _lib.oracle_orient_point.argtypes = [C.c_int, C.c_int32, C.c_int32, C.c_void_p]
        _lib.oracle_union_area.argtypes = [C.c_int, C.c_void_p]
        _lib.oracle_distance.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        _lib.oracle_set_size.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
        _lib.oracle_diverge_fallback.argtypes = [C.c_int, C.c_int, C.c_int]
        _lib.oracle_routability_recovery_attempt.argtypes = [C.c_int] * 5
        _lib.oracle_settle_wait_step.argtypes = [C.c_int] * 4 + [C.c_void_p]
        _lib.oracle_round_down_pow2.argtypes = [C.c_uint32]
    return _lib


def global_placement(design, args, router=None, trace=False):
    """Run the reference's `global_placement` command on the CPU; the JSON-shaped report."""
    L = lib()
    cd = design.c_struct()
    argv = (C.c_char_p * max(len(args), 1))(*[a.encode() for a in args])
    res = gpl_result_t()
    L.oracle_global_placement(C.byref(cd), len(args), argv, router, 1 if trace else 0, C.byref(res))
    try:
        return result_to_dict(res)
    finally:
        L.oracle_result_free(C.byref(res))


class Session:
    """The oracle's command with its Nesterov loop stepped by the caller."""

    def __init__(self, design, args, router=None):
        L = lib()
        L.oracle_session_open.restype = C.c_void_p
        L.oracle_session_open.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_char_p), C.c_void_p]
        L.oracle_session_iterate.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.oracle_session_trials.restype = C.c_int64
        L.oracle_session_trials.argtypes = [C.c_void_p]
        L.oracle_session_close.argtypes = [C.c_void_p, C.POINTER(gpl_result_t)]
        self._cd = design.c_struct()
        argv = (C.c_char_p * max(len(args), 1))(*[a.encode() for a in args])
        self._h = L.oracle_session_open(C.byref(self._cd), len(args), argv, router)
        self.done = False

    def iterate(self, n):
        d = C.c_int()
        k = lib().oracle_session_iterate(self._h, n, C.byref(d))
        self.done = bool(d.value)
        return k

    def trials(self):
        return lib().oracle_session_trials(self._h)

    def close(self):
        res = gpl_result_t()
        lib().oracle_session_close(self._h, C.byref(res))
        try:
            return result_to_dict(res)
        finally:
            lib().oracle_result_free(C.byref(res))


def _discard(self):
    lib().oracle_session_discard.argtypes = [C.c_void_p]
    lib().oracle_session_discard(self._h)
    self._h = None


Session.discard = _discard
