"""The engine's Python binding: `global_placement` through the C ABI (include/gpl.h).

`global_placement(design, args)` is the reference's `run::global_placement` (src/run.rs:115):
the command's arguments as the Tcl proc takes them, the report shaped as the CLI's JSON
(src/main.rs:249-262). It runs on a CUDA device through libgpl_b200.so and fails loudly when
the library or the device is missing: there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

from .design import Design, gpl_design_t, gpl_result_t, result_to_dict

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libgpl_b200.so")
_lib = None


class EngineUnavailable(RuntimeError):
    pass


def lib():
    """The engine library (built by gpl_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            raise EngineUnavailable(f"{SO} is missing: build it with `python -m gpl_b200.build`")
        L = C.CDLL(SO)
        L.gpl_create.restype = C.c_void_p
        L.gpl_create.argtypes = [C.c_int]
        L.gpl_destroy.argtypes = [C.c_void_p]
        L.gpl_set_option.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
        L.gpl_global_placement.argtypes = [C.c_void_p, C.POINTER(gpl_design_t), C.c_int, C.POINTER(C.c_char_p), C.c_void_p, C.POINTER(gpl_result_t)]
        L.gpl_result_free.argtypes = [C.POINTER(gpl_result_t)]
        L.gpl_synthetic_router_create.restype = C.c_void_p
        L.gpl_synthetic_router_create.argtypes = [C.POINTER(gpl_design_t), C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.c_uint8]
        L.gpl_synthetic_router_destroy.argtypes = [C.c_void_p]
        L.gpl_kernel_density_scatter.argtypes = [C.c_int64] + [C.c_void_p] * 6 + [C.c_int32] * 4 + [C.c_void_p] * 2 + [C.c_double, C.c_double, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
        L.gpl_kernel_poisson.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.gpl_kernel_wa.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_void_p]
        L.gpl_kernel_bicgstab.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.gpl_kernel_rudy.argtypes = [C.c_int64, C.c_void_p] + [C.c_int32] * 8 + [C.c_void_p, C.c_void_p]
        L.gpl_kernel_nesterov_step.argtypes = [C.c_int64] + [C.c_void_p] * 8 + [C.c_int32] * 4 + [C.c_void_p] * 2 + [C.c_double, C.c_double, C.c_float, C.c_float, C.c_float] + [C.c_void_p] * 6
        L.gpl_kernel_gradients.argtypes = [C.c_int64] + [C.c_void_p] * 7 + [C.c_int32] * 4 + [C.c_void_p] * 2 + [C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_float] + [C.c_void_p] * 6
        L.gpl_kernel_hpwl.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


class Placer:
    """One engine context on one CUDA device (`gpl_create`)."""

    def __init__(self, device=0, poisson="mixed", trace=False):
        L = lib()
        self._ctx = L.gpl_create(device)
        if not self._ctx:
            raise EngineUnavailable(f"CUDA device {device} cannot be used")
        self.set_option("poisson", poisson)
        self.set_option("trace", "1" if trace else "0")

    def set_option(self, name, value):
        if lib().gpl_set_option(self._ctx, name.encode(), str(value).encode()) != 0:
            raise ValueError(f"unknown option {name}={value}")

    def global_placement(self, design: Design, args, router=None) -> dict:
        L = lib()
        cd = design.c_struct()
        argv = (C.c_char_p * max(len(args), 1))(*[a.encode() for a in args])
        res = gpl_result_t()
        if isinstance(router, SyntheticRouter):
            router = router.ptr
        L.gpl_global_placement(self._ctx, C.byref(cd), len(args), argv, router, C.byref(res))
        try:
            return result_to_dict(res)
        finally:
            L.gpl_result_free(C.byref(res))

    def close(self):
        if self._ctx:
            lib().gpl_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def global_placement(design: Design, args, router=None, device=0, poisson="mixed") -> dict:
    """The `global_placement` command on one B200 (src/run.rs:115)."""
    p = Placer(device, poisson)
    try:
        return p.global_placement(design, args, router)
    finally:
        p.close()


class SyntheticRouter:
    """The stand-in router (`gpl_synthetic_router_create`): uniform tiles over the die."""

    def __init__(self, design: Design, tile_size, pitches=(380, 380, 380, 380), capacity=20):
        self._cd = design.c_struct()
        arr = (C.c_int32 * len(pitches))(*pitches)
        self.ptr = lib().gpl_synthetic_router_create(C.byref(self._cd), tile_size, len(pitches), arr, capacity)

    def close(self):
        if self.ptr:
            lib().gpl_synthetic_router_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        self.close()


def _session_lib():
    L = lib()
    if not getattr(L, "_session_ready", False):
        L.gpl_session_open.restype = C.c_void_p
        L.gpl_session_open.argtypes = [C.c_void_p, C.POINTER(gpl_design_t), C.c_int, C.POINTER(C.c_char_p), C.c_void_p]
        L.gpl_session_iterate.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
        L.gpl_session_set_option.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
        L.gpl_session_profile.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int]
        L.gpl_session_stream.restype = C.c_void_p
        L.gpl_session_stream.argtypes = [C.c_void_p]
        L.gpl_session_counters.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        L.gpl_session_tuning.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.gpl_session_regions.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_int]
        L.gpl_session_close.argtypes = [C.c_void_p, C.POINTER(gpl_result_t)]
        L._session_ready = True
    return L


PHASES = ("scatter", "bin_finalize", "density_solve", "wa", "gradients", "hpwl")


class Session:
    """The command with its Nesterov loop stepped by the caller (`gpl_session_*`)."""

    def __init__(self, placer: "Placer", design: Design, args, router=None):
        L = _session_lib()
        self._cd = design.c_struct()
        argv = (C.c_char_p * max(len(args), 1))(*[a.encode() for a in args])
        self._h = L.gpl_session_open(placer._ctx, C.byref(self._cd), len(args), argv, router)
        self.done = False

    def iterate(self, n) -> int:
        d = C.c_int()
        k = _session_lib().gpl_session_iterate(self._h, n, C.byref(d))
        self.done = bool(d.value)
        return k

    def set_option(self, name, value):
        if _session_lib().gpl_session_set_option(self._h, name.encode(), str(value).encode()) != 0:
            raise RuntimeError(f"session option {name}={value} failed")

    def profile(self):
        ms = (C.c_double * 8)()
        n = (C.c_int64 * 8)()
        k = _session_lib().gpl_session_profile(self._h, ms, n, 8)
        return {PHASES[i]: (ms[i], n[i]) for i in range(k)}

    def counters(self):
        out = (C.c_int64 * 6)()
        _session_lib().gpl_session_counters(self._h, out)
        return {"launches": out[0], "h2d_bytes": out[1], "d2h_bytes": out[2], "cells": out[3], "trials": out[4], "reorders": out[5]}

    def regions(self):
        """Each Nesterov region's bin grid, cells and density solver form (0 FP32, 1 split-BF16, 2 FP64)."""
        L = _session_lib()
        n = L.gpl_session_regions(self._h, None, 0)
        buf = (C.c_int32 * (4 * max(n, 1)))()
        L.gpl_session_regions(self._h, buf, n)
        return [dict(nx=buf[4 * b], ny=buf[4 * b + 1], cells=buf[4 * b + 2], form=buf[4 * b + 3]) for b in range(n)]

    def tuning(self) -> str:
        """The autotuner's choices so far and its candidates' median times (text)."""
        L = _session_lib()
        n = L.gpl_session_tuning(self._h, None, 0)
        buf = C.create_string_buffer(n + 1)
        L.gpl_session_tuning(self._h, buf, n + 1)
        return buf.value.decode()

    @property
    def stream(self):
        return _session_lib().gpl_session_stream(self._h)

    def close(self) -> dict:
        res = gpl_result_t()
        _session_lib().gpl_session_close(self._h, C.byref(res))
        self._h = None
        try:
            return result_to_dict(res)
        finally:
            lib().gpl_result_free(C.byref(res))


def _discard(self):
    """Drops the session where it stands (`gpl_session_discard`)."""
    L = _session_lib()
    L.gpl_session_discard.argtypes = [C.c_void_p]
    L.gpl_session_discard(self._h)
    self._h = None


Session.discard = _discard
