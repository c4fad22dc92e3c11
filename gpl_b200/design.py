"""The design records a `global_placement` run reads, as flat numpy arrays, and their C view.

`Design` mirrors the reference's `Design` (src/placer_base.rs:185-206) flattened into the
arrays of `gpl_design_t` (include/gpl.h). The numpy arrays stay owned by the `Design`; the
C struct only points at them.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

INST_CORE_AUTO_PLACEABLE = 1
INST_BLOCK = 2
INST_FIXED = 4
INST_PLACED = 8
INST_HAS_HALO = 16
BTERM_PLACED = 1
BTERM_FIXED = 2

_P = C.POINTER


class gpl_design_t(C.Structure):
    _fields_ = [
        ("dbu", C.c_int32), ("die", C.c_int32 * 4), ("core", C.c_int32 * 4),
        ("n_rows", C.c_int32), ("row_box", _P(C.c_int32)), ("row_pad", _P(C.c_uint8)), ("row_site", _P(C.c_int32)),
        ("n_insts", C.c_int32), ("inst_box", _P(C.c_int32)), ("inst_flags", _P(C.c_uint32)), ("inst_group", _P(C.c_int32)),
        ("inst_halo", _P(C.c_int32)), ("inst_signal_pins", _P(C.c_int32)), ("inst_orient", _P(C.c_uint8)),
        ("inst_master", _P(C.c_int32)), ("inst_name", _P(C.c_char_p)), ("inst_master_name", _P(C.c_char_p)),
        ("n_nets", C.c_int32), ("net_signal", _P(C.c_uint8)), ("net_iterm_start", _P(C.c_int64)), ("iterm_inst", _P(C.c_int32)),
        ("iterm_shape", _P(C.c_int32)), ("iterm_has_shape", _P(C.c_uint8)), ("iterm_order", _P(C.c_int32)),
        ("net_bterm_start", _P(C.c_int64)), ("bterm_box", _P(C.c_int32)), ("bterm_flags", _P(C.c_uint8)),
        ("net_name", _P(C.c_char_p)), ("bterm_name", _P(C.c_char_p)),
        ("n_groups", C.c_int32), ("group_name", _P(C.c_char_p)), ("group_visual_debug", _P(C.c_uint8)), ("group_region", _P(C.c_int32)),
        ("n_regions", C.c_int32), ("region_bound_start", _P(C.c_int32)), ("region_bounds", _P(C.c_int32)),
        ("region_group_start", _P(C.c_int32)), ("region_groups", _P(C.c_int32)),
        ("n_blockages", C.c_int32), ("blockage_box", _P(C.c_int32)), ("blockage_inst", _P(C.c_int32)),
        ("blockage_inst_fixed", _P(C.c_uint8)), ("blockage_max_density", _P(C.c_float)),
    ]


def _arr(a, dtype):
    a = np.ascontiguousarray(a, dtype=dtype)
    if a.size == 0:  # a valid pointer even for an empty array
        a = np.zeros(1, dtype=dtype)
    return a


def _ptr(a, ctype):
    return a.ctypes.data_as(_P(ctype))


@dataclass
class Design:
    """A design as the placer reads it (src/placer_base.rs:185-206), in DBU."""

    dbu: int
    die: tuple
    core: tuple
    row_box: np.ndarray                 # (R, 4) int32
    row_site: np.ndarray                # (R, 2) int32: site width, height
    inst_box: np.ndarray                # (I, 4) int32
    inst_flags: np.ndarray              # (I,) uint32
    inst_master: np.ndarray             # (I, 2) int32
    net_iterm_start: np.ndarray         # (N+1,) int64
    iterm_inst: np.ndarray              # (T,) int32
    iterm_shape: np.ndarray             # (T, 4) int32
    net_bterm_start: np.ndarray         # (N+1,) int64
    bterm_box: np.ndarray               # (B, 4) int32
    bterm_flags: np.ndarray             # (B,) uint8
    row_pad: np.ndarray = None
    inst_group: np.ndarray = None
    inst_orient: np.ndarray = None
    iterm_order: np.ndarray = None
    iterm_has_shape: np.ndarray = None
    inst_signal_pins: np.ndarray = None
    net_signal: np.ndarray = None
    group_visual_debug: np.ndarray = None
    group_region: np.ndarray = None
    region_bound_start: np.ndarray = None
    region_bounds: np.ndarray = None
    region_group_start: np.ndarray = None
    region_groups: np.ndarray = None
    group_names: list = None
    blockage_box: np.ndarray = None
    blockage_inst: np.ndarray = None
    blockage_inst_fixed: np.ndarray = None
    blockage_max_density: np.ndarray = None
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        n_insts = len(self.inst_box)
        n_iterms = len(self.iterm_inst)
        n_nets = len(self.net_iterm_start) - 1
        if self.row_pad is None:
            self.row_pad = np.zeros(len(self.row_box), np.uint8)
        if self.inst_group is None:
            self.inst_group = np.full(n_insts, -1, np.int32)
        if self.inst_orient is None:
            self.inst_orient = np.zeros(n_insts, np.uint8)
        if self.iterm_has_shape is None:
            self.iterm_has_shape = np.ones(n_iterms, np.uint8)
        if self.iterm_order is None:
            # position among the instance's terminals, in net order
            inst = np.asarray(self.iterm_inst, np.int64)
            srt = np.argsort(inst, kind="stable")
            first = np.searchsorted(inst[srt], inst[srt], side="left")
            order = np.empty(n_iterms, np.int32)
            order[srt] = (np.arange(n_iterms) - first).astype(np.int32)
            self.iterm_order = order
        if self.inst_signal_pins is None:
            self.inst_signal_pins = np.bincount(self.iterm_inst, minlength=n_insts).astype(np.int32)
        if self.net_signal is None:
            self.net_signal = np.ones(n_nets, np.uint8)
        if self.group_names is None:
            self.group_names = []
        ng = len(self.group_names)
        if self.group_visual_debug is None:
            self.group_visual_debug = np.zeros(ng, np.uint8)
        if self.group_region is None:
            self.group_region = np.arange(ng, dtype=np.int32)
        if self.region_bound_start is None:
            self.region_bound_start = np.zeros(1, np.int32)
            self.region_bounds = np.zeros((0, 4), np.int32)
            self.region_group_start = np.zeros(1, np.int32)
            self.region_groups = np.zeros(0, np.int32)
        if self.blockage_box is None:
            self.blockage_box = np.zeros((0, 4), np.int32)
            self.blockage_inst = np.zeros(0, np.int32)
            self.blockage_inst_fixed = np.zeros(0, np.uint8)
            self.blockage_max_density = np.zeros(0, np.float32)

    @property
    def n_insts(self):
        return len(self.inst_box)

    @property
    def n_nets(self):
        return len(self.net_iterm_start) - 1

    def c_struct(self) -> gpl_design_t:
        """The C view; keeps the contiguous arrays alive on the struct."""
        keep = {}

        def a(name, dtype):
            arr = _arr(getattr(self, name), dtype)
            keep[name] = arr
            return arr

        s = gpl_design_t()
        s.dbu = self.dbu
        s.die[:] = list(self.die)
        s.core[:] = list(self.core)
        s.n_rows = len(self.row_box)
        s.row_box = _ptr(a("row_box", np.int32), C.c_int32)
        s.row_pad = _ptr(a("row_pad", np.uint8), C.c_uint8)
        s.row_site = _ptr(a("row_site", np.int32), C.c_int32)
        s.n_insts = self.n_insts
        s.inst_box = _ptr(a("inst_box", np.int32), C.c_int32)
        s.inst_flags = _ptr(a("inst_flags", np.uint32), C.c_uint32)
        s.inst_group = _ptr(a("inst_group", np.int32), C.c_int32)
        s.inst_halo = None
        s.inst_signal_pins = _ptr(a("inst_signal_pins", np.int32), C.c_int32)
        s.inst_orient = _ptr(a("inst_orient", np.uint8), C.c_uint8)
        s.inst_master = _ptr(a("inst_master", np.int32), C.c_int32)
        s.inst_name = None
        s.inst_master_name = None
        s.n_nets = self.n_nets
        s.net_signal = _ptr(a("net_signal", np.uint8), C.c_uint8)
        s.net_iterm_start = _ptr(a("net_iterm_start", np.int64), C.c_int64)
        s.iterm_inst = _ptr(a("iterm_inst", np.int32), C.c_int32)
        s.iterm_shape = _ptr(a("iterm_shape", np.int32), C.c_int32)
        s.iterm_has_shape = _ptr(a("iterm_has_shape", np.uint8), C.c_uint8)
        s.iterm_order = _ptr(a("iterm_order", np.int32), C.c_int32)
        s.net_bterm_start = _ptr(a("net_bterm_start", np.int64), C.c_int64)
        s.bterm_box = _ptr(a("bterm_box", np.int32), C.c_int32)
        s.bterm_flags = _ptr(a("bterm_flags", np.uint8), C.c_uint8)
        s.net_name = None
        s.bterm_name = None
        ng = len(self.group_names)
        s.n_groups = ng
        names = (C.c_char_p * max(ng, 1))(*[g.encode() for g in self.group_names])
        keep["group_names"] = names
        s.group_name = C.cast(names, _P(C.c_char_p))
        s.group_visual_debug = _ptr(a("group_visual_debug", np.uint8), C.c_uint8)
        s.group_region = _ptr(a("group_region", np.int32), C.c_int32)
        s.n_regions = len(self.region_bound_start) - 1
        s.region_bound_start = _ptr(a("region_bound_start", np.int32), C.c_int32)
        s.region_bounds = _ptr(a("region_bounds", np.int32), C.c_int32)
        s.region_group_start = _ptr(a("region_group_start", np.int32), C.c_int32)
        s.region_groups = _ptr(a("region_groups", np.int32), C.c_int32)
        s.n_blockages = len(self.blockage_box)
        s.blockage_box = _ptr(a("blockage_box", np.int32), C.c_int32)
        s.blockage_inst = _ptr(a("blockage_inst", np.int32), C.c_int32)
        s.blockage_inst_fixed = _ptr(a("blockage_inst_fixed", np.uint8), C.c_uint8)
        s.blockage_max_density = _ptr(a("blockage_max_density", np.float32), C.c_float)
        s._keep = keep
        return s


class gpl_result_t(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("outcome", C.c_int32), ("code", C.c_char * 16), ("reason", C.c_char_p),
        ("lines", C.c_char_p), ("trace", C.c_char_p), ("insts", C.c_int64), ("nets", C.c_int64), ("pins", C.c_int64),
        ("iterations", C.c_int32), ("n_bases", C.c_int32), ("bases", _P(C.c_int32)),
        ("n_locations", C.c_int64), ("locations", _P(C.c_int32)), ("final_hpwl", C.c_int64),
        ("final_overflow", C.c_float), ("trials", C.c_int64), ("seconds_initial_place", C.c_double),
        ("seconds_nesterov", C.c_double), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64), ("launches", C.c_int64),
    ]


STATUS = {0: "placed", 2: "error", 3: "refused", -1: "device_fault"}


def result_to_dict(r: gpl_result_t) -> dict:
    """The run's report, shaped as the reference CLI's JSON (src/main.rs:249-262, :362-371)."""
    nloc = r.n_locations
    locs = np.ctypeslib.as_array(r.locations, shape=(nloc * 3,)).reshape(nloc, 3).copy() if nloc else np.zeros((0, 3), np.int32)
    bases = [dict(zip(("group", "place", "fixed", "dummies"), r.bases[4 * b:4 * b + 4])) for b in range(r.n_bases)]
    for b in bases:
        b["group"] = None if b["group"] < 0 else b["group"]
    out = {
        "status": STATUS.get(r.status, str(r.status)),
        "reason": (r.reason or b"").decode() or None,
        "code": r.code.decode() or None,
        "lines": (r.lines or b"").decode().split("\n")[:-1],
        "trace": (r.trace or b"").decode().split("\n")[:-1],
        "insts": r.insts, "nets": r.nets, "pins": r.pins,
        "nesterov_iterations": r.iterations if r.iterations >= 0 else None,
        "bases": bases,
        "locations": locs,
        "final_hpwl": r.final_hpwl, "final_overflow": r.final_overflow, "trials": r.trials,
        "seconds_initial_place": r.seconds_initial_place, "seconds_nesterov": r.seconds_nesterov,
        "outcome": "placed" if r.outcome == 0 else "initially_placed",
        "h2d_bytes": r.h2d_bytes, "d2h_bytes": r.d2h_bytes, "launches": r.launches,
    }
    return out
