#!/usr/bin/env python
"""Benchmark: Nesterov iterations/s of the global-placement engine on one B200 per rank.

Workload (one "step" = one Nesterov iteration with its back-tracking trials): the 1M-cell
synthetic design (about 1.05M nets, 4M pins, 32 macros over 15 % of the core) with a
1024 x 1024 bin grid, `-density 0.70 -bin_grid_count 1024`, the loop started from the
generator's spread placement with the initial placement skipped, after construction, the
Nesterov set-up and W warm-up iterations (untimed). Both arms time the same iterations of the
same loop from the same state. The mixed form (split-BF16 tcgen05 density solve) is the
headline; the plain FP32 form is timed on the next K iterations of the same run. `e2e` is the
whole command (construction and the device's initial placement included) through the C ABI.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

The timed iterations run as the engine runs them (the WA on its own stream beside the density
solve); a separate pass of 10 iterations with the WA after the solve times each phase with CUDA
events for the phase shares and the roofline of the dominant kernel.

N > 1 (under torchrun): one independent replica per GPU (the path has no exchange step), the
time is the max over ranks, `value` the iterations of all ranks over it.
--impl reference: the reference's CPU path (its restatement, single-threaded as the reference
is) on the same workload, the same W warm-up and K timed iterations; the GPU line's
cpu_baseline is the same sample.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Nesterov iters/s at 1M cells,1024² bins: mixed vs FP32 GPU at ≤0.1% HPWL"
CONFIGS = {
    "cfg3": dict(preset="cfg3", args=["-density", "0.70", "-bin_grid_count", "1024"], name="1M cells / 1.05M nets / 4M pins, 1024x1024 bins"),
    "cfg2": dict(preset="cfg2", args=["-density", "0.70", "-bin_grid_count", "512"], name="100k cells / 105k nets / 400k pins, 512x512 bins"),
    "cfg1": dict(preset="cfg1", args=["-density", "0.70", "-bin_grid_count", "64"], name="294 cells / 364 nets / 1122 pins, 64x64 bins"),
    # the batched form: 48 region groups and the top level, each its own bin grid (the placer's
    # rule: 32..256 a side for the groups, 1024 for the top level), one launch per phase
    "cfg4": dict(preset="cfg4", args=["-density", "0.70"], name="2.4M cells / 2.52M nets / 10M pins in 48 region groups and the top level, per-region bin grids"),
}


def grid_side(cfg):
    """The -bin_grid_count of a configuration, or None (each region's grid by the placer's rule)."""
    a = cfg["args"]
    return int(a[a.index("-bin_grid_count") + 1]) if "-bin_grid_count" in a else None


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class Clocks:
    """SM clock and throttle reasons sampled during the timed region: NVML (read-only queries)
    every 2 ms on a thread; a reading as the region opens and one as it closes stand in only when
    the region was too short for the poll; nvidia-smi when NVML cannot answer."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []  # (sm MHz, max sm MHz, set of reasons)
        self.nv = None
        self.h = None
        self.p = None
        self.f = None
        self.stop = None
        self.thread = None

    def _nvml_open(self):
        import pynvml as nv
        import torch
        nv.nvmlInit()
        try:
            props = torch.cuda.get_device_properties(self.device)
            bus = "%08x:%02x:%02x.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
            self.h = nv.nvmlDeviceGetHandleByPciBusId(bus)
            self.nv = nv
            self.bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                         nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            self._read()  # one trial query: a binding that cannot answer falls back to nvidia-smi
        except Exception:
            self.nv = None
            nv.nvmlShutdown()
            raise

    def _read(self):
        nv = self.nv
        sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        return (float(sm), float(mx), {n for n, b in zip(self.NAMES, self.bits) if r & b})

    def _sample(self, into):
        try:
            into.append(self._read())
        except Exception:
            self.errors += 1

    def __enter__(self):
        self.errors = 0
        self.edge = []  # the readings as the region opens and closes
        try:
            self._nvml_open()
        except Exception:
            self.nv = None
        if self.nv is not None:
            self.stop = threading.Event()

            def loop():
                while not self.stop.wait(0.002):
                    self._sample(self.rows)
            self._sample(self.edge)
            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return self
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.nv is not None:
            self._sample(self.edge)
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        # the readings taken while the work ran; the two edge readings only when the poll took
        # none (the opening one can catch a clock still ramping up)
        rows = list(self.rows) or list(getattr(self, "edge", []))
        source = "nvml"
        if self.f is not None:
            source = "nvidia-smi"
            self.f.flush()
            for line in open(self.f.name):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    mx = float(parts[2]) if parts[2].replace(".", "").isdigit() else 0.0
                    rows.append((float(parts[1]), mx, {self.NAMES[i] for i in range(4) if parts[5 + i].lower() in ("active", "1")}))
            os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock samples"]}
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(set().union(*(r[2] for r in rows))), "samples": len(rows), "source": source,
                "edge_only": not self.rows and self.f is None}


def solve_flops(regions):
    """The density solves' FLOPs over every region: six GEMMs of 2 nx ny K flops each (K = ny for
    the three y transforms, nx for the x ones), three products apiece in the split-BF16 form."""
    return sum((3.0 if r["form"] == 1 else 1.0) * 6.0 * r["nx"] * r["ny"] * (r["nx"] + r["ny"]) for r in regions)


def algorithmic(phase, C, P, N, B, mixed, flops):
    """Bytes (or FLOPs) one launch of a phase must move (compulsory traffic), over every region
    (B: the bins of every region; flops: the density solves' FLOPs)."""
    if phase == "scatter":
        return "hbm", C * 61 + B * 16  # cell state in, next/next_slp/centre out; the two int64 accumulators
    if phase == "bin_finalize":
        return "hbm", B * (56 + (4 if mixed else 0))
    if phase == "wa":
        return "hbm", N * 16 + P * 28
    if phase == "gradients":
        return "hbm", C * 64 + P * 12 + B * 8
    if phase == "hpwl":
        return "hbm", N * 8 + P * 20
    if phase == "density_solve":
        return "tensor" if mixed else "fp32", flops
    return "hbm", 0


def max_over_ranks(x, device=None):
    """The largest of every rank's x (each rank calls it at the same point); x itself on one rank."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def log(msg):
    print(f"[bench {time.perf_counter() - T0:8.2f}] {msg}", file=sys.stderr, flush=True)


T0 = time.perf_counter()


START = {
    "spread": "the generator's spread placement, initial placement skipped (both arms)",
    "ip": "after the initial placement (profiling case)",
}


def workload(a, design):
    """The workload as both arms name it: the same keys and values in either line."""
    cfg = CONFIGS[a.config]
    nx = grid_side(cfg)
    m = design.meta
    return {"workload": cfg["name"], "args": cfg["args"], "design": m["config"], "cells": m["cells"], "nets": m["nets"],
            "pins": m["pins"], "bins": nx * nx if nx else "each region its own grid", "start": START[a.start] if not a.start_from else "a saved initial placement",
            "timed": f"Nesterov iterations {a.warmup + 1}..{a.warmup + a.steps} of the loop (iteration = step)",
            "parallelism": "replicas x1", "l2": "working set > L2 (126 MB): cells, pins and bins stream from HBM each trial"}


def loop_design(a):
    """The design the timed loop starts from, and the command's arguments for it."""
    from gpl_b200 import synth
    cfg = CONFIGS[a.config]
    design = synth.generate(cfg["preset"], placed=a.start == "spread")
    if a.start_from:
        # the saved initial placement as the design's placement (lower-left corners), so the
        # loop starts where the initial placement left it without running it again
        loc = np.load(a.start_from)
        box = design.inst_box
        w, h = box[loc[:, 0], 2] - box[loc[:, 0], 0], box[loc[:, 0], 3] - box[loc[:, 0], 1]
        box[loc[:, 0], 0], box[loc[:, 0], 1] = loc[:, 1], loc[:, 2]
        box[loc[:, 0], 2], box[loc[:, 0], 3] = loc[:, 1] + w, loc[:, 2] + h
        design.inst_flags[loc[:, 0]] |= synth.INST_PLACED
    skip_ip = a.start == "spread" or bool(a.start_from)
    return design, cfg["args"] + (["-skip_initial_place"] if skip_ip else [])


def ours(a):
    import torch
    import torch.distributed as dist
    from gpl_b200 import engine, synth
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    cfg = CONFIGS[a.config]
    if a.initial_place_only:
        # a profiling case: the command through the initial placement only
        design = synth.generate(cfg["preset"])
        t0 = time.perf_counter()
        r = engine.global_placement(design, cfg["args"] + ["-skip_nesterov_place"], device=local)
        print(json.dumps({"case": "initial placement only", "config": cfg["name"], "status": r["status"],
                          "seconds": time.perf_counter() - t0, "seconds_initial_place": r["seconds_initial_place"]}))
        if a.save_placement:
            np.save(a.save_placement, r["locations"])
        return
    design, args = loop_design(a)
    log("design generated")
    placer = engine.Placer(local, a.form)
    placer.set_option("reorder", a.reorder)
    sess = engine.Session(placer, design, args)
    log("session open")
    sess.iterate(a.warmup)
    log("warm-up done")
    if sess.done:
        raise SystemExit("the loop ended during warm-up: " + json.dumps(sess.close().get("reason")))
    stream = torch.cuda.ExternalStream(sess.stream, device=local)

    def timed(k):
        c0 = sess.counters()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clk:
            e0.record(stream)
            t0 = time.perf_counter()
            done = sess.iterate(k)
            e1.record(stream)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
        if world > 1:
            dist.barrier()
        ms = e0.elapsed_time(e1)
        c1 = sess.counters()
        ms = max_over_ranks(ms, f"cuda:{local}")
        return {"ms": ms, "iters": done, "wall_s": wall, "clocks": clk.summary(), "launches": c1["launches"] - c0["launches"],
                "trials": c1["trials"] - c0["trials"]}

    def phase_times(k):
        # each phase's own device time: events around each phase's launches, with the WA after
        # the density solve instead of beside it (outside the timed region above)
        sess.set_option("overlap", "0")
        sess.set_option("profile", "1")
        sess.iterate(k)
        prof = sess.profile()
        sess.set_option("profile", "0")
        sess.set_option("overlap", "1")
        return prof

    cells_total = sess.counters()["cells"]
    regions = sess.regions()
    B = sum(r["nx"] * r["ny"] for r in regions)
    if a.form == "mixed":
        mixed = timed(a.steps)
        mixed["profile"] = phase_times(min(a.steps, 10))
        sess.set_option("poisson", "fp32")
        sess.iterate(min(a.warmup, 3))
    fp32 = timed(a.steps)
    fp32["profile"] = phase_times(min(a.steps, 10))
    if a.form == "fp32":
        mixed = fp32
    tuning = sess.tuning()
    log("timed")
    res = sess.close()
    log("session closed")
    P_pins, N_nets = res["pins"], res["nets"]
    nx = max(max(r["nx"], r["ny"]) for r in regions)
    # e2e: the whole command through the public C ABI, host arrays in (construction and the
    # initial placement included), locations out
    e2e = None
    if not a.no_e2e:
        full = synth.generate(cfg["preset"])
        t0 = time.perf_counter()
        r = engine.global_placement(full, cfg["args"], device=local, poisson=a.form)
        e2e_s = max_over_ranks(time.perf_counter() - t0, f"cuda:{local}")
        log("e2e run done")
        its = r["nesterov_iterations"] or 0
        e2e = {"value": its * world / e2e_s if e2e_s > 0 else 0.0, "unit": "iters/s", "seconds": e2e_s,
               "iterations": its, "trials": r["trials"], "status": r["status"],
               "what": "the whole global_placement command (construction, initial placement, Nesterov loop, written placement) through the C ABI with host arrays",
               "h2d_bytes_per_step": int(r["h2d_bytes"] / max(its, 1)), "d2h_bytes_per_step": int(r["d2h_bytes"] / max(its, 1)),
               "final_hpwl": r["final_hpwl"], "final_overflow": r["final_overflow"],
               "seconds_initial_place": r["seconds_initial_place"], "seconds_nesterov": r["seconds_nesterov"]}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    pk, pk_kind = peaks()
    value = mixed["iters"] * world / (mixed["ms"] / 1000.0)
    value_fp32 = fp32["iters"] * world / (fp32["ms"] / 1000.0)
    # the dominant kernel of the mixed form by device time
    prof = mixed["profile"]
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    name, (ms_tot, launches) = dom
    bound, work = algorithmic(name, cells_total, P_pins, N_nets, B, a.form == "mixed", solve_flops(regions))
    per_launch_s = ms_tot / 1000.0 / max(launches, 1)
    if bound == "fp32":
        achieved = work / per_launch_s / 1e12
        roof = {"bound": "fp32-simt", "achieved": achieved, "peak": 2 * 148 * 128 * pk.get("sm_max_mhz", 1965.0) * 1e6 / 1e12, "unit": "TFLOP/s"}
    elif bound == "tensor":
        achieved = work / per_launch_s / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": pk["bf16_tflops_sustained"], "unit": "TFLOP/s"}
    else:
        achieved = work / per_launch_s / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s"}
    roof["frac"] = roof["achieved"] / roof["peak"]
    roof["kernel"] = name
    roof["peak_source"] = pk_kind
    traffic = None
    try:
        summ = json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json")))
        traffic = summ.get(name, {}).get("bytes_per_launch")
    except Exception:
        pass
    roof["traffic"] = traffic
    phases = {k: {"ms_total": v[0], "launches": v[1], "share": v[0] / max(sum(x[0] for x in prof.values()), 1e-9)} for k, v in prof.items()}
    cpu = None
    if world == 1 and not a.no_cpu_baseline:
        cpu = cpu_sample(a)
    precision = precision_report(local, nx)
    if not a.no_precision_runs and world == 1:
        precision["runs"] = precision_runs(local, cfg)
    conf = workload(a, design)
    conf["parallelism"] = f"replicas x{world}"
    out = {
        "metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": mixed["ms"] / max(mixed["iters"], 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+bf16x3 (split-BF16 density solve), f64 reductions", "data": "synthetic",
        "config": conf, "form": a.form, "trials": mixed["trials"], "trials_per_s": mixed["trials"] * world / (mixed["ms"] / 1000.0),
        "forms": {"mixed": {"iters_per_s": value, "ms_per_iter": mixed["ms"] / max(mixed["iters"], 1), "iters": mixed["iters"], "trials": mixed["trials"]},
                  "fp32": {"iters_per_s": value_fp32, "ms_per_iter": fp32["ms"] / max(fp32["iters"], 1), "iters": fp32["iters"], "trials": fp32["trials"],
                           "note": "timed on the iterations after the mixed form's, from the same run"},
                  "mixed_over_fp32": value / value_fp32 if value_fp32 else None},
        "phases": phases, "roofline": roof, "gpu_launches": mixed["launches"], "clocks": mixed["clocks"],
        "e2e": e2e, "cpu_baseline": cpu, "precision": precision, "tuning": tuning,
    }
    print(json.dumps(out))


# ---- the cuFFT comparison point for the density solve (a measurement, not an engine form):
# the same four transforms (src/nesterov.rs:412-444: the forward 2-D DCT, then the DST-DCT
# and DCT-DST inverses for the two fields) through FFTs (torch.fft runs cuFFT) in FP32, each
# 1-D transform by Makhoul's reordering (a DCT-II of length N is one complex FFT of the
# even-then-reversed-odd samples and a twiddle), the inverse by the same in reverse, and the
# shifted DST-III (its k = 0 term the (-1)^n one) as (-1)^n times the DCT-III of the
# coefficients in reverse order.
def _dct2(a, dim):
    import math
    import torch
    a = a.movedim(dim, -1)
    N = a.shape[-1]
    v = torch.cat([a[..., ::2], a[..., 1::2].flip(-1)], dim=-1)
    k = torch.arange(N, device=a.device, dtype=a.dtype)
    return (torch.fft.fft(v, dim=-1) * torch.polar(torch.ones_like(k), -math.pi * k / (2 * N))).real.movedim(-1, dim)


def _dct3(X, dim):
    """y[n] = sum_k X[k] cos(pi k (2n+1) / 2N), every weight 1."""
    import math
    import torch
    X = X.movedim(dim, -1)
    N = X.shape[-1]
    Y = torch.cat([X[..., :1] * N, X[..., 1:] * (N / 2.0)], dim=-1)
    Yr = torch.cat([torch.zeros_like(Y[..., :1]), Y[..., 1:].flip(-1)], dim=-1)
    k = torch.arange(N, device=X.device, dtype=X.dtype)
    v = torch.fft.ifft(torch.polar(torch.ones_like(k), math.pi * k / (2 * N)) * torch.complex(Y, -Yr), dim=-1).real
    y = torch.empty_like(v)
    y[..., ::2] = v[..., : (N + 1) // 2]
    y[..., 1::2] = v[..., (N + 1) // 2:].flip(-1)
    return y.movedim(-1, dim)


def _dst3(S, dim):
    """y[n] = sum_u S[u] sin(pi k'_u (2n+1) / 2N), k'_0 = N, k'_u = u."""
    import torch
    S = S.movedim(dim, -1)
    N = S.shape[-1]
    y = _dct3(torch.cat([S[..., :1], S[..., 1:].flip(-1)], dim=-1), -1)
    sign = 1.0 - 2.0 * (torch.arange(N, device=S.device) % 2).to(S.dtype)
    return (y * sign).movedim(-1, dim)


def fft_density_solve(rho, wx, wy):
    """The fields (x-major [x][y]) of a density by FFTs: the transforms above with the
    forward scaling (1/n for the first coefficient, 2/n for the rest, each axis) and the
    spectral step of the engine's forms (the (0, 0) term zero). No host value is copied in
    (it runs inside a CUDA graph capture)."""
    import torch
    nx, ny = rho.shape
    ix, iy = torch.arange(nx, device=rho.device), torch.arange(ny, device=rho.device)
    hx = torch.full((nx,), 2.0 / nx, dtype=rho.dtype, device=rho.device).masked_fill(ix == 0, 1.0 / nx)
    hy = torch.full((ny,), 2.0 / ny, dtype=rho.dtype, device=rho.device).masked_fill(iy == 0, 1.0 / ny)
    A = _dct2(_dct2(rho, 1), 0) * hx[:, None] * hy[None, :]
    z00 = (ix[:, None] == 0) & (iy[None, :] == 0)
    d = (wx[:, None] * wx[:, None] + wy[None, :] * wy[None, :]).masked_fill(z00, 1.0)
    P = (A / d).masked_fill(z00, 0.0)
    return _dst3(_dct3(P * wx[:, None], 1), 0), _dct3(_dst3(P * wy[None, :], 1), 0)


def cufft_point(local, n, dens, ex, ey, wx, wy):
    """The FFT solve in FP32 on the device, captured in a CUDA graph (so the host's launches
    do not set the pace), timed over 50 replays with CUDA events; its field error against the
    FP64 yardstick as for the engine's forms."""
    import torch
    dev = f"cuda:{local}"
    rho = dens.view(n, n)
    twx, twy = torch.from_numpy(wx).to(dev), torch.from_numpy(wy).to(dev)
    s = torch.cuda.Stream(dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(s):
        for _ in range(3):
            fx, fy = fft_density_solve(rho, twx, twy)
    torch.cuda.current_stream(dev).wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fx, fy = fft_density_solve(rho, twx, twy)
    for _ in range(3):
        g.replay()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    e0.record()
    for _ in range(50):
        g.replay()
    e1.record()
    torch.cuda.synchronize(dev)
    us = e0.elapsed_time(e1) * 1000.0 / 50
    err = max(float((fx.reshape(-1).double() - ex).abs().max() / ex.abs().max()), float((fy.reshape(-1).double() - ey).abs().max() / ey.abs().max()))
    del g
    return {"what": "torch.fft (cuFFT) FP32: the four transforms as FFTs with Makhoul's reordering, one CUDA graph", "us_per_solve": us, "field_rel_err": err}


def precision_report(local, n):
    """Each form's field error against the FP64 device solve (the same transforms in double),
    on a seeded density of the workload's grid: max |error| over max |field|."""
    import ctypes as C
    import torch
    from gpl_b200 import engine
    L = engine.lib()
    L.gpl_kernel_poisson_fp64.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(n)
    dens = torch.from_numpy((rng.random(n * n) * 1.5).astype(np.float32)).cuda(local)
    wx = (np.pi * np.arange(n) / n).astype(np.float32)
    wy = wx.copy()
    st = C.c_void_p(torch.cuda.current_stream(local).cuda_stream)
    ex, ey = torch.zeros(n * n, dtype=torch.float64, device=f"cuda:{local}"), torch.zeros(n * n, dtype=torch.float64, device=f"cuda:{local}")
    if L.gpl_kernel_poisson_fp64(n, n, wx.ctypes.data, wy.ctypes.data, C.c_void_p(dens.data_ptr()), C.c_void_p(ex.data_ptr()), C.c_void_p(ey.data_ptr()), st) != 0:
        return None
    out = {"yardstick": f"FP64 device solve, {n}x{n} seeded density"}
    for name, mode in (("mixed", 1), ("fp32", 0)):
        gx, gy = torch.zeros(n * n, device=f"cuda:{local}"), torch.zeros(n * n, device=f"cuda:{local}")
        if L.gpl_kernel_poisson(n, n, wx.ctypes.data, wy.ctypes.data, C.c_void_p(dens.data_ptr()), C.c_void_p(gx.data_ptr()), C.c_void_p(gy.data_ptr()), mode, st) != 0:
            continue
        torch.cuda.synchronize(local)
        e = max(float((gx.double() - ex).abs().max() / ex.abs().max()), float((gy.double() - ey).abs().max() / ey.abs().max()))
        out[f"field_rel_err_{name}"] = e
    try:
        out["cufft_fp32"] = cufft_point(local, n, dens, ex, ey, wx, wy)
    except Exception as err:  # a comparison point: its failure leaves the report as it was
        out["cufft_fp32"] = {"unavailable": str(err)[:200]}
    return out


def precision_runs(local, cfg):
    """Each form's whole command against the same command with the FP64 density solve (the
    transforms in double throughout) on the workload's design: final HPWL and overflow, and
    the written placement's coordinates (DBU), as errors against the FP64 run."""
    from gpl_b200 import engine, synth
    design = synth.generate(cfg["preset"])
    runs = {f: engine.global_placement(design, cfg["args"], device=local, poisson=f) for f in ("fp64", "mixed", "fp32")}
    ref = runs["fp64"]
    out = {"yardstick": "the same command with the FP64 density solve", "fp64": {"final_hpwl": ref["final_hpwl"], "final_overflow": ref["final_overflow"], "iterations": ref["nesterov_iterations"]}}
    for f in ("mixed", "fp32"):
        r = runs[f]
        d = np.abs(r["locations"][:, 1:].astype(np.int64) - ref["locations"][:, 1:].astype(np.int64)) if len(r["locations"]) == len(ref["locations"]) else np.zeros(1)
        out[f] = {"final_hpwl_rel_err": abs(r["final_hpwl"] - ref["final_hpwl"]) / max(ref["final_hpwl"], 1), "final_overflow_err": abs(r["final_overflow"] - ref["final_overflow"]),
                  "iterations": r["nesterov_iterations"], "coord_err_dbu": {"median": float(np.median(d)), "p99": float(np.quantile(d, 0.99)), "max": float(d.max())}}
    return out


def cpu_sample(a):
    """The oracle (the reference's CPU path restated; one thread, as the reference runs) on the
    same workload as the device's timed loop: the same design, start and arguments, the same
    warm-up iterations untimed, then the same K iterations timed, or the first of them that
    end within --cpu-seconds (a bounded sample). The reference arm and the GPU line's
    cpu_baseline are this one sample."""
    import oracle
    design, args = loop_design(a)
    t0 = time.perf_counter()
    s = oracle.Session(design, args)
    setup = time.perf_counter() - t0
    s.iterate(a.warmup)
    tr0 = s.trials()
    # a bounded sample: the K iterations, or as many of them as end within --cpu-seconds
    t0 = time.perf_counter()
    done = 0
    while done < a.steps:
        k = s.iterate(1)
        done += k
        if k == 0 or time.perf_counter() - t0 > a.cpu_seconds:
            break
    dt = time.perf_counter() - t0
    trials = s.trials() - tr0
    s.discard()
    v = done / dt if dt > 0 else 0.0
    return {"value": v, "unit": "iters/s", "cores": 1, "kind": "port", "trials": trials, "trials_per_s": trials / dt if dt > 0 else 0.0,
            "seconds_per_iter": dt / max(done, 1), "seconds": dt,
            "sample": f"Nesterov iterations {a.warmup + 1}..{a.warmup + done} ({trials} trials) of the same design from {START[a.start]}, after {a.warmup} untimed warm-up iterations and the set-up ({setup:.1f} s); one host thread (the reference is single-threaded)"}


def reference(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    design, _ = loop_design(a)
    cpu = cpu_sample(a)
    v = cpu["value"]
    out = {"metric": METRIC, "value": v, "unit": "iters/s", "impl": "reference", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": 1000.0 * cpu["seconds_per_iter"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 (the reference's float order), f64 where the reference uses double", "data": "synthetic",
           "config": workload(a, design), "trials": cpu["trials"], "trials_per_s": cpu["trials_per_s"], "cpu_baseline": cpu,
           "e2e": {"value": v, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="cfg3", choices=list(CONFIGS))
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=30.0, help="the CPU sample's bound: the timed iterations end once they have taken this long")
    ap.add_argument("--no-precision-runs", action="store_true", help="skip the three whole commands (mixed, FP32, FP64 density solves) of the precision report")
    ap.add_argument("--form", default="mixed", choices=["mixed", "fp32"], help="the density solve timed as the headline")
    ap.add_argument("--start", default="spread", choices=["spread", "ip"],
                    help="time the loop from the generator's spread placement with the initial placement skipped (both arms, the default), or after the device's initial placement (a profiling case)")
    ap.add_argument("--initial-place-only", action="store_true",
                    help="run the command through the initial placement once and print its time (a profiling case)")
    ap.add_argument("--save-placement", default="", help="with --initial-place-only: save the locations (.npy)")
    ap.add_argument("--start-from", default="", help="start the loop from saved initial-placement locations (a profiling case)")
    ap.add_argument("--reorder", default="1", choices=["0", "1"], help="keep the device's cell order coherent as cells move (the default) or as uploaded")
    a = ap.parse_args()
    if a.warmup < 3:
        a.warmup = 3
    if a.impl == "reference":
        reference(a)
    else:
        ours(a)


if __name__ == "__main__":
    main()
