"""Writes tests/golden/oracle_runs.json: the oracle's whole `global_placement` run on the
100k-cell, 1M-cell and 2.4M-cell (48 region groups) synthetic designs, summarised (the report's construction lines, the
`[InitialPlace]` rows, the iteration count, final HPWL and overflow, and a checksum of the
written placement).

These runs take minutes (100k cells) to about an hour (1M cells) on one CPU thread, so the
GPU tests compare against this summary instead of re-running the oracle. Run from the
repository root:

    python tests/golden/make_oracle_runs.py [cfg2] [cfg3] [cfg2_route] [cfg4]
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from gpl_b200 import synth  # noqa: E402

ARGS = {
    "cfg2": ["-density", "0.70", "-bin_grid_count", "512"],
    "cfg3": ["-density", "0.70", "-bin_grid_count", "1024"],
    # routability-driven, with the synthetic router: 3000-DBU tiles, one 1200-DBU pitch (so the
    # RUDY map overflows and the passes inflate cells), capacity 20
    "cfg2_route": ["-density", "0.70", "-bin_grid_count", "512", "-routability_driven"],
    # 48 uneven region groups and the top level, each with the bin grid the placer's rule gives
    "cfg4": ["-density", "0.70"],
}
ROUTER = {"cfg2_route": dict(tile=3000, pitches=(1200,), capacity=20)}
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_runs.json")


def _codes(lines, code):
    return [l for l in lines if f"GPL-{code}]" in l]


def summarise(cfg, res, seconds):
    lines = res["lines"]
    header = []
    for l in lines:
        if l.startswith("[InitialPlace]"):
            break
        header.append(l)
    loc = res["locations"]
    return {
        "config": cfg, "args": ARGS[cfg], "status": res["status"],
        "insts": res["insts"], "nets": res["nets"], "pins": res["pins"],
        "header": header,
        "initial_place": [l for l in lines if l.startswith("[InitialPlace]")],
        "nesterov_iterations": res["nesterov_iterations"],
        "final_hpwl": res["final_hpwl"], "final_overflow": res["final_overflow"],
        "locations": int(len(loc)),
        "location_sums": [int(loc[:, 1].astype("int64").sum()), int(loc[:, 2].astype("int64").sum())] if len(loc) else [0, 0],
        "seconds": seconds,
        # the routability passes: the snapshot line, each pass's line, the final area line
        "route": {"snapshot": _codes(lines, "0038"), "passes": _codes(lines, "0040"), "area": _codes(lines, "1014"),
                  "recovery": _codes(lines, "0112")},
    }


def main(cfgs):
    out = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for cfg in cfgs:
        d = synth.generate(cfg.split("_")[0])
        router = None
        if cfg in ROUTER:
            from gpl_b200 import engine  # the synthetic router only (host code, no device)
            rt = ROUTER[cfg]
            router = engine.SyntheticRouter(d, rt["tile"], pitches=rt["pitches"], capacity=rt["capacity"])
        t0 = time.perf_counter()
        res = oracle.global_placement(d, ARGS[cfg], router=router.ptr if router else None)
        out[cfg] = summarise(cfg, res, time.perf_counter() - t0)
        print(cfg, out[cfg]["status"], out[cfg]["nesterov_iterations"], out[cfg]["final_hpwl"], out[cfg]["final_overflow"], flush=True)
        # merged into the file as it is now (another configuration may have been written since)
        now = json.load(open(OUT)) if os.path.exists(OUT) else {}
        now[cfg] = out[cfg]
        with open(OUT, "w") as f:
            json.dump(now, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1:] or ["cfg2"])
