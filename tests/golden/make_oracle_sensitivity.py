"""Writes tests/golden/oracle_sensitivity.json: the oracle's initial placement of the 2.4M-cell,
48-group design (cfg4) with its BiCGSTAB inner products summed in double and rounded once
(ORACLE_SUM_DOUBLE=1) instead of in float in Eigen's packet order, the reference's. Against the
oracle's own recorded run (tests/golden/oracle_runs.json, cfg4) it measures how far the rounding
of the inner products alone moves the rounds where the solves stop far from converged; the
engine's inner products are doubles, so this bounds what its cfg4 parity can be held to.
About half an hour of one CPU thread. Run from the repository root:

    python tests/golden/make_oracle_sensitivity.py
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
os.environ["ORACLE_SUM_DOUBLE"] = "1"  # read once, at the oracle's first inner product

import oracle  # noqa: E402
from gpl_b200 import synth  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_sensitivity.json")

if __name__ == "__main__":
    design = synth.generate("cfg4")
    t0 = time.time()
    res = oracle.global_placement(design, ["-density", "0.70", "-skip_nesterov_place"])
    rows = [l for l in res["lines"] if l.startswith("[InitialPlace]")]
    json.dump({"config": "cfg4", "inner_products": "double, rounded once", "initial_place": rows, "seconds": time.time() - t0}, open(OUT, "w"), indent=1)
    print("wrote", OUT)
