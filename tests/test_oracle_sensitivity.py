"""The recorded sensitivity of the oracle's cfg4 initial placement to the rounding of its
inner products (tests/golden/oracle_sensitivity.json, written by make_oracle_sensitivity.py):
the same first round (the solves start from the same point), and later rounds that move by
about a percent. The cfg4 parity bounds (test_gpu_scale.py: rounds within 2 %) rest on it."""
import json
import os

import pytest

G = os.path.join(os.path.dirname(__file__), "golden")


def _hpwl(rows):
    return [int(r.split()[8]) for r in rows]


def test_inner_product_rounding_moves_the_cfg4_rounds_by_about_a_percent():
    p = os.path.join(G, "oracle_sensitivity.json")
    runs = json.load(open(os.path.join(G, "oracle_runs.json")))
    if not os.path.exists(p) or "cfg4" not in runs:
        pytest.skip("no recorded cfg4 sensitivity run")
    a, b = _hpwl(json.load(open(p))["initial_place"]), _hpwl(runs["cfg4"]["initial_place"])
    assert len(a) == len(b) == 20 and a[0] == b[0]
    dev = [abs(x - y) / y for x, y in zip(a, b)]
    assert 0.005 < max(dev) < 0.02
