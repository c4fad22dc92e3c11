"""The whole command on the device against the oracle on the same synthetic design.

Tolerances: the report's construction lines are identical (integer work); the final HPWL is
within 0.1 % and the final overflow within 0.005 of the oracle's (the trajectories part after
the first reordered float sum, so only the end state is compared)."""
import numpy as np
import pytest

import oracle
from gpl_b200 import engine, synth

pytestmark = pytest.mark.gpu

ARGS = ["-density", "0.70", "-bin_grid_count", "64"]


@pytest.fixture(scope="module")
def cfg1():
    d = synth.generate("cfg1")
    return d, oracle.global_placement(d, ARGS)


def header(lines):
    out = []
    for l in lines:
        if l.startswith("[InitialPlace]"):
            break
        out.append(l)
    return out


@pytest.mark.parametrize("mode", ["fp32", "mixed"])
def test_cfg1_matches_the_oracle(cfg1, mode):
    d, ref = cfg1
    got = engine.global_placement(d, ARGS, poisson=mode)
    assert got["status"] == "placed", got["reason"]
    assert header(got["lines"]) == header(ref["lines"])
    assert (got["insts"], got["nets"], got["pins"]) == (ref["insts"], ref["nets"], ref["pins"])
    assert abs(got["final_hpwl"] - ref["final_hpwl"]) <= 1e-3 * ref["final_hpwl"]
    assert abs(got["final_overflow"] - ref["final_overflow"]) <= 0.005
    assert got["final_overflow"] <= 0.1
    assert len(got["locations"]) == len(ref["locations"])
    np.testing.assert_array_equal(got["locations"][:, 0], ref["locations"][:, 0])


def test_skip_nesterov_initial_placement_is_close(cfg1):
    d, _ = cfg1
    ref = oracle.global_placement(d, ARGS + ["-skip_nesterov_place"])
    got = engine.global_placement(d, ARGS + ["-skip_nesterov_place"])
    assert got["outcome"] == "initially_placed"
    a, b = got["locations"][:, 1:].astype(float), ref["locations"][:, 1:].astype(float)
    # per-coordinate: within 1e-5 of the core size (the coordinates are truncated integers)
    assert np.max(np.abs(a - b)) <= max(2.0, 1e-5 * 60000)
