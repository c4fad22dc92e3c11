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


def _ip_rows(lines):
    rows = []
    for l in lines:
        if l.startswith("[InitialPlace]"):
            parts = l.split()
            rows.append((int(parts[2]), float(parts[6]), int(parts[8])))
    return rows


def test_initial_place_rounds_match_the_oracle(cfg1):
    d, _ = cfg1
    ref = oracle.global_placement(d, ARGS + ["-skip_nesterov_place"])
    got = engine.global_placement(d, ARGS + ["-skip_nesterov_place"])
    a, b = _ip_rows(got["lines"]), _ip_rows(ref["lines"])
    assert len(a) == len(b) and len(a) >= 5
    # round 1's HPWL reads the design's boxes only: exact; later rounds follow solves whose dot
    # products are FP64 on the device (the oracle keeps the reference's f32 packet order)
    assert a[0][2] == b[0][2]
    for (ia, ra, ha), (ib, rb, hb) in zip(a, b):
        assert ia == ib
        assert abs(ha - hb) <= 1e-3 * hb


def test_initial_place_spmv_forms_agree(cfg1, monkeypatch):
    """The initial placement with each SpMV form forced (GPL_SPMV_FORM: a thread per row,
    block-staged, sliced): the solves' products are the same bit for bit in every form, so the
    placed locations and every report line are identical."""
    d, _ = cfg1
    runs = []
    for form in ("0", "1", "2"):
        monkeypatch.setenv("GPL_SPMV_FORM", form)
        runs.append(engine.global_placement(d, ARGS + ["-skip_nesterov_place"]))
    for r in runs[1:]:
        assert np.array_equal(r["locations"], runs[0]["locations"])
        assert r["lines"] == runs[0]["lines"]


def test_initial_place_row_order_keeps_the_rounds(monkeypatch):
    """The solver's row order (each round's systems renumbered by the Hilbert index of the
    rows' centres, entries kept in their own order, so every row product is unchanged) against
    the rows as built (GPL_IP_ORDER=0), on the 100k-cell design: only the inner products see
    their terms in another order, so every round's HPWL agrees within 1e-5 and the placed
    centres within 1e-5 of the core's side."""
    d = synth.generate("cfg2")
    args = ["-density", "0.70", "-bin_grid_count", "512", "-skip_nesterov_place"]
    runs = {}
    for on in ("1", "0"):
        monkeypatch.setenv("GPL_IP_ORDER", on)
        runs[on] = engine.global_placement(d, args)
    a, b = _ip_rows(runs["1"]["lines"]), _ip_rows(runs["0"]["lines"])
    assert len(a) == len(b) and a[0] == b[0]
    for (ia, ra, ha), (ib, rb, hb) in zip(a, b):
        assert ia == ib
        assert abs(ha - hb) <= 1e-5 * hb
    la, lb = runs["1"]["locations"], runs["0"]["locations"]
    assert np.array_equal(la[:, 0], lb[:, 0])
    side = max(d.core[2] - d.core[0], d.core[3] - d.core[1])
    assert np.abs(la[:, 1:].astype(np.int64) - lb[:, 1:].astype(np.int64)).max() <= 1e-5 * side


def _lines_with(lines, code):
    return [l for l in lines if f"GPL-{code}]" in l]


def test_routability_driven_matches_the_oracle(cfg1):
    """-routability_driven with the synthetic router (one wide routing pitch, so the RUDY map
    overflows and the pass inflates cells, cuts fillers and reverts to its snapshot several
    times). The trajectories part after the first reordered sum, so the comparison is of the
    course, not of bits: the snapshot within 10 iterations, the same number of passes (+-1),
    both ending placed under the overflow target, final HPWL within 5 % and the final
    placement area (cells as inflated) within 1 %."""
    d, _ = cfg1
    args = ARGS + ["-routability_driven"]
    rt = engine.SyntheticRouter(d, 3000, pitches=(1200,))
    ref = oracle.global_placement(d, args, router=rt.ptr)
    got = engine.global_placement(d, args, router=rt)
    assert ref["status"] == "placed" and got["status"] == "placed", got["reason"]
    snap = lambda r: int(_lines_with(r["lines"], "0038")[0].split("=")[-1])
    assert abs(snap(got) - snap(ref)) <= 10
    assert abs(len(_lines_with(got["lines"], "0040")) - len(_lines_with(ref["lines"], "0040"))) <= 1
    assert len(_lines_with(got["lines"], "0040")) >= 2
    assert got["final_overflow"] <= 0.1
    assert abs(got["final_hpwl"] - ref["final_hpwl"]) <= 0.05 * ref["final_hpwl"]
    area = lambda r: float(_lines_with(r["lines"], "1014")[0].split(":")[1].split("(")[0])
    assert abs(area(got) - area(ref)) <= 0.01 * area(ref)


def test_region_groups_match_the_oracle():
    """Four region groups beside the top level (five Nesterov regions, each with its own bin
    grid, sharing the WA coefficient and the back-tracking): identical construction lines,
    every region finishing within 10 iterations of the oracle's, final HPWL within 0.1 % and
    overflow within 0.005."""
    d = synth.generate("cfg4s")
    args = ["-density", "0.70"]
    ref = oracle.global_placement(d, args)
    got = engine.global_placement(d, args)
    assert got["status"] == "placed", got["reason"]
    assert header(got["lines"]) == header(ref["lines"])
    assert got["bases"] == ref["bases"]
    fin = lambda r: {l.split("'")[1] if "'" in l else "top": int(l.split()[-1]) for l in r["lines"] if "GPL-1016]" in l or "GPL-1001]" in l}
    a, b = fin(got), fin(ref)
    assert a.keys() == b.keys() and len(a) == 5
    for k in a:
        assert abs(a[k] - b[k]) <= 10, (k, a[k], b[k])
    assert abs(got["final_hpwl"] - ref["final_hpwl"]) <= 1e-3 * ref["final_hpwl"]
    assert abs(got["final_overflow"] - ref["final_overflow"]) <= 0.005


def _run_packed(d, args, packed):
    p = engine.Placer(0)
    try:
        p.set_option("packed", packed)
        return p.global_placement(d, args)
    finally:
        p.close()


@pytest.mark.parametrize("cfg,over", [("cfg4s", {}), ("cfg4", dict(cells=120_000, nets=126_000, region_cells=(48, 300, 8_000)))])
def test_packed_launches_give_the_same_run(cfg, over):
    """Every region's scatter, bin finalize, FP32 density solve and gradient update as one
    launch per phase (the default with regions) against one launch per region: each region's
    blocks do what its own launch's would, so the runs are identical bit for bit (report lines,
    iterations, final HPWL and overflow, written placement). The second design has 48 uneven
    region groups beside the top level (bin grids from 16 to 128 a side)."""
    d = synth.generate(cfg, **over)
    args = ["-density", "0.70"]
    a = _run_packed(d, args, "1")
    b = _run_packed(d, args, "0")
    assert a["status"] == b["status"] == "placed", (a["reason"], b["reason"])
    assert a["lines"] == b["lines"]
    assert a["nesterov_iterations"] == b["nesterov_iterations"]
    assert a["final_hpwl"] == b["final_hpwl"] and a["final_overflow"] == b["final_overflow"]
    assert np.array_equal(a["locations"], b["locations"])
    assert a["launches"] < b["launches"]


DIVERGE = ("GPL-0323", "GPL-0324", "GPL-0998", "GPL-0997", "GPL-0307")


def _divergence_course(lines):
    return [c for l in lines for c in DIVERGE if c in l]


def test_divergence_revert_takes_the_oracles_course(cfg1):
    """An overflow target the design cannot reach (0.03) runs the loop on until it diverges
    (`check_divergence`, src/nesterov.rs:2976-2991): the oracle then reverts to the minimum-HPWL
    snapshot and resumes twice (GPL-0998) and reverts and stops the third time (GPL-0997,
    :3009-3052, :4406-4414). The engine must take the same course on the device's snapshots,
    and end at a minimum-HPWL state close to the oracle's. (Such a run is chaotic after the
    first reverts: with -max_phi_coef 1.05 and -init_density_penalty 8e-5 the engine's run
    diverged differently and stopped with an error status, so only this course is asserted.)"""
    d, _ = cfg1
    args = ARGS + ["-max_phi_coef", "1.15", "-init_density_penalty", "0.001", "-overflow", "0.03"]
    ref = oracle.global_placement(d, args)
    got = engine.global_placement(d, args)
    course = _divergence_course(ref["lines"])
    assert course[-1] == "GPL-0997" and course.count("GPL-0998") == 2  # the oracle's course, as recorded
    assert got["status"] == ref["status"] == "placed", got["reason"]
    print("divergence course", _divergence_course(got["lines"]), course, "iterations", got["nesterov_iterations"], ref["nesterov_iterations"],
          "hpwl", got["final_hpwl"], ref["final_hpwl"], "overflow", got["final_overflow"], ref["final_overflow"])
    assert _divergence_course(got["lines"]) == course
    # the "(k of 3 reverts allowed)" counts, in order
    reverts = lambda r: [l.split("(")[1] for l in r["lines"] if "GPL-0998" in l]
    assert reverts(got) == reverts(ref)
    assert abs(got["final_hpwl"] - ref["final_hpwl"]) <= 0.02 * ref["final_hpwl"]
    assert abs(got["final_overflow"] - ref["final_overflow"]) <= 0.01
