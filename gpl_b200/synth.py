"""Seeded synthetic netlists with the shapes of the benchmark configurations.

No design ships with the reference, so every run here reads a generated one. The rules (one
generator for every size):

* DBU 1000; rows 1.4 um (1400) high; one non-PAD site 0.19 um (190) wide; rows tile the core.
* Standard cells: one row high, widths uniform in [w_min, w_max] sites; unplaced (their
  database box at the origin), so initial placement starts them at the core centre. With
  `placed=True` each cell is instead placed at its latent position (the point the locality
  window is drawn around), snapped to the site/row grid inside the core: a spread start for
  runs that skip the initial placement (`-skip_initial_place`).
* Nets: degree 2 (55 %), 3 (20 %), 4 (10 %), else uniform 5..16 (with `max_degree` above 16,
  one net in a hundred is uniform 17..max_degree instead). Each net's terminals are cells drawn
  within a window of +-15 % of the core around an anchor (a cell, or the net's IO port);
  a terminal's pin is a 1x1 DBU shape uniform inside its cell.
* IO ports: fixed, evenly spaced on the die perimeter, one per net on the first nets.
* Macros: fixed BLOCK squares, sides drawn uniform 20..60 um and then scaled together so they
  cover the stated fraction of the core; non-overlapping, on the site/row grid.
* Core: the stated size, or square and sized for the stated utilisation
  (movable area / (core area - macro area)).
* Region groups (`regions=(kx, ky, k)`): the core is cut into kx x ky tiles on the site/row
  grid and the first k tiles (row by row) become regions, one group each; a cell joins the
  group whose tile holds its latent position, the rest stay top-level. No fixed instance
  then (a fixed instance against a region's boundary is outside the placer's model).
* Uneven region groups (`region_cells=(k, lo, hi)`): k cell counts drawn log-uniform in
  [lo, hi] (seeded; drawn again while they leave under 2 % of the cells to the top level),
  and the core cut into k + 1 boxes whose areas follow the counts (a squarified treemap on
  the site/row grid; the last box is the top level's). Since the latent positions are
  uniform, each region then holds about its drawn count.
"""
from __future__ import annotations

import numpy as np

from .design import (BTERM_FIXED, BTERM_PLACED, INST_BLOCK, INST_CORE_AUTO_PLACEABLE, INST_FIXED,
                     INST_PLACED, Design)

SITE_W = 190
ROW_H = 1400
DBU = 1000

PRESETS = {
    # 294 cells / 364 nets / 1122 pins in a 60 x 60 um core, 24 IO ports, no macro.
    "cfg1": dict(cells=294, nets=364, pins=1122, w_min=2, w_max=12, core_um=(60.0, 60.0), n_io=24,
                 macros=0, macro_frac=0.0, max_degree=16, seed=1),
    # 100k cells, ~105k nets, ~400k pins, 8 macros over 12 % of a core at 60 % utilisation.
    "cfg2": dict(cells=100_000, nets=105_000, w_min=2, w_max=24, util=0.60, n_io=256,
                 macros=8, macro_frac=0.12, max_degree=64, seed=2),
    # 1M cells, ~1.05M nets, ~4M pins, 32 macros over 15 % of the core.
    "cfg3": dict(cells=1_000_000, nets=1_050_000, w_min=2, w_max=24, util=0.60, n_io=256,
                 macros=32, macro_frac=0.15, max_degree=64, seed=3),
    # 4 region groups over a 3 x 2 grid of core tiles (2000 cells, no macro): the small
    # multi-region case the parity tests run on both sides.
    "cfg4s": dict(cells=2000, nets=2100, w_min=2, w_max=12, util=0.55, n_io=32,
                  macros=0, macro_frac=0.0, max_degree=16, seed=4, regions=(3, 2, 4)),
    # 48 region groups of uneven size (log-uniform 2k..200k cells) beside the top level, 2.4M
    # cells in all, no macro. The placer's own bin-count rule gives each region a grid of
    # 32..256 bins a side, rising with its count, and the top level 1024 x 1024.
    "cfg4": dict(cells=2_400_000, nets=2_520_000, w_min=2, w_max=24, util=0.60, n_io=256,
                 macros=0, macro_frac=0.0, max_degree=64, seed=4, region_cells=(48, 2_000, 200_000)),
    # 2M cells, ~2.1M nets, ~8M pins, as cfg3.
    "cfg5": dict(cells=2_000_000, nets=2_100_000, w_min=2, w_max=24, util=0.60, n_io=256,
                 macros=32, macro_frac=0.15, max_degree=64, seed=5),
}


def _degrees(rng, n, max_degree):
    u = rng.random(n)
    deg = np.where(u < 0.55, 2, np.where(u < 0.75, 3, np.where(u < 0.85, 4, 0)))
    rest = deg == 0
    deg[rest] = rng.integers(5, 17, rest.sum())
    if max_degree > 16:
        big = rest & (rng.random(n) < 1.0 / 15.0)
        deg[big] = rng.integers(17, max_degree + 1, big.sum())
    return deg.astype(np.int64)


def _fit_total(rng, deg, total, lo=2, hi=16):
    """Nudge degrees one at a time (seeded) until they sum to `total`."""
    deg = deg.copy()
    while deg.sum() > total:
        cand = np.flatnonzero(deg > lo)
        deg[cand[rng.integers(len(cand))]] -= 1
    while deg.sum() < total:
        cand = np.flatnonzero(deg < hi)
        deg[cand[rng.integers(len(cand))]] += 1
    return deg


def _place_macros(rng, n, frac, core_w, core_h):
    if n == 0:
        return np.zeros((0, 4), np.int64)
    sides = rng.uniform(20.0, 60.0, n) * DBU
    scale = np.sqrt(frac * core_w * core_h / np.sum(sides ** 2))
    sides = sides * scale
    boxes = []
    gap = 2 * ROW_H
    for s in sorted(sides, reverse=True):
        w = max(SITE_W, int(round(s / SITE_W)) * SITE_W)
        h = max(ROW_H, int(round(s / ROW_H)) * ROW_H)
        for _ in range(20000):
            lx = int(rng.integers(0, max(1, (core_w - w) // SITE_W + 1))) * SITE_W
            ly = int(rng.integers(0, max(1, (core_h - h) // ROW_H + 1))) * ROW_H
            ok = all(lx >= bx1 + gap or lx + w + gap <= bx0 or ly >= by1 + gap or ly + h + gap <= by0
                     for bx0, by0, bx1, by1 in boxes)
            if ok:
                boxes.append((lx, ly, lx + w, ly + h))
                break
        else:
            raise RuntimeError("could not place the macros without overlap")
    return np.array(boxes, np.int64)


def _region_counts(rng, k, lo, hi, total):
    """k counts log-uniform in [lo, hi] that leave at least 2 % of `total` to the top level."""
    for _ in range(1000):
        c = np.exp(rng.uniform(np.log(lo), np.log(hi), k)).astype(np.int64)
        if c.sum() <= 0.98 * total:
            return c
    raise ValueError("region counts do not fit the cell total")


def _treemap_boxes(areas, box):
    """Boxes on the site/row grid whose areas follow `areas`: the squarified treemap (Bruls,
    Huizing and van Wijk, 2000). Items in falling area fill strips along the shorter side of
    the box still free, a strip taking items while that does not worsen its worst aspect
    ratio; each strip's cut and each item's edge inside a strip land on the site/row grid."""
    order = sorted(range(len(areas)), key=lambda i: -areas[i])
    out = [None] * len(areas)
    lx, ly, ux, uy = box
    left = float(sum(areas))

    def worst(row, side, scale):
        s = sum(row) * scale
        t = s / side  # the strip's thickness
        return max(max(t / (a * scale / t), (a * scale / t) / t) for a in row)

    k = 0
    while k < len(order):
        w, h = ux - lx, uy - ly
        scale = w * h / left  # area units per input unit
        side = min(w, h)
        row = [areas[order[k]]]
        while k + len(row) < len(order) and worst(row + [areas[order[k + len(row)]]], side, scale) <= worst(row, side, scale):
            row.append(areas[order[k + len(row)]])
        last = k + len(row) == len(order)
        frac = sum(row) / left
        items = order[k:k + len(row)]
        if w >= h:  # a vertical strip at the left
            x = ux if last else min(max(lx + int(round(w * frac / SITE_W)) * SITE_W, lx + SITE_W), ux - SITE_W)
            cum, y0 = 0.0, ly
            for n, i in enumerate(items):
                cum += areas[i]
                y1 = uy if n == len(items) - 1 else min(max(ly + int(round(h * cum / sum(row) / ROW_H)) * ROW_H, y0 + ROW_H), uy - ROW_H)
                out[i] = (lx, y0, x, y1)
                y0 = y1
            lx = x
        else:  # a horizontal strip at the bottom
            y = uy if last else min(max(ly + int(round(h * frac / ROW_H)) * ROW_H, ly + ROW_H), uy - ROW_H)
            cum, x0 = 0.0, lx
            for n, i in enumerate(items):
                cum += areas[i]
                x1 = ux if n == len(items) - 1 else min(max(lx + int(round(w * cum / sum(row) / SITE_W)) * SITE_W, x0 + SITE_W), ux - SITE_W)
                out[i] = (x0, ly, x1, y)
                x0 = x1
            ly = y
        left -= sum(row)
        k += len(row)
    return out


def generate(cfg="cfg1", **over) -> Design:
    """A seeded synthetic design: a preset name, optionally with parameters overridden."""
    p = dict(PRESETS[cfg]) if isinstance(cfg, str) else dict(cfg)
    placed = bool(over.pop("placed", False))
    p.update(over)
    rng = np.random.default_rng(p["seed"])
    m = int(p["cells"])
    w_sites = rng.integers(p["w_min"], p["w_max"] + 1, m)
    cw = w_sites.astype(np.int64) * SITE_W
    ch = np.full(m, ROW_H, np.int64)
    cell_area = float(np.sum(cw * ch))

    if "core_um" in p:
        die_w, die_h = int(p["core_um"][0] * DBU), int(p["core_um"][1] * DBU)
        core_w, core_h = die_w // SITE_W * SITE_W, die_h // ROW_H * ROW_H
    else:
        core_area = cell_area / (p["util"] * (1.0 - p["macro_frac"]))
        side = np.sqrt(core_area)
        core_w = int(round(side / SITE_W)) * SITE_W
        core_h = int(round(side / ROW_H)) * ROW_H
        die_w, die_h = core_w, core_h
    macros = _place_macros(rng, int(p["macros"]), float(p["macro_frac"]), core_w, core_h)

    # nets and their degrees (IO ports count toward the degree)
    n_nets = int(p["nets"])
    deg = _degrees(rng, n_nets, int(p["max_degree"]))
    if "pins" in p:
        deg = _fit_total(rng, deg, int(p["pins"]), 2, max(16, int(p["max_degree"])))
    n_io = min(int(p["n_io"]), n_nets)
    has_io = np.zeros(n_nets, bool)
    has_io[:n_io] = True
    n_iterm = deg - has_io
    n_iterm = np.maximum(n_iterm, 1)

    # IO ports evenly spaced on the die perimeter (a 140 x 140 box inside the die)
    perim = 2 * (die_w + die_h)
    t = (np.arange(n_io) + 0.5) * perim / max(n_io, 1)
    px = np.zeros(n_io, np.int64)
    py = np.zeros(n_io, np.int64)
    for k, s in enumerate(t):
        if s < die_w:
            px[k], py[k] = s, 0
        elif s < die_w + die_h:
            px[k], py[k] = die_w, s - die_w
        elif s < 2 * die_w + die_h:
            px[k], py[k] = die_w - (s - die_w - die_h), die_h
        else:
            px[k], py[k] = 0, die_h - (s - 2 * die_w - die_h)
    half = 70
    bx0 = np.clip(px - half, 0, die_w - 2 * half)
    by0 = np.clip(py - half, 0, die_h - 2 * half)
    bterm_box = np.stack([bx0, by0, bx0 + 2 * half, by0 + 2 * half], 1).astype(np.int32)

    # latent cell positions, bucketed for the locality window
    lat_x = rng.uniform(0, core_w, m)
    lat_y = rng.uniform(0, core_h, m)
    g = max(1, int(np.sqrt(m / 8)))
    bxi = np.minimum((lat_x / core_w * g).astype(np.int64), g - 1)
    byi = np.minimum((lat_y / core_h * g).astype(np.int64), g - 1)
    bucket = byi * g + bxi
    order = np.argsort(bucket, kind="stable")
    counts = np.bincount(bucket, minlength=g * g)
    bstart = np.concatenate([[0], np.cumsum(counts)])

    starts = np.concatenate([[0], np.cumsum(n_iterm)]).astype(np.int64)
    total = int(starts[-1])
    net_of = np.repeat(np.arange(n_nets), n_iterm)
    slot = np.arange(total) - starts[net_of]
    anchor_cell = rng.integers(0, m, n_nets)
    cxn = np.where(has_io, np.r_[px, np.zeros(n_nets - n_io)], lat_x[anchor_cell])
    cyn = np.where(has_io, np.r_[py, np.zeros(n_nets - n_io)], lat_y[anchor_cell])
    wx, wy = 0.15 * core_w, 0.15 * core_h

    def draw(idx):
        out = np.empty(len(idx), np.int64)
        todo = np.arange(len(idx))
        while len(todo):
            k = idx[todo]
            x = np.clip(cxn[net_of[k]] + rng.uniform(-wx, wx, len(k)), 0, core_w - 1e-6)
            y = np.clip(cyn[net_of[k]] + rng.uniform(-wy, wy, len(k)), 0, core_h - 1e-6)
            b = np.minimum((y / core_h * g).astype(np.int64), g - 1) * g + np.minimum((x / core_w * g).astype(np.int64), g - 1)
            c = counts[b]
            good = c > 0
            pick = bstart[b[good]] + (rng.random(good.sum()) * c[good]).astype(np.int64)
            out[todo[good]] = order[pick]
            todo = todo[~good]
        return out

    cell = draw(np.arange(total))
    first = (slot == 0) & ~has_io[net_of]
    cell[first] = anchor_cell[net_of[first]]
    for _ in range(50):  # a net does not hold one cell twice
        key = net_of * m + cell
        srt = np.argsort(key, kind="stable")
        dup = np.zeros(total, bool)
        dup[srt[1:]] = key[srt[1:]] == key[srt[:-1]]
        dup &= ~first
        if not dup.any():
            break
        idx = np.flatnonzero(dup)
        cell[idx] = draw(idx)

    # pin shapes: a 1x1 box uniform inside the cell, in master coordinates
    ox = (rng.random(total) * cw[cell]).astype(np.int64)
    oy = (rng.random(total) * ch[cell]).astype(np.int64)
    iterm_shape = np.stack([ox, oy, ox + 1, oy + 1], 1).astype(np.int32)

    n_mac = len(macros)
    n_inst = m + n_mac
    inst_box = np.zeros((n_inst, 4), np.int32)
    inst_box[:m, 2] = cw
    inst_box[:m, 3] = ch
    inst_box[m:] = macros
    inst_master = np.zeros((n_inst, 2), np.int32)
    inst_master[:m, 0] = cw
    inst_master[:m, 1] = ch
    inst_master[m:, 0] = macros[:, 2] - macros[:, 0] if n_mac else 0
    inst_master[m:, 1] = macros[:, 3] - macros[:, 1] if n_mac else 0
    inst_flags = np.full(n_inst, INST_CORE_AUTO_PLACEABLE, np.uint32)
    inst_flags[m:] |= INST_BLOCK | INST_FIXED | INST_PLACED
    if placed:
        llx = np.clip(np.round((lat_x - cw / 2) / SITE_W) * SITE_W, 0, core_w - cw).astype(np.int64)
        lly = np.clip(np.round((lat_y - ch / 2) / ROW_H) * ROW_H, 0, core_h - ch).astype(np.int64)
        inst_box[:m, 0], inst_box[:m, 1] = llx, lly
        inst_box[:m, 2], inst_box[:m, 3] = llx + cw, lly + ch
        inst_flags[:m] |= INST_PLACED

    n_rows = core_h // ROW_H
    row_box = np.zeros((n_rows, 4), np.int32)
    row_box[:, 1] = np.arange(n_rows) * ROW_H
    row_box[:, 2] = core_w
    row_box[:, 3] = row_box[:, 1] + ROW_H
    row_site = np.tile(np.array([SITE_W, ROW_H], np.int32), (n_rows, 1))

    groups = {}
    if p.get("region_cells"):
        k, lo, hi = p["region_cells"]
        if n_mac:
            raise ValueError("region groups and fixed macros do not mix")
        counts_r = _region_counts(np.random.default_rng([p["seed"], 1]), int(k), lo, hi, m)
        areas = np.r_[counts_r, m - counts_r.sum()].astype(np.float64)
        boxes = _treemap_boxes(areas, (0, 0, core_w, core_h))
        inst_group = np.full(n_inst, -1, np.int32)
        gi = np.full(m, -1, np.int64)
        for t, (x0, y0, x1, y1) in enumerate(boxes[:k]):
            gi[(lat_x >= x0) & (lat_x < x1) & (lat_y >= y0) & (lat_y < y1)] = t
        inst_group[:m] = gi
        groups = dict(
            inst_group=inst_group, group_names=[f"region{g}" for g in range(k)],
            group_region=np.arange(k, dtype=np.int32),
            region_bound_start=np.arange(k + 1, dtype=np.int32), region_bounds=np.array(boxes[:k], np.int32).reshape(k, 4),
            region_group_start=np.arange(k + 1, dtype=np.int32), region_groups=np.arange(k, dtype=np.int32))
    elif p.get("regions"):
        kx, ky, k = p["regions"]
        if n_mac:
            raise ValueError("region groups and fixed macros do not mix")
        xs = [int(round(core_w * i / kx / SITE_W)) * SITE_W for i in range(kx + 1)]
        ys = [int(round(core_h * j / ky / ROW_H)) * ROW_H for j in range(ky + 1)]
        boxes = [(xs[t % kx], ys[t // kx], xs[t % kx + 1], ys[t // kx + 1]) for t in range(k)]
        tx = np.minimum((lat_x * kx / core_w).astype(np.int64), kx - 1)
        ty = np.minimum((lat_y * ky / core_h).astype(np.int64), ky - 1)
        tile = ty * kx + tx
        inst_group = np.full(n_inst, -1, np.int32)
        inst_group[:m] = np.where(tile < k, tile, -1)
        groups = dict(
            inst_group=inst_group, group_names=[f"region{g}" for g in range(k)],
            group_region=np.arange(k, dtype=np.int32),
            region_bound_start=np.arange(k + 1, dtype=np.int32), region_bounds=np.array(boxes, np.int32).reshape(k, 4),
            region_group_start=np.arange(k + 1, dtype=np.int32), region_groups=np.arange(k, dtype=np.int32))

    bstart_n = np.concatenate([[0], np.cumsum(has_io.astype(np.int64))])
    return Design(
        dbu=DBU, die=(0, 0, die_w, die_h), core=(0, 0, core_w, core_h),
        row_box=row_box, row_site=row_site,
        inst_box=inst_box, inst_flags=inst_flags, inst_master=inst_master,
        net_iterm_start=starts, iterm_inst=cell.astype(np.int32), iterm_shape=iterm_shape,
        net_bterm_start=bstart_n.astype(np.int64), bterm_box=bterm_box,
        bterm_flags=np.full(n_io, BTERM_PLACED | BTERM_FIXED, np.uint8),
        meta=dict(config=cfg if isinstance(cfg, str) else "custom", params=p, placed=placed,
                  cells=m, macros=n_mac, nets=n_nets, pins=int(total + n_io)),
        **groups,
    )
