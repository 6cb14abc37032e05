"""Measure the engine crossovers of the slime-chunk search on the local GPU and write the rule.

    python -m slime_b200.autotune [--out slime_b200/tuning_b200.json] [--quick]

For each (radius, threshold) point of a grid the search is timed with every engine that applies
(the general scan, independent bands, grouped bands where the area spans a period, and the
shared-LCG band engine where it spans two, the shared-LCG and independent-band engines also with
bit-sliced exact counts at low thresholds), forced through slime_b200_set_engine; every engine
must return the same total and the same ranked sites. From the timings it derives the eleven
numbers of slime_b200_set_engine_rule:

  band_min_threshold, band_min_periods   shared LCG from this threshold on areas this many
  band_fast_threshold, band_fast_periods 2^17-chunk periods wide (two branches of the rule)
  indep_min_threshold, indep_min_centres independent bands instead of the general scan
  exact_below_threshold, exact_min_centres  exact counts below this threshold on areas this large
  grouped_min_threshold, grouped_min_width, grouped_max_width
                                         grouped bands from this threshold on areas this wide
  exact_wide_below_threshold             exact counts below this threshold on areas 4+ periods wide

and writes them with the raw timings to a JSON file. SlimeCoreB200 applies that file when it
loads the library. The general scan's rate does not depend on the area once it fills the GPU, so
it is timed on the smaller areas only and extrapolated to the larger ones.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time
from pathlib import Path

import numpy as np

PERIOD = 1 << 17
DEFAULT_OUT = Path(__file__).with_name("tuning_b200.json")
SEED = 0x5EED_B200  # any world seed: rates do not depend on it


def _time(core, mode, radius, thr, reps=2):
    core.lib.slime_b200_set_engine(mode, 0)
    best, out = None, None
    for _ in range(reps):
        core.lib.reset_cancel()
        t = time.perf_counter()
        out = core.search(SEED, radius, thr, 221, 0, 0, 0, 200)
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    return best, out


GROUPED_MAX_PERIODS = 16  # grouped bands hold at most 16 period copies
GROUPED_EXACT_MIN_PERIODS = 4  # the library's width from which exact counts may run as grouped bands
EXACT_MAX_THRESHOLD = 50  # the exact modes are timed up to here (their cost does not depend on it)


def measure(core, quick=False):
    radii = [10_000, 30_000, 100_000, 150_000, 200_000, 300_000, 600_000] + ([] if quick else [1_000_000])
    rows = []
    general_rate = {}
    for r in radii:
        w = 2 * r + 1
        for thr in range(40, 62, 4 if quick else 2):
            point = {"radius": r, "threshold": thr, "centres": w * w}
            ref = None
            engines = []
            if thr >= 42 or r <= 100_000:
                engines += [("indep", 3)] + ([("band", 2)] if w >= 2 * PERIOD else [])
                engines += [("grouped", 6)] if PERIOD < w <= GROUPED_MAX_PERIODS * PERIOD else []
            if thr <= EXACT_MAX_THRESHOLD:
                engines += [("indep_exact", 5)] + ([("band_exact", 4)] if w >= 2 * PERIOD else [])
                engines += [("grouped_exact", 7)] if PERIOD < w <= GROUPED_MAX_PERIODS * PERIOD else []
            if r <= 100_000:
                engines.insert(0, ("general", 1))
            for name, mode in engines:
                dt, out = _time(core, mode, r, thr, reps=1 if r >= 600_000 else 2)
                if ref is None:
                    ref = out
                elif out[0] != ref[0] or not np.array_equal(out[1], ref[1]):
                    raise RuntimeError(f"engines disagree at radius {r} threshold {thr}")
                point[name + "_s"] = dt
            if "general_s" in point:
                general_rate[thr] = point["centres"] / point["general_s"]
            else:
                point["general_s"] = point["centres"] / general_rate.get(thr, min(general_rate.values()))
            for k in ("indep", "band", "grouped"):  # bounded engines below 42 on large areas: never chosen
                if k + "_s" not in point and (k == "indep" or (k == "band" and w >= 2 * PERIOD) or
                                              (k == "grouped" and PERIOD < w <= GROUPED_MAX_PERIODS * PERIOD)):
                    point[k + "_s"] = float("inf")
            rows.append(point)
    core.lib.slime_b200_set_engine(0, 0)
    return rows


def derive(rows):
    """The rule numbers from the timings. Independent bands take a threshold when they beat
    the general scan there and at every higher measured threshold of the area. The two
    shared-LCG branches are chosen among the measured (threshold, periods) crossovers as the pair
    whose rule costs least over the whole grid (sum of each point's time over its best time), and
    the grouped-band branch (threshold, width range) is chosen the same way among the measured
    thresholds and widths."""
    def min_winning_thr(pts, a, b):
        pts = sorted(pts, key=lambda p: p["threshold"])
        best = 222
        for p in reversed(pts):
            if a in p and b in p and p[a] < p[b]:
                best = p["threshold"]
            else:
                break
        return best

    by_r = {}
    for p in rows:
        by_r.setdefault(p["radius"], []).append(p)
    indep_thr = {r: min_winning_thr(pts, "indep_s", "general_s") for r, pts in by_r.items()}
    indep_min_threshold = max(indep_thr.values())
    wins = [r for r, t in indep_thr.items() if t <= indep_min_threshold]
    indep_min_centres = (2 * min(wins) + 1) ** 2 if wins else 1 << 62
    band_thr = {r: min_winning_thr(pts, "band_s", "indep_s") for r, pts in by_r.items()
                if any("band_s" in p for p in pts)}
    cands = sorted({(t, (2 * r + 1) // PERIOD) for r, t in band_thr.items()} | {(222, 64)})
    widths = sorted({2 * p["radius"] + 1 for p in rows if "grouped_s" in p})
    g_cands = [(t, lo, hi) for t in sorted({p["threshold"] for p in rows} | {222})
               for lo in widths for hi in widths if lo <= hi] or [(222, 1 << 40, 0)]

    def cost(a, b, g):
        total = 0.0
        for p in rows:
            w = 2 * p["radius"] + 1
            best = min(p[k] for k in ("general_s", "indep_s", "band_s", "grouped_s") if k in p)
            thr = p["threshold"]
            if "grouped_s" in p and thr >= g[0] and g[1] <= w <= g[2]:
                t_rule = p["grouped_s"]
            elif "band_s" in p and any(thr >= t and w >= n * PERIOD for t, n in (a, b)):
                t_rule = p["band_s"]
            elif w * w >= indep_min_centres and thr >= indep_min_threshold:
                t_rule = p["indep_s"]
            else:
                t_rule = p["general_s"]
            total += t_rule / best
        return total

    # Coordinate descent: the shared-LCG pair without grouped bands, the grouped triple given the
    # pair, then the pair again given the triple.
    g = (222, 1 << 40, 0)
    a, b = min(((x, y) for x in cands for y in cands), key=lambda ab: cost(*ab, g))
    g = min(g_cands, key=lambda gg: cost(a, b, gg))
    a, b = min(((x, y) for x in cands for y in cands), key=lambda ab: cost(*ab, g))
    return ([a[0], max(2, a[1]), b[0], max(2, b[1]), indep_min_threshold, indep_min_centres] + derive_exact(rows)
            + [g[0], g[1], g[2], derive_exact_wide(rows)])


def derive_exact(rows):
    """exact_below_threshold: the exact modes take every threshold below it on the areas where
    they win -- one above the highest threshold at which the best exact mode still beats every
    other engine on all areas of at least exact_min_centres centres, the smallest measured area
    where it wins at the lowest threshold."""
    def exact_best(p):
        return min(p[k] for k in ("indep_exact_s", "band_exact_s", "grouped_exact_s") if k in p)

    def other_best(p):
        return min(p[k] for k in ("general_s", "indep_s", "band_s", "grouped_s") if k in p)

    pts = [p for p in rows if "indep_exact_s" in p]
    if not pts:
        return [0, 1 << 62]
    lowest = min(p["threshold"] for p in pts)
    winners = sorted(p["centres"] for p in pts if p["threshold"] == lowest and exact_best(p) < other_best(p))
    if not winners:
        return [0, 1 << 62]
    min_centres = winners[0]
    below = 0
    for thr in sorted({p["threshold"] for p in pts}):
        big = [p for p in pts if p["threshold"] == thr and p["centres"] >= min_centres]
        if big and all(exact_best(p) < other_best(p) for p in big):
            below = thr + 1
        else:
            break
    return [below, min_centres]


def derive_exact_wide(rows):
    """exact_wide_below_threshold: one above the highest threshold up to which the best exact mode
    beats every other engine on every measured area at least GROUPED_EXACT_MIN_PERIODS wide."""
    def exact_best(p):
        return min(p[k] for k in ("indep_exact_s", "band_exact_s", "grouped_exact_s") if k in p)

    def other_best(p):
        return min(p[k] for k in ("general_s", "indep_s", "band_s", "grouped_s") if k in p)

    pts = [p for p in rows if "indep_exact_s" in p and 2 * p["radius"] + 1 >= GROUPED_EXACT_MIN_PERIODS * PERIOD]
    below = 0
    for thr in sorted({p["threshold"] for p in pts}):
        at = [p for p in pts if p["threshold"] == thr]
        if all(exact_best(p) < other_best(p) for p in at):
            below = thr + 1
        else:
            break
    return below


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(DEFAULT_OUT))
    ap.add_argument("--quick", action="store_true", help="coarser grid (threshold step 4, no 1M radius)")
    ap.add_argument("--rederive", action="store_true", help="recompute the rule from the file's timings")
    args = ap.parse_args()
    from slime_b200 import build
    from slime_b200.lib import SlimeCoreB200
    build.build()
    core = SlimeCoreB200(apply_tuning=False)
    name = ctypes.create_string_buffer(256)
    core.lib.get_cuda_device_name(name, 256)
    device = name.value.decode(errors="replace")
    if args.rederive:
        old = json.loads(Path(args.out).read_text())
        rows, device = old["points"], old.get("device", device)
    else:
        rows = measure(core, quick=args.quick)
    rule = derive(rows)
    doc = {"device": device,
           "rule": dict(zip(["band_min_threshold", "band_min_periods", "band_fast_threshold",
                             "band_fast_periods", "indep_min_threshold", "indep_min_centres",
                             "exact_below_threshold", "exact_min_centres", "grouped_min_threshold",
                             "grouped_min_width", "grouped_max_width", "exact_wide_below_threshold"], rule)),
           "seed": SEED, "max_results": 200, "points": rows}
    Path(args.out).write_text(json.dumps(doc, indent=1) + "\n")
    print(json.dumps(doc["rule"]))


if __name__ == "__main__":
    main()
