"""CPU checks of the autotuner's rule derivation (slime_b200/autotune.py) on synthetic timings."""
from slime_b200.autotune import PERIOD, derive


def grid(indep_from, band_rule):
    rows = []
    for r in (30_000, 100_000, 300_000, 600_000, 1_000_000):
        w = 2 * r + 1
        for thr in range(40, 62, 2):
            p = {"radius": r, "threshold": thr, "centres": w * w, "general_s": 1.0,
                 "indep_s": 0.5 if thr >= indep_from else 2.0}
            if w >= 2 * PERIOD:
                p["band_s"] = 0.2 if band_rule(w // PERIOD, thr) else 0.9
            rows.append(p)
    return rows


def test_derive_recovers_the_crossovers():
    # Shared LCG wins from 48 on 9+ periods and from 54 on 4+ periods.
    rows = grid(44, lambda periods, thr: (periods >= 9 and thr >= 48) or (periods >= 4 and thr >= 54))
    band_thr, band_periods, fast_thr, fast_periods, indep_thr, indep_centres, ex_thr, ex_centres, *grp = derive(rows)
    assert grp[0] == 222  # no grouped timings: the grouped branch is off
    assert ex_thr == 0  # no exact timings: the exact modes are off
    assert indep_thr == 44 and indep_centres == (2 * 30_000 + 1) ** 2
    branches = {(band_thr, band_periods), (fast_thr, fast_periods)}
    assert branches == {(48, 9), (54, 4)}


def test_derive_never_picks_an_engine_that_loses_above_its_threshold():
    # Independent bands win at 46 and above except at 50: the rule must start above 50.
    rows = grid(46, lambda periods, thr: False)
    for p in rows:
        if p["threshold"] == 50:
            p["indep_s"] = 1.5
    assert derive(rows)[4] == 52


def test_derive_exact_modes():
    # Exact counts win below 46 on areas of 100k radius and more, and lose on the 30k area.
    rows = grid(44, lambda periods, thr: periods >= 9 and thr >= 48)
    for p in rows:
        if p["threshold"] <= 50:
            p["indep_exact_s"] = 0.1 if (p["threshold"] < 46 and p["radius"] >= 100_000) else 3.0
    rule = derive(rows)
    assert rule[6] == 45 and rule[7] == (2 * 100_000 + 1) ** 2  # wins at 44, loses at 46


def test_derive_grouped_bands():
    # Grouped bands win from threshold 50 on areas 1.5-6 periods wide (radius 100k..300k); the
    # shared LCG keeps the wider areas.
    rows = grid(44, lambda periods, thr: periods >= 4 and thr >= 48)
    for p in rows:
        w = 2 * p["radius"] + 1
        if PERIOD < w <= 16 * PERIOD:
            p["grouped_s"] = 0.1 if (p["threshold"] >= 50 and p["radius"] <= 300_000 and p["radius"] >= 100_000) else 5.0
    rule = derive(rows)
    assert rule[8:11] == [50, 2 * 100_000 + 1, 2 * 300_000 + 1]
    assert (rule[2], rule[3]) in {(48, 4), (48, 9)} or (rule[0], rule[1]) in {(48, 4), (48, 9)}


def test_derive_exact_wide():
    # Exact counts win below 46 on areas 4+ periods wide (radius 300k and up), below 42 elsewhere.
    rows = grid(40, lambda periods, thr: periods >= 9 and thr >= 48)
    for p in rows:
        if p["threshold"] <= 50:
            wide = 2 * p["radius"] + 1 >= 4 * PERIOD
            p["indep_exact_s"] = 0.1 if (p["threshold"] < (46 if wide else 42)) else 3.0
    rule = derive(rows)
    assert rule[11] == 45  # wins at 44, loses at the next measured threshold (46)
    assert rule[6] == 41
