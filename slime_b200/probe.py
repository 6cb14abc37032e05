"""Small, fixed workloads that each run one kernel family once, for profiling and timing.

    python -m slime_b200.probe <case> [--repeat N]

Each case runs its workload `repeat` times (default 2: one warm-up, one to capture) through the C
ABI and prints one JSON line with the event-timed kernel milliseconds of the last run where the
library reports them. Cases (sizes chosen so that one launch holds a few GB at most and takes well
under a second):

  general40   general_scan_kernel: the 4,001^2 threshold-40 search about (0, 0)
  exact40     band_scan_kernel, independent bands with bit-sliced exact counts: radius 100,000,
              threshold 40
  band60      band_scan_kernel, shared LCG: radius 600,000 (9+ periods), threshold 60
  grouped60   band_scan_kernel, grouped bands: radius 200,000 (3 periods: 4 groups x 4 copies),
              threshold 60
  world60     band_scan_kernel, shared LCG: the full-world threshold-60 scan (36 launches of ~60 ms,
              under 1 GB on the device); profile one launch of it (`-c 1`)
  precise     precise_kernel: precise AFK scores of the best 20,000 sites of a threshold-36 search
  biome       biome chunk_kernel: the Deep Dark / Mushroom Fields filter of 4,096 threshold-48
              sites (version 26.2)
"""
from __future__ import annotations

import argparse
import json
import time

SEED = -6166315385447640203


def run(case: str, repeat: int) -> dict:
    from slime_b200 import build
    from slime_b200.lib import BiomeFilter, SlimeCoreB200
    build.build()
    core = SlimeCoreB200()
    core.set_y_scan_config(0, -64, -64, 64, 4)
    out = {"case": case}
    for _ in range(repeat):
        core.lib.reset_cancel()
        t0 = time.perf_counter()
        if case == "general40":
            core.lib.slime_b200_set_engine(1, 0)
            total, _ = core.search(SEED, 2000, 40, 221, 0, 0, 0, 100_000)
            out.update(total=int(total), kernel_ms=core.last_search_stats()[0])
        elif case == "exact40":
            core.lib.slime_b200_set_engine(5, 0)
            total, _ = core.search(SEED, 100_000, 40, 221, 0, 0, 0, 1000)
            out.update(total=int(total), kernel_ms=core.last_search_stats()[0],
                       T_centres_per_s=(2 * 100_000 + 1) ** 2 / core.last_search_stats()[0] / 1e9)
        elif case == "band60":
            core.lib.slime_b200_set_engine(2, 0)
            total, _ = core.search(SEED, 600_000, 60, 221, 0, 0, 0, 1000)
            out.update(total=int(total), kernel_ms=core.last_search_stats()[0],
                       T_centres_per_s=(2 * 600_000 + 1) ** 2 / core.last_search_stats()[0] / 1e9)
        elif case == "grouped60":
            core.lib.slime_b200_set_engine(6, 0)
            total, _ = core.search(SEED, 200_000, 60, 221, 0, 0, 0, 1000)
            out.update(total=int(total), kernel_ms=core.last_search_stats()[0],
                       T_centres_per_s=(2 * 200_000 + 1) ** 2 / core.last_search_stats()[0] / 1e9)
        elif case == "world60":
            from slime_b200 import workloads
            spec = workloads.full_world_scan()
            core.lib.slime_b200_set_engine(2, 0)
            total, _ = core.search(spec.seed, spec.radius, 60, 221, 0, 0, 0, 1000)
            out.update(total=int(total), kernel_ms=core.last_search_stats()[0],
                       T_centres_per_s=(2 * spec.radius + 1) ** 2 / core.last_search_stats()[0] / 1e9)
        elif case == "precise":
            core.lib.slime_b200_set_engine(0, 0)
            _, sites = core.search(SEED, 20_000, 36, 221, 0, 0, 0, 20_000)
            t0 = time.perf_counter()
            scored = core.score_precise(SEED, sites, 1)
            out.update(sites=len(scored), best_obs=int(scored["obs_count"].max()))
        elif case == "biome":
            core.lib.slime_b200_set_engine(0, 0)
            _, sites = core.search(SEED, 300_000, 48, 221, 0, 0, 0, 4096)
            cx = (sites["center_x"] - 8) // 16
            cz = (sites["center_z"] - 8) // 16
            t0 = time.perf_counter()
            with BiomeFilter(2602, SEED, len(cx), core=core) as f:
                mask = f.filter(cx, cz, 3)
                kms, unique = f.last_stats()
            out.update(candidates=len(cx), excluded=int((mask != 0).sum()), unique_chunks=int(unique),
                       kernel_ms=kms)
        else:
            raise SystemExit(f"unknown case {case}")
        out["wall_ms"] = (time.perf_counter() - t0) * 1e3
    core.lib.slime_b200_set_engine(0, 0)
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("case", choices=["general40", "exact40", "band60", "grouped60", "world60", "precise", "biome"])
    ap.add_argument("--repeat", type=int, default=2)
    a = ap.parse_args()
    print(json.dumps(run(a.case, a.repeat)))


if __name__ == "__main__":
    main()
