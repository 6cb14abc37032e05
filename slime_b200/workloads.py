"""Seeded synthetic workloads for the slime-chunk cluster search.

Every draw comes from ``numpy.random.Generator(PCG64(cfg_seed))`` with a fixed per-workload seed,
so the tests, the bench and the fixtures all see the same inputs. Sizes follow the five search
shapes of the project: a plain 4,001^2 search, the full-world threshold-60 scan, a 64-seed mixed
batch, a 16-seed precise-score + biome pass and a 10,000-request served stream.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# World border: chunk centres in [-1,875,000, 1,875,000] on each axis (radius 1,875,000 about 0).
WORLD_RADIUS = 1_875_000

PLAIN_SEED = 1001
FULL_WORLD_SEED = 1002
BATCH_SEED = 1003
PRECISE_BIOME_SEED = 1004
SERVED_SEED = 1005


@dataclass(frozen=True)
class Search:
    seed: int
    center_x: int
    center_z: int
    radius: int
    min_size: int
    max_size: int = 221
    rd_min: int = 0
    max_results: int = 1000
    precise_afk: int = 0
    biome_flags: int = 0
    biome_version: int = 2602   # Minecraft 26.2, the version of the reference's biome data

    @property
    def centres(self) -> int:
        return (2 * self.radius + 1) ** 2


def _world_seed(rng: np.random.Generator) -> int:
    return int(rng.integers(-(2**63), 2**63, dtype=np.int64))


def plain_search() -> Search:
    """4,001 x 4,001 centres about (0,0), threshold 40."""
    rng = np.random.Generator(np.random.PCG64(PLAIN_SEED))
    return Search(seed=_world_seed(rng), center_x=0, center_z=0, radius=2000, min_size=40,
                  max_results=100_000)


def full_world_scan() -> Search:
    """Every chunk centre of the world (3,750,001^2 = 1.40625e13), threshold 60, top 1,000."""
    rng = np.random.Generator(np.random.PCG64(FULL_WORLD_SEED))
    return Search(seed=_world_seed(rng), center_x=0, center_z=0, radius=WORLD_RADIUS,
                  min_size=60, max_results=1000)


def batch_searches(n: int = 64) -> list[Search]:
    """64 seeds; centres uniform in +-1e6 chunks, radii log-uniform in [1e3, 2e5], thresholds
    uniform in [45, 60]."""
    rng = np.random.Generator(np.random.PCG64(BATCH_SEED))
    out = []
    for _ in range(n):
        seed = _world_seed(rng)
        cx = int(rng.integers(-1_000_000, 1_000_001))
        cz = int(rng.integers(-1_000_000, 1_000_001))
        radius = int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e5)))))
        thr = int(rng.integers(45, 61))
        out.append(Search(seed=seed, center_x=cx, center_z=cz, radius=radius, min_size=thr))
    return out


def precise_biome_seeds(n: int = 16) -> list[Search]:
    """16 full-world threshold-50 scans, precise scoring and biome exclusion (flags 3)."""
    rng = np.random.Generator(np.random.PCG64(PRECISE_BIOME_SEED))
    return [Search(seed=_world_seed(rng), center_x=0, center_z=0, radius=WORLD_RADIUS,
                   min_size=50, max_results=500, precise_afk=1, biome_flags=3)
            for _ in range(n)]


def served_stream(n: int = 10_000, rate_per_s: float = 1.0):
    """Request stream: (arrival_s, Search). Centres uniform in +-1.8e6, radii log-uniform in
    [100, 1,875,000], thresholds uniform in [40, 65], biome filter with probability 0.25.
    The arrival rate is a parameter: the server bench sets it to 0.8x the measured capacity."""
    rng = np.random.Generator(np.random.PCG64(SERVED_SEED))
    t = 0.0
    out = []
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate_per_s))
        seed = _world_seed(rng)
        cx = int(rng.integers(-1_800_000, 1_800_001))
        cz = int(rng.integers(-1_800_000, 1_800_001))
        radius = int(round(math.exp(rng.uniform(math.log(100), math.log(WORLD_RADIUS)))))
        thr = int(rng.integers(40, 66))
        biome = 3 if rng.uniform() < 0.25 else 0
        out.append((t, Search(seed=seed, center_x=cx, center_z=cz, radius=radius, min_size=thr,
                              biome_flags=biome)))
    return out
