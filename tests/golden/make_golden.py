"""Generate the golden vectors under tests/golden/ by running the reference's own CPU library.

The reference library is SlimeCore.cpp compiled from the reference source tree by
``oracle/Makefile`` (``make -C oracle ref``). Run from the repository root:

    python tests/golden/make_golden.py

Outputs (small .npz files, committed):
  predicate.npz  per-chunk slime bits for random, edge-of-range and crafted rejection-path inputs
  search.npz     full ranked outputs of several centred searches (configs in SEARCHES)
  precise.npz    precise AFK scores (score_candidates_precise / refine_candidates_y)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import RESULT_DTYPE, RefCpu  # noqa: E402
from slime_b200 import workloads  # noqa: E402

OUT = Path(__file__).resolve().parent
M48 = (1 << 48) - 1
M64 = (1 << 64) - 1
LCG = 0x5DEECE66D
SCRAMBLE = 0x3AD8025F
LCG_INV = pow(LCG, -1, 1 << 48)

# (name, seed, rd_max, min_size, max_size, rd_min, center_x, center_z, max_results)
SEARCHES = [
    ("plain_4001", None, 2000, 40, 221, 0, 0, 0, 100_000),
    ("offset_annulus", 0x1234_5678_9ABC_DEF0 - (1 << 63), 300, 35, 45, 100, 12345, -67890, 5000),
    ("truncated_top50", -4551278310048043, 500, 30, 221, 0, -1_874_000, 1_874_500, 50),
    ("all_centres", 123456789, 20, 0, 221, 0, 1_000_000, -1_000_000, 2000),
    ("none", 987654321, 200, 221, 221, 0, 0, 0, 10),
    ("single_centre", 42, 0, 0, 221, 0, -5, 7, 4),
    ("upper_bounded", 77, 700, 10, 18, 0, 131_072, -131_072, 3000),
    ("border", -1, 600, 38, 221, 0, 1_874_999, -1_874_999, 2000),
]


def s32(v: int) -> int:
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v & 0x80000000 else v


def mix_terms(x: int, z: int) -> int:
    x, z = s32(x), s32(z)
    return (s32(x * x * 0x4C1906) + s32(x * 0x5AC0DB) + s32(z * z) * 0x4307A7
            + s32(z * 0x5F24F)) & M64


def to_i64(v: int) -> int:
    v &= M64
    return v - (1 << 64) if v >> 63 else v


def crafted_seed(x: int, z: int, state1: int, high: int) -> int:
    """A world seed whose first LCG output at chunk (x, z) is `state1`."""
    state0 = (LCG_INV * (state1 - 0xB)) & M48
    mix = (state0 ^ SCRAMBLE ^ LCG) & M48 | (high << 48)
    return to_i64(mix - mix_terms(x, z))


def predicate_cases(rng: np.random.Generator):
    cases = []
    for _ in range(3000):
        seed = int(rng.integers(-(2**63), 2**63, dtype=np.int64))
        if rng.uniform() < 0.5:
            x, z = (int(v) for v in rng.integers(-(2**31), 2**31, size=2))
        else:
            x, z = (int(v) for v in rng.integers(-1_875_008, 1_875_009, size=2))
        cases.append((seed, x, z))
    edges = [0, 1, -1, 2**31 - 1, -(2**31), 2**31 - 9, -(2**31) + 8, 1_875_000, -1_875_000,
             1_875_008, -1_875_008, 65_536, -65_536, 131_072, -131_072, 262_144, 46_341, -46_341]
    for seed in (0, 1, -1, 2**63 - 1, -(2**63), 123456789, -4551278310048043):
        for x in edges:
            for z in edges[::3]:
                cases.append((seed, x, z))
    # Rejection path: the first draw lies in the top 2^20 LCG states (bits >= 2^31 - 8), so
    # Java redraws. Every one of the 8 rejected `bits` values appears, with random low bits.
    for k in range(1200):
        x = int(rng.integers(-1_875_008, 1_875_009))
        z = int(rng.integers(-1_875_008, 1_875_009))
        bits = (1 << 31) - 8 + (k % 8)
        state1 = (bits << 17) | int(rng.integers(0, 1 << 17))
        cases.append((crafted_seed(x, z, state1, int(rng.integers(0, 1 << 16))), x, z))
    # Accepted draws just below the rejection boundary (bits = 2^31 - 9 ... 2^31 - 40).
    for k in range(200):
        x = int(rng.integers(-100_000, 100_000))
        z = int(rng.integers(-100_000, 100_000))
        bits = (1 << 31) - 9 - (k % 32)
        state1 = (bits << 17) | int(rng.integers(0, 1 << 17))
        cases.append((crafted_seed(x, z, state1, 0), x, z))
    return cases


def main() -> None:
    ref = RefCpu()
    rng = np.random.Generator(np.random.PCG64(20240601))

    cases = predicate_cases(rng)
    seeds = np.array([c[0] for c in cases], dtype=np.int64)
    xs = np.array([c[1] for c in cases], dtype=np.int64)
    zs = np.array([c[2] for c in cases], dtype=np.int64)
    expect = np.zeros(len(cases), dtype=np.uint8)
    for i, (seed, x, z) in enumerate(cases):
        # build_chunk_cache's base chunk is floor(ox/16) - 10, so ox = 16x + 160 puts (x, z)
        # at cache bit [0][0].
        bits, bx, bz = ref.chunk_cache(seed, 16 * x + 160, 16 * z + 160)
        assert bx == x and bz == z
        expect[i] = bits[0, 0]
    np.savez_compressed(OUT / "predicate.npz", seed=seeds, x=xs, z=zs, slime=expect)
    print("predicate cases", len(cases), "slime", int(expect.sum()))

    plain = workloads.plain_search()
    arrays = {}
    meta = []
    for name, seed, rd_max, lo, hi, rd_min, cx, cz, maxr in SEARCHES:
        if seed is None:
            seed = plain.seed
        ref.set_y_scan_config(0, -64, -64, 64, 4)
        total, res = ref.search(seed, rd_max, lo, hi, rd_min, cx, cz, maxr, precise_afk=0)
        arrays[f"{name}_results"] = res
        meta.append((name, seed, rd_max, lo, hi, rd_min, cx, cz, maxr, total))
        print(name, total, len(res))
    meta_arr = np.array([m[1:] for m in meta], dtype=np.int64)
    np.savez_compressed(OUT / "search.npz", names=np.array([m[0] for m in meta]), params=meta_arr,
                        **arrays)

    # Precise AFK scores of the best 64 plain-search sites, and of shifted arbitrary centres.
    top = arrays["plain_4001_results"][:64].copy()
    odd = top.copy()
    odd["center_x"] += rng.integers(-7, 8, size=len(odd)).astype(np.int32)
    odd["center_z"] += rng.integers(-7, 8, size=len(odd)).astype(np.int32)
    ref.set_y_scan_config(0, -64, -64, 64, 4)
    xz = ref.score_precise(plain.seed, top, scan_xz=1)
    single = ref.score_precise(plain.seed, top, scan_xz=0)
    xz_odd = ref.score_precise(plain.seed, odd, scan_xz=1)
    ref.set_y_scan_config(1, -64, -64, 64, 16)
    yscan = ref.score_precise(plain.seed, top[:16], scan_xz=1)
    refine = ref.refine_y(plain.seed, top[:16])
    ref.set_y_scan_config(0, 70, -64, 64, 4)
    platform70 = ref.score_precise(plain.seed, top[:16], scan_xz=1)
    ref.set_y_scan_config(0, -64, -64, 64, 4)
    np.savez_compressed(OUT / "precise.npz", seed=np.int64(plain.seed), sites=top,
                        sites_odd=odd, xz=xz, single=single, xz_odd=xz_odd, yscan=yscan,
                        refine=refine, platform70=platform70)
    print("precise", xz["obs_count"][:5], yscan["obs_count"][:3])
    assert xz.dtype == RESULT_DTYPE


if __name__ == "__main__":
    main()
