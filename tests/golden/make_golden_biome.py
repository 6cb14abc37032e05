"""Generate tests/golden/biome.npz by running the reference biome module's own code on the CPU.

The reference code is MinecraftGPUNoise.cu's device math compiled for the host by oracle/Makefile
(`make -C oracle ref_biome REF_DIR=<reference tree>` -> oracle/_ref/libmcgpu_host_ref.so). Run from
the repository root:

    python tests/golden/make_golden_biome.py

Contents (all seeded; world seeds from the 16-seed precise/biome workload):
  xr_*        Xoroshiro128++ nextLong sequences of 64 seeds (8 draws each)
  perlin_*    single improved-noise samples (seed, x, y, z), a third of them at y = 0
  spline_*    depth-spline values of 4,096 (c, e, pv, w) inputs, as float bits
  c6_*        climate6 {T, H, C, E, depth, W} of 4,096 quarts (normal) and 1,024 (large biomes)
  bio_*       biome ids of 8,192 quarts, version 26.2, and 2,048 at versions 1.18-1.21.5
  flt_*       filter masks (flags 3, version 26.2) of 160 candidates: random centres, centres whose
              window holds exactly one Deep Dark quart (border cases) and centres on a slime chunk
              inside Mushroom Fields
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import RefBiomeHost  # noqa: E402
from slime_b200 import workloads  # noqa: E402

OUT = Path(__file__).resolve().parent / "biome.npz"
VERSION = 2602


def u64(a):
    return np.asarray(a, dtype=np.uint64)


def deep_hits(ref, ws, cx, cz):
    """Number of (slime chunk, quart, layer) Deep Dark hits in the window of centre (cx, cz)."""
    from oracle.oracle import python_is_slime
    xs, ys, zs = [], [], []
    for dx in range(-8, 9):
        for dz in range(-8, 9):
            if dx * dx + dz * dz > 68 or not python_is_slime(ws, cx + dx, cz + dz):
                continue
            for q in range(16):
                for y in range(-16, 1):
                    xs.append((cx + dx) * 4 + q // 4)
                    zs.append((cz + dz) * 4 + q % 4)
                    ys.append(y)
    if not xs:
        return 0
    return int((ref.biome_at(VERSION, ws, xs, ys, zs) == 183).sum())


def main():
    ref = RefBiomeHost()
    rng = np.random.Generator(np.random.PCG64(20261204))
    seeds16 = [q.seed for q in workloads.precise_biome_seeds()]
    ws = seeds16[0] & (2**64 - 1)
    out = {"world_seed": np.array([ws], dtype=np.uint64)}

    xr_seeds = u64(rng.integers(0, 2**63, 64, dtype=np.int64)) * u64(2) + u64(rng.integers(0, 2, 64))
    out["xr_seeds"] = xr_seeds
    out["xr_out"] = ref.xoroshiro(xr_seeds, 8)

    n = 512
    ps = u64(rng.integers(0, 2**63, n, dtype=np.int64)) * u64(2) + u64(rng.integers(0, 2, n))
    px = rng.uniform(-2e6, 2e6, n)
    py = np.where(rng.uniform(size=n) < 1 / 3, 0.0, rng.uniform(-512, 512, n))
    pz = rng.uniform(-2e6, 2e6, n)
    out.update(perlin_seeds=ps, perlin_x=px, perlin_y=py, perlin_z=pz, perlin_out=ref.perlin(ps, px, py, pz))

    v = np.concatenate([rng.uniform(-1.3, 1.3, (3072, 4)),
                        rng.choice(np.linspace(-1.2, 1.2, 49), (1024, 4))]).astype(np.float32)
    out["spline_in"] = v
    out["spline_out"] = np.array([ref.depth_spline(r) for r in v], dtype=np.float32).view(np.uint32)

    for tag, large, m in (("", 0, 4096), ("_large", 1, 1024)):
        qx = rng.integers(-7_500_000, 7_500_001, m, dtype=np.int64).astype(np.int32)
        qz = rng.integers(-7_500_000, 7_500_001, m, dtype=np.int64).astype(np.int32)
        qy = rng.integers(-16, 17, m, dtype=np.int64).astype(np.int32)
        out[f"c6{tag}_xyz"] = np.stack([qx, qy, qz], 1)
        out[f"c6{tag}_out"] = ref.climate6(ws, qx, qy, qz, large)

    m = 8192
    qx = rng.integers(-7_500_000, 7_500_001, m, dtype=np.int64).astype(np.int32)
    qz = rng.integers(-7_500_000, 7_500_001, m, dtype=np.int64).astype(np.int32)
    qy = np.where(rng.uniform(size=m) < 0.7, rng.integers(-16, 1, m), rng.integers(-16, 17, m)).astype(np.int32)
    out["bio_xyz"] = np.stack([qx, qy, qz], 1)
    out["bio_out"] = ref.biome_at(VERSION, ws, qx, qy, qz)
    out["bio_large_out"] = ref.biome_at(VERSION, ws, qx, qy, qz, 1)
    vers = np.array([1180, 1192, 1194, 1206, 1214, 1215], dtype=np.int32)
    out["bio_versions"] = vers
    out["bio_versions_out"] = np.stack([ref.biome_at(int(vv), ws, qx[:2048], qy[:2048], qz[:2048]) for vv in vers])

    # Candidates: random centres, single-hit border cases and mushroom-field centres.
    cand = [(int(x), int(z)) for x, z in rng.integers(-1_800_000, 1_800_001, (96, 2))]
    border = []
    tries = 0
    while len(border) < 32 and tries < 4000:
        tries += 1
        x, z = (int(a) for a in rng.integers(-1_800_000, 1_800_001, 2))
        if deep_hits(ref, ws, x, z) == 1:
            border.append((x, z))
    mush = []
    tries = 0
    from oracle.oracle import python_is_slime
    while len(mush) < 32 and tries < 400_000:
        tries += 1
        x, z = (int(a) for a in rng.integers(-1_800_000, 1_800_001, 2))
        if ref.biome_at(VERSION, ws, [x * 4], [16], [z * 4])[0] != 14:
            continue
        for dx in range(-3, 4):
            if python_is_slime(ws, x + dx, z):
                mush.append((x + dx, z))
                break
    cand += border + mush
    cx = np.array([c[0] for c in cand], dtype=np.int32)
    cz = np.array([c[1] for c in cand], dtype=np.int32)
    out["flt_cx"], out["flt_cz"] = cx, cz
    out["flt_kind"] = np.array([0] * 96 + [1] * len(border) + [2] * len(mush), dtype=np.int8)
    out["flt_mask"] = ref.filter(VERSION, ws, cx, cz, 3)
    out["flt_mask_deep"] = ref.filter(VERSION, ws, cx, cz, 1)
    out["flt_mask_mush"] = ref.filter(VERSION, ws, cx, cz, 2)
    np.savez_compressed(OUT, **out)
    print(OUT, {k: v.shape for k, v in out.items()})
    print("mask counts", np.bincount(out["flt_mask"], minlength=4), "border", len(border), "mushroom", len(mush))


if __name__ == "__main__":
    main()
