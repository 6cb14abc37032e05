"""The biome oracle (oracle/biome_oracle.c) against golden vectors made by the reference's own code.

tests/golden/biome.npz comes from MinecraftGPUNoise.cu's device math compiled for the CPU
(tests/golden/make_golden_biome.py). Every stage is compared exactly: Xoroshiro draws, Perlin
samples (double bits), depth-spline values (float bits), quantised climate parameters, biome ids
and filter masks. Where the reference's host build is present (built from the reference tree),
fresh random inputs are compared too."""
import numpy as np
import pytest

from oracle.oracle import REF_BIOME_HOST_SO, BiomeOracle

GOLD = None


@pytest.fixture(scope="module")
def g():
    from pathlib import Path
    return np.load(Path(__file__).resolve().parent / "golden" / "biome.npz")


@pytest.fixture(scope="module")
def o():
    return BiomeOracle()


def test_xoroshiro(o, g):
    assert np.array_equal(o.xoroshiro(g["xr_seeds"], 8), g["xr_out"])


def test_perlin_bits(o, g):
    got = o.perlin(g["perlin_seeds"], g["perlin_x"], g["perlin_y"], g["perlin_z"])
    assert np.array_equal(got.view(np.uint64), g["perlin_out"].view(np.uint64))


def test_depth_spline_bits(o, g):
    got = np.array([o.depth_spline(v) for v in g["spline_in"]], dtype=np.float32).view(np.uint32)
    assert np.array_equal(got, g["spline_out"])


@pytest.mark.parametrize("large", [0, 1])
def test_climate6(o, g, large):
    tag = "_large" if large else ""
    xyz = g[f"c6{tag}_xyz"]
    ws = int(g["world_seed"][0])
    assert np.array_equal(o.climate6(ws, xyz[:, 0], xyz[:, 1], xyz[:, 2], large), g[f"c6{tag}_out"])


def test_biome_ids(o, g):
    xyz = g["bio_xyz"]
    ws = int(g["world_seed"][0])
    assert np.array_equal(o.biome_at(2602, ws, xyz[:, 0], xyz[:, 1], xyz[:, 2]), g["bio_out"])
    assert np.array_equal(o.biome_at(2602, ws, xyz[:, 0], xyz[:, 1], xyz[:, 2], 1), g["bio_large_out"])
    for v, want in zip(g["bio_versions"], g["bio_versions_out"]):
        got = o.biome_at(int(v), ws, xyz[:2048, 0], xyz[:2048, 1], xyz[:2048, 2])
        assert np.array_equal(got, want), v
    # Both verdict biomes occur among the golden quarts.
    assert (g["bio_out"] == 183).any() and (g["bio_out"] == 14).any()


@pytest.mark.parametrize("flags,key", [(3, "flt_mask"), (1, "flt_mask_deep"), (2, "flt_mask_mush")])
def test_filter_masks(o, g, flags, key):
    ws = int(g["world_seed"][0])
    got = o.filter(2602, ws, g["flt_cx"], g["flt_cz"], flags)
    assert np.array_equal(got, g[key])
    kinds = g["flt_kind"]
    assert (g["flt_mask"][kinds == 1] & 1).all() and (g["flt_mask"][kinds == 2] & 2).all()


@pytest.mark.skipif(not REF_BIOME_HOST_SO.exists(), reason="reference biome host build absent")
def test_oracle_vs_reference_host_build_random():
    from oracle.oracle import RefBiomeHost
    o, r = BiomeOracle(), RefBiomeHost()
    rng = np.random.default_rng(99)
    ws = int(rng.integers(-2**63, 2**63, dtype=np.int64)) & (2**64 - 1)
    n = 3000
    qx = rng.integers(-30_000_000, 30_000_000, n)
    qz = rng.integers(-30_000_000, 30_000_000, n)
    qy = rng.integers(-64, 64, n)
    for large in (0, 1):
        assert np.array_equal(o.climate6(ws, qx, qy, qz, large), r.climate6(ws, qx, qy, qz, large))
        assert np.array_equal(o.biome_at(2602, ws, qx, qy, qz, large), r.biome_at(2602, ws, qx, qy, qz, large))
    cx = rng.integers(-1_800_000, 1_800_000, 24)
    cz = rng.integers(-1_800_000, 1_800_000, 24)
    assert np.array_equal(o.filter(2602, ws, cx, cz, 3), r.filter(2602, ws, cx, cz, 3))
