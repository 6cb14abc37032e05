"""GPU parity of the band engine (shared-LCG generator + rare redraw correction).

The band engine must return exactly what the general scan, the oracle and the reference return:
same totals, same ranked records."""
import numpy as np
import pytest

from oracle.oracle import REF_GPU_SO, python_is_slime

pytestmark = pytest.mark.gpu

M48 = (1 << 48) - 1
M64 = (1 << 64) - 1
LCG = 0x5DEECE66D
LCG_INV = pow(LCG, -1, 1 << 48)
SCRAMBLE = 0x3AD8025F


def s32(v):
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v & 0x80000000 else v


def mix_terms(x, z):
    x, z = s32(x), s32(z)
    return (s32(x * x * 0x4C1906) + s32(x * 0x5AC0DB) + s32(z * z) * 0x4307A7 + s32(z * 0x5F24F)) & M64


def rare_seed(x, z, k=0):
    """A world seed whose chunk (x, z) has a rejected first draw and is a slime chunk after
    Java's redraw (one of the 104,848 rare states; k picks which)."""
    found = 0
    for s1 in range((1 << 48) - (1 << 20), 1 << 48):
        st = s1
        while True:
            st = (st * LCG + 0xB) & M48
            bits = st >> 17
            if bits < 2147483640:
                break
        if bits % 10 == 0:
            if found == k:
                state0 = (LCG_INV * (s1 - 0xB)) & M48
                mix = (state0 ^ SCRAMBLE ^ LCG) & M48 | (0x1234 << 48)
                seed = (mix - mix_terms(x, z)) & M64
                return seed - (1 << 64) if seed >> 63 else seed
            found += 1


@pytest.fixture(scope="module")
def core():
    from slime_b200 import build
    from slime_b200.lib import SlimeCoreB200
    build.build()
    c = SlimeCoreB200()
    c.set_y_scan_config(0, -64, -64, 64, 4)
    yield c
    c.lib.slime_b200_set_engine(0, 0)


def run(core, mode, *args, **kw):
    core.lib.slime_b200_set_engine(mode, 0)
    core.lib.reset_cancel()
    try:
        return core.search(*args, **kw)
    finally:
        core.lib.slime_b200_set_engine(0, 0)


# Engine modes: 2 = shared-LCG band engine, 3 = independent-band engine, 4 / 5 = the same with
# bit-sliced exact counts of every centre (any threshold), 6 / 7 = grouped bands (X phase pairs with
# groups of Z period copies), bounded / with exact counts.
ALGO = {2: 200, 3: 300, 4: 210, 5: 310, 6: 220, 7: 230}
MODES = [2, 3, 4, 5, 6, 7]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("idx", range(8))
def test_band_engine_search_golden(core, golden, idx, mode):
    g = golden["search"]
    name = str(g["names"][idx])
    seed, rd_max, lo, hi, rd_min, cx, cz, maxr, total = (int(v) for v in g["params"][idx])
    if mode in (2, 3, 6) and lo < 28:
        pytest.skip("the bounded band engines need a threshold of 28 or more")
    got_total, got = run(core, mode, seed, rd_max, lo, hi, rd_min, cx, cz, maxr)
    assert core.lib.get_gpu_v1_algorithm() == ALGO[mode]
    assert got_total == total, name
    assert np.array_equal(got, g[f"{name}_results"]), name


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("k,thr", [(0, 30), (1, 28), (2, 33), (3, 29)])
def test_band_engine_planted_rare_chunk(core, oracle, k, thr, mode):
    x, z = 123_457 + 17 * k, -98_765 - 11 * k
    seed = rare_seed(x, z, k)
    assert python_is_slime(seed, x, z)
    args = (seed, 60, thr, 221, 0, x + 5, z - 3, 5000)
    t_o, r_o = oracle.search(*args)
    t_b, r_b = run(core, mode, *args)
    assert core.lib.slime_b200_last_rare_chunks() >= 1
    assert t_b == t_o
    assert np.array_equal(r_b, r_o)
    # The rare chunk must matter: some centre's count differs from the first-draw count.
    t_g, r_g = run(core, 1, *args)
    assert t_g == t_o and np.array_equal(r_g, r_o)


@pytest.mark.parametrize("mode", MODES)
def test_band_engine_planted_rare_upper_bound(core, oracle, mode):
    x, z = -1_500_000, 1_400_000
    seed = rare_seed(x, z, 5)
    args = (seed, 40, 30, 34, 7, x, z, 2000)
    t_o, r_o = oracle.search(*args)
    t_b, r_b = run(core, mode, *args)
    assert t_b == t_o and np.array_equal(r_b, r_o)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case", [
    (20240607, 140_000, 54, 221, 0, 0, 0, 2000),          # 2 phases x 3 bands, wide tiles
    (-31337, 300_000, 57, 221, 0, 400_000, -250_000, 500),  # 5 x 5 periods, offset centre
    (77, 270_000, 50, 60, 90_000, -1_000_000, 1_000_000, 3000),  # upper bound + annulus
    (5, 20_000, 45, 221, 0, 1_874_000, -1_874_000, 800),  # independent bands: 40,001^2 at the border
    (9, 3_000, 38, 221, 0, -7, 7, 100_000),               # small area, many sites
])
def test_band_vs_general_medium(core, case, mode):
    t_g, r_g = run(core, 1, *case)
    t_b, r_b = run(core, mode, *case)
    assert t_b == t_g
    assert np.array_equal(r_b, r_g)


@pytest.mark.parametrize("mode", MODES)
def test_band_vs_general_low_threshold_millions_of_sites(core, mode):
    """Threshold 42 on a 280,001^2 area: 3.1 million sites, a survivor queue that overflows in
    every tile, and ~30 rare chunks whose distance test to far-away sites must not wrap."""
    from slime_b200 import workloads
    seed = workloads.full_world_scan().seed
    case = (seed, 140_000, 42, 221, 0, 0, 0, 4_000_000)
    t_g, r_g = run(core, 1, *case)
    t_b, r_b = run(core, mode, *case)
    assert t_g > 3_000_000
    assert core.lib.slime_b200_last_rare_chunks() > 0
    assert t_b == t_g
    assert np.array_equal(r_b, r_g)


@pytest.mark.parametrize("mode", [4, 5, 7])
@pytest.mark.parametrize("case", [
    (20240607, 140_000, 40, 221, 0, 0, 0, 2000),             # threshold 40, shared LCG: 2 x 3 bands
    (-4242, 30_000, 36, 44, 5_000, 1_000_000, -3_000, 500),   # low threshold, upper bound, annulus
    (123, 2_500, 25, 221, 0, 0, 0, 200_000),                  # below the bounded engines' range
])
def test_exact_counts_vs_general_low_thresholds(core, case, mode):
    t_g, r_g = run(core, 1, *case)
    t_b, r_b = run(core, mode, *case)
    assert core.lib.get_gpu_v1_algorithm() == ALGO[mode]
    assert t_b == t_g
    assert np.array_equal(r_b, r_g)


@pytest.mark.skipif(not REF_GPU_SO.exists(), reason="reference GPU library not built")
def test_band_full_world_vs_reference_gpu(core):
    from oracle.oracle import RefGpu
    from slime_b200 import workloads
    spec = workloads.full_world_scan()
    t_b, r_b = run(core, 0, spec.seed, spec.radius, 60, 221, 0, 0, 0, 1000)
    assert core.lib.get_gpu_v1_algorithm() == 200
    t_r, r_r = RefGpu().search(spec.seed, spec.radius, 60, 221, 0, 0, 0, 1000)
    assert t_b == t_r
    assert np.array_equal(r_b, r_r)


@pytest.mark.parametrize("mode", [1, 4, 5])
@pytest.mark.parametrize("case", [
    (2718281828, 20_000, 40, 221, 18_000, 250_000, -90_000, 3000),   # rd_min = 0.9 rd_max
    (-161803, 6_000, 38, 45, 5_400, -1_000_000, 1_000_000, 800),     # with an upper bound
])
def test_annulus_skips_against_the_reference(core, case, mode):
    """Tiles (general scan) and strips (exact counts) wholly inside the rd_min disc are skipped;
    the result must still be the reference CPU library's."""
    from slime_b200.workloads import Search
    from tests.refcheck import check_against_reference
    seed, r, lo, hi, rdm, cx, cz, maxr = case
    total, res = run(core, mode, seed, r, lo, hi, rdm, cx, cz, maxr)
    check_against_reference(Search(seed=seed, center_x=cx, center_z=cz, radius=r, min_size=lo, max_size=hi,
                                   rd_min=rdm, max_results=maxr), total, res, f"annulus mode {mode}")


@pytest.mark.parametrize("mode", [2, 3, 5, 6, 7])
def test_bounded_wait_gives_up_cleanly(core, mode):
    """With a poll limit of 0 the first row-term wait of every CTA gives up: the CTA drains its
    copies in flight and flags the search, which returns -1 with an error text; with the default
    limit restored the library searches as before (no GPU fault is involved)."""
    case = (20240607, 140_000, 54, 221, 0, 0, 0, 2000)
    t_ok, r_ok = run(core, 1, *case)
    core.lib.slime_b200_set_wait_limit(0)
    try:
        core.lib.slime_b200_set_engine(mode, 0)
        core.lib.reset_cancel()
        buf = np.zeros(2000, dtype=r_ok.dtype)
        import ctypes
        total = core.lib.search_slime_clusters_gpu_v1_centered(*case[:7], buf.ctypes.data_as(ctypes.c_void_p),
                                                               2000, 0)
        assert total == -1
        assert b"timed out" in core.lib.slime_b200_last_error()
    finally:
        core.lib.slime_b200_set_wait_limit(-1)
        core.lib.slime_b200_set_engine(0, 0)
    t_b, r_b = run(core, mode, *case)
    assert t_b == t_ok and np.array_equal(r_b, r_ok)


@pytest.mark.parametrize("case", [
    (777, 100_000, 40, 221, 0, 300_000, 300_000, 2000),       # ~6.8e6 sites: the emission gate is raised
    (-888, 150_000, 41, 45, 60_000, 0, -1_500_000, 5000),    # gate with an upper bound and an annulus
])
def test_emission_gate_all_engines_agree_and_match_the_reference(core, case):
    """Single band searches count every centre on the device and send only those at or above a
    gate; totals come from the device histogram (corrected for rare chunks). All engines must give
    the general scan's answer, and the reference GPU library's."""
    t_g, r_g = run(core, 1, *case)
    for mode in (3, 4, 5, 6, 7):
        t_b, r_b = run(core, mode, *case)
        assert t_b == t_g, mode
        assert np.array_equal(r_b, r_g), mode
    from tests.refcheck import ref_gpu
    seed, r, lo, hi, rdm, cx, cz, maxr = case
    t_r, r_r = ref_gpu().search(seed, r, lo, hi, rdm, cx, cz, maxr)
    assert t_g == t_r and np.array_equal(r_g, r_r)


@pytest.mark.parametrize("case", [
    (424242, 100_000, 47, 221, 0, 600_000, -600_000, 3000),     # 1.5 periods: 2 copies x 8 groups
    (-99, 230_000, 52, 221, 0, -1_200_000, 350_000, 2000),      # 3.5 periods: 4 copies x 4 groups
    (31415, 180_585, 48, 58, 40_000, 123_456, -654_321, 4000),  # 2.8 periods, upper bound + annulus
    (8, 70_000, 44, 221, 0, 1_800_000, 1_800_000, 1500),        # 1.07 periods at the world border
])
def test_grouped_bands_vs_general_and_reference(core, case):
    """Grouped bands (X phase pairs, groups of Z period copies that share their low bits) must
    return the general scan's answer and the reference GPU library's."""
    t_g, r_g = run(core, 1, *case)
    for mode in (6, 7):
        t_b, r_b = run(core, mode, *case)
        assert core.lib.get_gpu_v1_algorithm() == ALGO[mode]
        assert t_b == t_g, mode
        assert np.array_equal(r_b, r_g), mode
    if REF_GPU_SO.exists():
        from tests.refcheck import ref_gpu
        seed, r, lo, hi, rdm, cx, cz, maxr = case
        t_r, r_r = ref_gpu().search(seed, r, lo, hi, rdm, cx, cz, maxr)
        assert t_b == t_r and np.array_equal(r_b, r_r)
