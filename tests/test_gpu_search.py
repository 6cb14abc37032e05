"""GPU parity of the search, the predicate and precise scoring, through the C ABI.

Every comparison is bit-exact: the same totals, the same ranked records (all six fields) and the
same per-chunk bits as the reference's own CPU library (golden vectors) or the oracle."""
import numpy as np
import pytest

from oracle.oracle import YConfig

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def core():
    from slime_b200 import build
    from slime_b200.lib import SlimeCoreB200
    build.build()
    c = SlimeCoreB200()
    assert c.lib.get_cuda_device_count() > 0
    c.set_y_scan_config(0, -64, -64, 64, 4)
    c.lib.reset_cancel()
    return c


def test_predicate_golden(core, golden):
    g = golden["predicate"]
    # One seed per call: the batch entry takes one world seed.
    got = np.zeros(len(g["seed"]), dtype=np.uint8)
    seeds = g["seed"]
    for s in np.unique(seeds):
        idx = np.nonzero(seeds == s)[0]
        got[idx] = core.is_slime_batch(int(s), g["x"][idx], g["z"][idx])
    assert np.array_equal(got, g["slime"])


def test_predicate_random_block(core, oracle):
    seed, x0, z0, w, h = -123456789012345, -1_875_008, 1_874_900, 300, 200
    xs, zs = np.meshgrid(np.arange(x0, x0 + w), np.arange(z0, z0 + h))
    got = core.is_slime_batch(seed, xs.ravel(), zs.ravel()).reshape(h, w)
    assert np.array_equal(got, oracle.bitmap(seed, x0, z0, w, h))


@pytest.mark.parametrize("idx", range(8))
def test_search_golden(core, golden, idx):
    g = golden["search"]
    name = str(g["names"][idx])
    seed, rd_max, lo, hi, rd_min, cx, cz, maxr, total = (int(v) for v in g["params"][idx])
    core.lib.reset_cancel()
    got_total, got = core.search(seed, rd_max, lo, hi, rd_min, cx, cz, maxr)
    assert got_total == total, name
    assert np.array_equal(got, g[f"{name}_results"]), name
    # Every centre of the square is visited (cf. the reference's own check, xp_scan.py:585).
    assert core.lib.get_processed_centers() == (2 * rd_max + 1) ** 2


@pytest.mark.parametrize("case", [
    (7, 1500, 45, 221, 0, 300_000, -200_000, 200),
    (-99, 900, 20, 30, 400, -1_000_000, 5, 500),
    (2**62 + 12345, 4100, 50, 221, 0, 0, 0, 50),
    (31337, 64, 0, 221, 0, 17, 17, 10_000),
    (5, 1, 0, 221, 1, 0, 0, 9),
])
def test_search_vs_oracle(core, oracle, case):
    seed, rd, lo, hi, rdm, cx, cz, maxr = case
    t_o, r_o = oracle.search(seed, rd, lo, hi, rdm, cx, cz, maxr)
    t_g, r_g = core.search(seed, rd, lo, hi, rdm, cx, cz, maxr)
    assert t_g == t_o
    assert np.array_equal(r_g, r_o)


def test_search_precise_vs_oracle(core, oracle):
    seed, rd, thr = 4242, 1200, 42
    core.set_y_scan_config(0, -64, -64, 64, 4)
    t_o, r_o = oracle.search(seed, rd, thr, 221, max_results=300, precise_afk=1, precise_limit=100)
    t_g, r_g = core.search(seed, rd, thr, 221, max_results=300, precise_afk=1)
    assert t_g == t_o and np.array_equal(r_g, r_o)


def test_search_precise_yscan_vs_oracle(core, oracle):
    seed, rd, thr = -77, 800, 40
    core.set_y_scan_config(1, -60, -64, 40, 8)
    try:
        t_o, r_o = oracle.search(seed, rd, thr, 221, max_results=120, precise_afk=1,
                                 precise_limit=100, ycfg=YConfig(1, -60, -64, 40, 8))
        t_g, r_g = core.search(seed, rd, thr, 221, max_results=120, precise_afk=1)
    finally:
        core.set_y_scan_config(0, -64, -64, 64, 4)
    assert t_g == t_o and np.array_equal(r_g, r_o)


def test_precise_golden(core, golden):
    g = golden["precise"]
    seed = int(g["seed"])
    core.set_y_scan_config(0, -64, -64, 64, 4)
    assert np.array_equal(core.score_precise(seed, g["sites"], 1), g["xz"])
    assert np.array_equal(core.score_precise(seed, g["sites"], 0), g["single"])
    assert np.array_equal(core.score_precise(seed, g["sites_odd"], 1), g["xz_odd"])
    core.set_y_scan_config(1, -64, -64, 64, 16)
    assert np.array_equal(core.score_precise(seed, g["sites"][:16], 1), g["yscan"])
    assert np.array_equal(core.refine_y(seed, g["sites"][:16]), g["refine"])
    core.set_y_scan_config(0, 70, -64, 64, 4)
    assert np.array_equal(core.score_precise(seed, g["sites"][:16], 1), g["platform70"])
    core.set_y_scan_config(0, -64, -64, 64, 4)


def test_precise_random_sites_vs_oracle(core, oracle):
    rng = np.random.default_rng(7)
    from slime_b200.lib import RESULT_DTYPE
    sites = np.zeros(200, dtype=RESULT_DTYPE)
    sites["center_x"] = rng.integers(-30_000_000, 30_000_000, size=200)
    sites["center_z"] = rng.integers(-30_000_000, 30_000_000, size=200)
    core.set_y_scan_config(0, -64, -64, 64, 4)
    assert np.array_equal(core.score_precise(99, sites, 1), oracle.score_precise(99, sites, 1))


def test_cancel_returns_partial_but_valid(core):
    core.lib.reset_cancel()
    core.lib.request_cancel()
    total, res = core.search(1, 3000, 45, 221, max_results=10)
    assert total >= 0 and len(res) <= 10
    core.lib.reset_cancel()
