"""The oracle (oracle/slime_oracle.c) pinned against golden vectors made by the reference's own
CPU library (tests/golden/make_golden.py), and against the compiled reference where present."""
import numpy as np
import pytest

from oracle.oracle import RESULT_DTYPE, YConfig, python_is_slime


def test_predicate_golden(oracle, golden):
    g = golden["predicate"]
    got = np.array([oracle.is_slime(int(s), int(x), int(z))
                    for s, x, z in zip(g["seed"], g["x"], g["z"])], dtype=np.uint8)
    assert np.array_equal(got, g["slime"])


def test_predicate_python_restatement(golden):
    g = golden["predicate"]
    idx = np.arange(0, len(g["seed"]), 7)
    for i in idx:
        assert python_is_slime(int(g["seed"][i]), int(g["x"][i]), int(g["z"][i])) == bool(g["slime"][i])


def test_rejection_cases_present(golden):
    """The golden set must exercise Java's nextInt(10) redraw: some crafted first draws are
    rejected and still end as slime chunks, and some do not."""
    g = golden["predicate"]
    crafted = g["slime"][-1400:-200]
    assert 0 < crafted.sum() < len(crafted)


@pytest.mark.parametrize("idx", range(8))
def test_search_golden(oracle, golden, idx):
    g = golden["search"]
    name = str(g["names"][idx])
    seed, rd_max, lo, hi, rd_min, cx, cz, maxr, total = (int(v) for v in g["params"][idx])
    got_total, got = oracle.search(seed, rd_max, lo, hi, rd_min, cx, cz, maxr)
    assert got_total == total, name
    assert np.array_equal(got, g[f"{name}_results"]), name


def test_precise_golden(oracle, golden):
    g = golden["precise"]
    seed = int(g["seed"])
    assert np.array_equal(oracle.score_precise(seed, g["sites"], scan_xz=1), g["xz"])
    assert np.array_equal(oracle.score_precise(seed, g["sites"], scan_xz=0), g["single"])
    assert np.array_equal(oracle.score_precise(seed, g["sites_odd"], scan_xz=1), g["xz_odd"])
    y = YConfig(1, -64, -64, 64, 16)
    assert np.array_equal(oracle.score_precise(seed, g["sites"][:16], 1, y), g["yscan"])
    assert np.array_equal(oracle.refine_y(seed, g["sites"][:16], y), g["refine"])
    p70 = YConfig(0, 70, -64, 64, 4)
    assert np.array_equal(oracle.score_precise(seed, g["sites"][:16], 1, p70), g["platform70"])


def test_window_counts_brute_force(oracle):
    seed, cx0, cz0, w, h = 99, -1234, 5678, 23, 19
    bm = oracle.bitmap(seed, cx0 - 8, cz0 - 8, w + 16, h + 16)
    mask = np.array([[dx * dx + dz * dz <= 68 for dx in range(-8, 9)] for dz in range(-8, 9)])
    assert mask.sum() == 221
    want = np.zeros((h, w), dtype=np.int32)
    for j in range(h):
        for i in range(w):
            want[j, i] = (bm[j:j + 17, i:i + 17] * mask).sum()
    assert np.array_equal(oracle.window_counts(seed, cx0, cz0, w, h), want)


def test_invalid_arguments(oracle):
    assert oracle.search(1, -1, 40, 221)[0] == -1
    assert oracle.search(1, 10, 222, 221)[0] == -1
    assert oracle.search(1, 10, 40, 39)[0] == -1
    assert oracle.search(1, 10, 40, 221, rd_min=11)[0] == -1
    assert oracle.search(1, 10, 40, 221, center_x=2**31 - 10)[0] == -1


def test_reference_library_agrees(oracle):
    """Direct differential check when the compiled reference library is present."""
    from oracle.oracle import REF_SO, RefCpu
    if not REF_SO.exists():
        pytest.skip("reference CPU library not built")
    ref = RefCpu()
    for seed, r, lo, hi, rdm, cx, cz in [(5, 150, 30, 221, 0, 77, -99), (-8, 90, 20, 40, 30, 0, 0)]:
        t1, a = ref.search(seed, r, lo, hi, rdm, cx, cz, 10_000)
        t2, b = oracle.search(seed, r, lo, hi, rdm, cx, cz, 10_000)
        assert t1 == t2 and np.array_equal(a, b)
