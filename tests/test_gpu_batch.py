"""GPU parity of the batched search (slime_b200_search_batch).

Every request of a batch must come back exactly as the single search returns it (same total,
same ranked records), whether it ran in the shared persistent launch or on its own, and exactly as
the reference returns it: requests up to radius 20k against the reference CPU library, and the
largest ones against the reference GPU library built for sm_100a (tests/refcheck.py)."""
import numpy as np
import pytest

from slime_b200.workloads import Search
from tests.refcheck import CPU_MAX_RADIUS, check_against_reference

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def core():
    from slime_b200 import build
    from slime_b200.lib import SlimeCoreB200
    build.build()
    c = SlimeCoreB200()
    c.set_y_scan_config(0, -64, -64, 64, 4)
    c.lib.reset_cancel()
    yield c
    c.lib.slime_b200_set_engine(0, 0)


def singles(core, searches):
    out = []
    for q in searches:
        core.lib.reset_cancel()
        out.append(core.search(q.seed, q.radius, q.min_size, q.max_size, q.rd_min, q.center_x,
                               q.center_z, q.max_results, q.precise_afk))
    return out


def check_same(batch, single):
    assert len(batch) == len(single)
    for i, ((tb, rb), (ts, rs)) in enumerate(zip(batch, single)):
        assert tb == ts, i
        assert np.array_equal(rb, rs), i


def test_batch_mixed_requests(core):
    from tests.test_gpu_band import rare_seed
    searches = [
        Search(seed=11, center_x=0, center_z=0, radius=300, min_size=30, max_results=5000),
        Search(seed=-12, center_x=500_000, center_z=-20, radius=20_000, min_size=45, max_results=300),
        Search(seed=13, center_x=-1_874_500, center_z=1_874_600, radius=60_000, min_size=50, max_results=200),
        Search(seed=14, center_x=7, center_z=7, radius=2_000, min_size=28, max_size=33, max_results=50),
        Search(seed=15, center_x=0, center_z=9_000, radius=9_000, min_size=40, rd_min=5_000, max_results=700),
        Search(seed=16, center_x=1, center_z=2, radius=1_500, min_size=20, max_results=100),   # below 28: alone
        Search(seed=17, center_x=0, center_z=0, radius=30_000, min_size=47, max_results=100, precise_afk=1),
        Search(seed=rare_seed(123_457, -98_765, 0), center_x=123_462, center_z=-98_768, radius=60,
               min_size=30, max_results=5000),
        Search(seed=18, center_x=0, center_z=0, radius=100, min_size=60, max_results=10),     # no sites
        Search(seed=19, center_x=-3, center_z=3, radius=0, min_size=0, max_results=4),        # one centre
        Search(seed=20, center_x=100, center_z=100, radius=4_000, min_size=36, max_results=3), # truncated
        Search(seed=21, center_x=-300_000, center_z=0, radius=140_000, min_size=56, max_results=50),  # shared LCG
        Search(seed=22, center_x=0, center_z=300_000, radius=140_000, min_size=50, rd_min=100_000,
               max_results=400),
    ]
    single = singles(core, searches)
    assert core.lib.get_gpu_v1_algorithm() in (220, 300)  # grouped or independent bands
    batch = core.search_batch(searches)
    check_same(batch, single)
    for i, (q, (total, res)) in enumerate(zip(searches, batch)):
        check_against_reference(q, total, res, f"mixed batch request {i}")


def test_batch_invalid_request_is_reported_and_others_run(core):
    good = Search(seed=5, center_x=0, center_z=0, radius=1_000, min_size=35, max_results=100)
    bad = Search(seed=5, center_x=0, center_z=0, radius=1_000, min_size=40, max_size=39, max_results=100)
    out = core.search_batch([good, bad, good])
    assert out[1][0] == -1 and len(out[1][1]) == 0
    ref = singles(core, [good])[0]
    for k in (0, 2):
        assert out[k][0] == ref[0] and np.array_equal(out[k][1], ref[1])


def test_batch_empty(core):
    assert core.search_batch([]) == []


def test_batch_of_the_64_seed_workload(core):
    from slime_b200 import workloads
    searches = workloads.batch_searches()
    assert len(searches) == 64
    batch = core.search_batch(searches)
    check_same(batch, singles(core, searches))
    # Against the reference: every request the CPU library runs in well under a second, and the
    # four largest on the reference GPU library.
    small = [i for i, q in enumerate(searches) if q.radius <= CPU_MAX_RADIUS]
    large = sorted(range(len(searches)), key=lambda i: -searches[i].radius)[:4]
    assert len(small) >= 30
    for i in small + large:
        check_against_reference(searches[i], *batch[i], f"64-seed batch request {i}")


def test_batch_low_threshold_wide_requests(core):
    """Low thresholds on areas 4+ periods wide run as grouped bands with exact counts (their own
    launch class) inside the batch, beside bounded grouped and independent-band searches; every
    result equals the single search's and the reference's."""
    searches = [
        Search(seed=51, center_x=-400_000, center_z=200_000, radius=300_000, min_size=44, max_results=3000),
        Search(seed=-52, center_x=0, center_z=0, radius=280_000, min_size=43, max_size=50, rd_min=100_000,
               max_results=1000),
        Search(seed=53, center_x=1_000_000, center_z=-1_000_000, radius=150_000, min_size=52, max_results=200),
        Search(seed=54, center_x=7, center_z=-7, radius=15_000, min_size=46, max_results=500),
    ]
    single = singles(core, searches)
    assert core.lib.get_gpu_v1_algorithm() in (100, 300)  # the last, small search
    core.lib.reset_cancel()
    core.search(searches[0].seed, searches[0].radius, searches[0].min_size, 221, 0, searches[0].center_x,
                searches[0].center_z, 10)
    assert core.lib.get_gpu_v1_algorithm() == 230  # grouped bands, exact counts
    batch = core.search_batch(searches)
    check_same(batch, single)
    for i, (q, (total, res)) in enumerate(zip(searches, batch)):
        check_against_reference(q, total, res, f"low-threshold batch request {i}")
