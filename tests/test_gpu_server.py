"""GPU tests of the search server (slime_b200_server_*): results in the mix are exactly the
single search's results and the reference's (tests/refcheck.py: the reference CPU library up to
radius 20k, its GPU library above), admission respects the device-memory budget, and continuous
batching lets small requests finish while a large one is in flight."""
import numpy as np
import pytest

from slime_b200.workloads import Search
from tests.refcheck import check_against_reference

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def core():
    from slime_b200 import build
    from slime_b200.lib import SlimeCoreB200
    build.build()
    c = SlimeCoreB200()
    c.set_y_scan_config(0, -64, -64, 64, 4)
    c.lib.reset_cancel()
    return c


def single(core, q):
    core.lib.reset_cancel()
    return core.search(q.seed, q.radius, q.min_size, q.max_size, q.rd_min, q.center_x, q.center_z,
                       q.max_results, q.precise_afk)


MIX = [
    Search(seed=31, center_x=0, center_z=0, radius=300, min_size=30, max_results=5000),
    Search(seed=-32, center_x=500_000, center_z=-20, radius=20_000, min_size=45, max_results=300),
    Search(seed=33, center_x=-1_874_500, center_z=1_874_600, radius=60_000, min_size=50, max_results=200),
    Search(seed=34, center_x=7, center_z=7, radius=2_000, min_size=28, max_size=33, max_results=50),
    Search(seed=35, center_x=0, center_z=9_000, radius=9_000, min_size=40, rd_min=5_000, max_results=700),
    Search(seed=36, center_x=1, center_z=2, radius=1_500, min_size=20, max_results=100),   # general scan
    Search(seed=37, center_x=0, center_z=0, radius=30_000, min_size=47, max_results=100, precise_afk=1),
    Search(seed=38, center_x=-300_000, center_z=0, radius=140_000, min_size=56, max_results=50),
    Search(seed=39, center_x=0, center_z=300_000, radius=140_000, min_size=50, rd_min=100_000, max_results=400),
    Search(seed=40, center_x=-3, center_z=3, radius=0, min_size=0, max_results=4),
]


def run_all(server, searches):
    tickets = [server.submit(q) for q in searches]
    out = []
    for t, q in zip(tickets, searches):
        assert server.wait(t) == server.DONE
        out.append(server.take(t, q.max_results))
    return out


def test_server_results_in_the_mix_equal_the_single_search(core):
    from slime_b200.lib import SlimeServer
    with SlimeServer(core=core) as server:
        got = run_all(server, MIX)
    for i, (q, (total, res, lat)) in enumerate(zip(MIX, got)):
        t_s, r_s = single(core, q)
        assert total == t_s
        assert np.array_equal(res, r_s)
        assert lat > 0
        check_against_reference(q, total, res, f"served request {i}")


def test_server_near_world_request_against_the_reference(core):
    """A near-world request (radius 1.5M, 9e12 centres) served beside small ones, compared with
    the reference GPU library."""
    from slime_b200.lib import SlimeServer
    near_world = Search(seed=-5_501_234_567_890, center_x=200_000, center_z=-300_000,
                        radius=1_500_000, min_size=60, max_results=500)
    with SlimeServer(core=core) as server:
        got = run_all(server, [near_world] + MIX[:4])
    for i, (q, (total, res, _)) in enumerate(zip([near_world] + MIX[:4], got)):
        check_against_reference(q, total, res, f"near-world mix request {i}")


def test_server_memory_budget_admission(core):
    from slime_b200.lib import SlimeServer
    # 64 MB admits the mix a few requests at a time (a general-scan request holds the 48 MB hit
    # buffer); a full-world threshold-40 general scan needs more than the whole budget (term
    # tables of 3,750,017 rows and columns plus the hit buffer) and fails without running.
    with SlimeServer(device_bytes=64 << 20, core=core) as server:
        big = Search(seed=41, center_x=0, center_z=0, radius=1_875_000, min_size=40, max_results=10)
        t_big = server.submit(big)
        got = run_all(server, MIX)
        assert server.wait(t_big) == server.FAILED
        assert server.take(t_big, 10)[0] == -1
    for q, (total, res, _) in zip(MIX, got):
        t_s, r_s = single(core, q)
        assert total == t_s and np.array_equal(res, r_s)


def test_server_small_requests_finish_while_a_large_one_runs(core):
    from slime_b200.lib import SlimeServer
    large = Search(seed=42, center_x=0, center_z=0, radius=600_000, min_size=55, max_results=100)
    small = [Search(seed=43 + k, center_x=1000 * k, center_z=0, radius=2_000, min_size=45, max_results=100)
             for k in range(5)]
    with SlimeServer(core=core) as server:
        t_large = server.submit(large)
        t_small = [server.submit(q) for q in small]
        res_small = []
        for t, q in zip(t_small, small):
            assert server.wait(t) == server.DONE
            res_small.append(server.take(t, q.max_results))
        assert server.wait(t_large) == server.DONE
        total_l, res_l, lat_l = server.take(t_large, large.max_results)
    assert max(lat for _, _, lat in res_small) < lat_l
    t_s, r_s = single(core, large)
    assert total_l == t_s and np.array_equal(res_l, r_s)
    check_against_reference(large, total_l, res_l, "large request")
    for q, (total, res, _) in zip(small, res_small):
        t_s, r_s = single(core, q)
        assert total == t_s and np.array_equal(res, r_s)


def test_server_destroy_with_requests_in_flight(core):
    """Closing the server while a large request runs and others wait ends the worker cleanly; the
    library then serves ordinary searches as before."""
    from slime_b200.lib import SlimeServer
    server = SlimeServer(core=core)
    big = Search(seed=50, center_x=0, center_z=0, radius=1_000_000, min_size=55, max_results=10)
    tickets = [server.submit(big)] + [server.submit(q) for q in MIX[:3]]
    assert all(server.poll(t) in (server.QUEUED, server.RUNNING, server.DONE) for t in tickets)
    server.close()
    q = MIX[1]
    t_s, r_s = single(core, q)
    assert t_s >= 0 and len(r_s) == min(t_s, q.max_results)


def test_server_gated_low_threshold_requests(core):
    """Requests with tens of millions of sites in range (thresholds 40-44 on wide areas) run in the
    batch kernel with an emission gate: only centres at or above it are sent, the totals come
    from the device histogram (rare-chunk corrected), and a gate that proves too high triggers a
    second pass. Results must be the single search's, beside small requests in the same steps."""
    from slime_b200.lib import SlimeServer
    reqs = [
        Search(seed=91, center_x=100_000, center_z=-250_000, radius=300_000, min_size=40, max_results=2000),
        Search(seed=-92, center_x=0, center_z=0, radius=200_000, min_size=42, max_size=47, max_results=500),
        Search(seed=93, center_x=-1_000_000, center_z=5_000, radius=250_000, min_size=44, rd_min=120_000,
               max_results=50_000),
        Search(seed=94, center_x=3, center_z=-3, radius=2_500, min_size=45, max_results=100),
    ]
    with SlimeServer(core=core) as server:
        got = run_all(server, reqs)
    for i, (q, (total, res, lat)) in enumerate(zip(reqs, got)):
        t_s, r_s = single(core, q)
        assert total == t_s, i
        assert np.array_equal(res, r_s), i
    assert got[0][0] > 10_000_000  # far more sites in range than the job's hit slice holds
