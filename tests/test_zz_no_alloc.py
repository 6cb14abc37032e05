"""The allocation-free search entry point (slime_b200_search_noalloc).

It exists for callers that cannot allocate GPU memory while they search (their own pool or
caching allocator owns the device memory, or the request path must not take cudaMalloc's implicit
synchronisation). It must return exactly what the regular entry point returns. Both are called
through the C ABI; the comparison is exact (integer results, no tolerance). This file is collected
last, so a run that stops at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    (-6166315385447640203, 2000, 40, 221, 0, 0, 0, 5000),     # plain 4,001^2 search, threshold 40
    (987654321, 700, 30, 36, 150, 123_456, -654_321, 300),     # annulus, upper bound, truncated
    (-77001234567, 8191, 30, 221, 0, -4_000, 9_000, 65536),    # widest area: 1,024-column tiles
    # Dense and upper-bounded: every centre with count 22 ties at the gate, so the first pass-2
    # launch emits ~2.4e7 hits and the slab is split until each launch fits the scratch list.
    (31337, 8191, 0, 22, 0, 1_000, -1_000, 65536),
]


@pytest.fixture(scope="module")
def lib():
    from slime_b200 import build
    from slime_b200.lib import load
    build.build()
    lib = load()
    lib.slime_b200_set_engine(0, 0)
    return lib


def _call(fn, case):
    from slime_b200.lib import RESULT_DTYPE
    seed, r, lo, hi, rdm, cx, cz, maxr = case
    buf = np.zeros(maxr, dtype=RESULT_DTYPE)
    ptr = buf.ctypes.data_as(ctypes.c_void_p)
    if fn.__name__ == "slime_b200_search_noalloc":
        total = fn(seed, r, lo, hi, rdm, cx, cz, ptr, maxr)
    else:
        total = fn(seed, r, lo, hi, rdm, cx, cz, ptr, maxr, 0)
    assert total >= 0
    return total, buf[: min(total, maxr)]


def test_noalloc_matches_regular_search_twice(lib):
    # Two calls in a row: the second must not see the first call's scratch contents.
    for case in CASES:
        t_ref, r_ref = _call(lib.search_slime_clusters_gpu_v1_centered, case)
        t_na, r_na = _call(lib.slime_b200_search_noalloc, case)
        assert t_na == t_ref, case
        assert np.array_equal(r_na, r_ref), case


def test_noalloc_leaves_device_memory_unchanged(lib):
    # After a first (set-up) call, a call takes no device memory: free memory is the same after it.
    import torch
    case = CASES[0]
    _call(lib.slime_b200_search_noalloc, case)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    t, r = _call(lib.slime_b200_search_noalloc, case)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert t > 0 and len(r) > 0


def test_noalloc_rejects_sizes_beyond_its_limit(lib):
    from slime_b200.lib import RESULT_DTYPE
    buf = np.zeros(65537, dtype=RESULT_DTYPE)
    ptr = buf.ctypes.data_as(ctypes.c_void_p)
    assert lib.slime_b200_search_noalloc(1, 8192, 40, 221, 0, 0, 0, ptr, 8) == -1
    assert b"8191" in lib.slime_b200_last_error()
    assert lib.slime_b200_search_noalloc(1, 100, 40, 221, 0, 0, 0, ptr, 65537) == -1
    assert b"65536" in lib.slime_b200_last_error()
