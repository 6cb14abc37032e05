"""Reference checks for searches in the tests: the reference's own libraries, not this project's.

A search small enough for the reference CPU library (SlimeCore.cpp compiled from source, all host
threads) is checked against it; a larger one against the reference GPU library (SlimeCoreGPU.cu
compiled for sm_100a). Both return the total and the ranked 24-byte records; the comparison is
exact on every field. Precise AFK scores are compared against the reference CPU routine
(score_candidates_precise, scan_xz = 1), whose semantics this project follows.
"""
from __future__ import annotations

import numpy as np

# Areas up to (2 * 20,000 + 1)^2 = 1.6e9 centres run on the reference CPU library (well under a
# second with all host threads); larger ones on the reference GPU library.
CPU_MAX_RADIUS = 20_000

_cpu = None
_gpu = None


def ref_cpu():
    global _cpu
    if _cpu is None:
        from oracle.oracle import RefCpu
        _cpu = RefCpu()
        _cpu.set_y_scan_config(0, -64, -64, 64, 4)
    return _cpu


def ref_gpu():
    global _gpu
    if _gpu is None:
        from oracle.oracle import RefGpu
        _gpu = RefGpu()
    return _gpu


def reference_search(q):
    """(total, ranked records) of search q from the reference, without precise scoring."""
    if q.radius <= CPU_MAX_RADIUS:
        return ref_cpu().search(q.seed, q.radius, q.min_size, q.max_size, q.rd_min, q.center_x,
                                q.center_z, q.max_results)
    return ref_gpu().search(q.seed, q.radius, q.min_size, q.max_size, q.rd_min, q.center_x,
                            q.center_z, q.max_results)


def check_against_reference(q, total, res, label=""):
    """Exact comparison of one search's output with the reference's. With precise_afk, the
    unscored fields are compared with the reference search and the scores of the best
    min(n, 100) with the reference CPU scoring of the same sites (SlimeCoreGPU.cu:3884 scores
    the best 100 at search time)."""
    t_r, r_r = reference_search(q)
    assert total == t_r, (label, q, total, t_r)
    assert len(res) == len(r_r), (label, q)
    if not q.precise_afk:
        assert np.array_equal(res, r_r), (label, q)
        return
    for f in ("size", "center_x", "center_z"):
        assert np.array_equal(res[f], r_r[f]), (label, q, f)
    n = min(len(res), 100)
    if n:
        base = r_r[:n].copy()
        base["obs_count"] = 0
        base["afk_x"] = base["center_x"]
        base["afk_z"] = base["center_z"]
        scored = ref_cpu().score_precise(q.seed, base, scan_xz=1)
        assert np.array_equal(res[:n], scored), (label, q)
    if len(res) > n:
        assert np.array_equal(res[n:], r_r[n:]), (label, q)
