"""CPU-side checks of the C-ABI library: it builds, loads without a GPU and exports every
symbol that include/*.h declares (no compute calls are made here)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while")))


@pytest.fixture(scope="module")
def lib():
    from slime_b200 import build, lib as L
    build.build()
    return L.load()


def test_header_declares_reference_abi():
    names = declared_functions()
    for ref in ["search_slime_clusters_gpu_v1", "search_slime_clusters_gpu_v1_centered",
                "search_slime_clusters_gpu_v34", "search_slime_clusters_gpu_v34_centered",
                "refine_candidates_y", "score_candidates_precise", "set_y_scan_config",
                "request_cancel", "request_pause", "resume_search", "reset_cancel", "get_progress",
                "get_processed_centers", "get_gpu_scan_work_ns", "get_cuda_device_count",
                "get_cuda_device_name", "get_gpu_v1_shape", "get_gpu_v1_algorithm",
                "get_gpu_v1_rng", "set_gpu_v1_rng_override", "get_gpu_v34_shape",
                "get_gpu_v34_rng", "set_gpu_v34_rng_override", "cleanup_gpu_resources",
                "is_slime_chunk_c"]:
        assert ref in names, ref


def test_every_declared_symbol_is_exported(lib):
    from slime_b200.lib import SIGNATURES
    for name in declared_functions():
        assert hasattr(lib, name), name
        assert name in SIGNATURES, name


def test_result_record_layout():
    from slime_b200.lib import RESULT_DTYPE
    from oracle.oracle import ExtChunkResult
    assert RESULT_DTYPE.itemsize == 24 == ctypes.sizeof(ExtChunkResult)


def test_control_plane_without_gpu(lib):
    lib.reset_cancel()
    assert lib.get_progress() == 0
    lib.request_pause()
    lib.resume_search()
    lib.request_cancel()
    lib.reset_cancel()
    assert lib.get_processed_centers() == 0
    lib.set_y_scan_config(0, -64, -64, 64, 4)
    assert lib.slime_b200_version().startswith(b"slime_b200")


def test_invalid_arguments_rejected_before_device(lib):
    from slime_b200.lib import RESULT_DTYPE
    buf = np.zeros(4, dtype=RESULT_DTYPE)
    p = buf.ctypes.data_as(ctypes.c_void_p)
    assert lib.search_slime_clusters_gpu_v1_centered(1, -1, 40, 221, 0, 0, 0, p, 4, 0) == -1
    assert lib.search_slime_clusters_gpu_v1_centered(1, 10, 50, 40, 0, 0, 0, p, 4, 0) == -1
    assert lib.search_slime_clusters_gpu_v1_centered(1, 10, 40, 221, 11, 0, 0, p, 4, 0) == -1
    assert lib.search_slime_clusters_gpu_v1_centered(1, 10, 40, 221, 0, 0, 0, None, 4, 0) == -1
    assert lib.search_slime_clusters_gpu_v1_centered(1, 10, 40, 221, 0, 0, 0, p, 0, 0) == -1
    assert lib.search_slime_clusters_gpu_v1_centered(1, (2**31 - 1 - 19) // 2 + 1, 40, 221, 0, 0, 0, p, 4, 0) == -1
    assert lib.search_slime_clusters_gpu_v1_centered(1, 100, 40, 221, 0, 2**31 - 100, 0, p, 4, 0) == -1


def test_engine_rule_round_trip_and_range_checks(lib):
    from slime_b200.lib import RULE_KEYS, SlimeCoreB200
    core = SlimeCoreB200(apply_tuning=False)
    before = core.engine_rule()
    assert set(before) == set(RULE_KEYS)
    try:
        rule = dict(before, band_min_threshold=52, band_fast_periods=5, indep_min_centres=123)
        core.set_engine_rule(rule)
        assert core.engine_rule() == rule
        bad = np.array([27, 7, 56, 4, 44, 10], dtype=np.int64)  # threshold below the band range
        assert lib.slime_b200_set_engine_rule(bad.ctypes.data_as(ctypes.c_void_p), 6) == -1
        assert lib.slime_b200_set_engine_rule(bad.ctypes.data_as(ctypes.c_void_p), 5) == -1
        assert core.engine_rule() == rule
    finally:
        core.set_engine_rule(before)


def test_committed_tuning_file_is_a_valid_rule():
    import json
    from slime_b200.lib import RULE_KEYS, TUNING
    doc = json.loads(TUNING.read_text())
    assert set(doc["rule"]) == set(RULE_KEYS)
    assert 28 <= doc["rule"]["band_min_threshold"] <= 222 and doc["points"]
    for p in doc["points"]:
        assert p["indep_s"] > 0 and p["general_s"] > 0
