"""ctypes binding of libslime_b200.so -- the same entry points a ctypes frontend of the reference
GPU library (`slimecore_gpu`) binds, plus this library's additions.

There is no fallback: if the shared library is missing or no CUDA device is usable, calls fail
loudly (the search returns -1 and :class:`SlimeCoreB200` raises).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .build import LIB

RESULT_DTYPE = np.dtype(
    [("size", "<i4"), ("center_x", "<i4"), ("center_z", "<i4"), ("obs_count", "<i4"),
     ("afk_x", "<i4"), ("afk_z", "<i4")]
)

i64, i32, vp, u8p = C.c_int64, C.c_int32, C.c_void_p, C.c_void_p

# name -> (restype, argtypes); one line per symbol of include/slimecore_b200.h.
SIGNATURES = {
    "search_slime_clusters_gpu_v1": (i64, [i64, i64, i32, i32, i64, vp, i32, i32]),
    "search_slime_clusters_gpu_v1_centered": (i64, [i64, i64, i32, i32, i64, i32, i32, vp, i32, i32]),
    "search_slime_clusters_gpu_v34": (i64, [i64, i64, i32, i32, i64, vp, i32, i32]),
    "search_slime_clusters_gpu_v34_centered": (i64, [i64, i64, i32, i32, i64, i32, i32, vp, i32, i32]),
    "refine_candidates_y": (None, [i64, vp, i32]),
    "score_candidates_precise": (None, [i64, vp, i32, i32, i32]),
    "set_y_scan_config": (None, [i32, i32, i32, i32, i32]),
    "request_cancel": (None, []),
    "request_pause": (None, []),
    "resume_search": (None, []),
    "reset_cancel": (None, []),
    "get_progress": (i32, []),
    "get_processed_centers": (i64, []),
    "get_gpu_scan_work_ns": (i64, []),
    "get_cuda_device_count": (i32, []),
    "get_cuda_device_name": (i32, [C.c_char_p, i32]),
    "get_gpu_v1_shape": (i32, []),
    "get_gpu_v1_algorithm": (i32, []),
    "get_gpu_v1_rng": (i32, []),
    "set_gpu_v1_rng_override": (None, [i32]),
    "get_gpu_v34_shape": (i32, []),
    "get_gpu_v34_rng": (i32, []),
    "set_gpu_v34_rng_override": (None, [i32]),
    "cleanup_gpu_resources": (None, []),
    "is_slime_chunk_c": (C.c_bool, [i64, i64, i64]),
    "slime_b200_version": (C.c_char_p, []),
    "slime_b200_last_error": (C.c_char_p, []),
    "slime_b200_last_search_stats": (None, [C.POINTER(C.c_double), C.POINTER(i64)]),
    "slime_b200_is_slime_batch": (i32, [i64, vp, vp, u8p, i64]),
    "slime_b200_last_rare_chunks": (i64, []),
    "slime_b200_set_engine": (None, [i32, i32]),
    "slime_b200_set_tuning": (None, [i32]),
    "slime_b200_set_wait_limit": (i64, [i64]),
    "slime_b200_microbench": (i32, [i32, i32, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "slime_b200_search_noalloc": (i64, [i64, i64, i32, i32, i64, i32, i32, vp, i32]),
    "slime_b200_search_batch": (i32, [vp, i32, vp, vp]),
    "slime_b200_set_engine_rule": (i32, [vp, i32]),
    "slime_b200_get_engine_rule": (i32, [vp, i32]),
    "slime_b200_server_create": (vp, [i64, i32]),
    "slime_b200_server_submit": (i64, [vp, vp]),
    "slime_b200_server_poll": (i32, [vp, i64]),
    "slime_b200_server_wait": (i32, [vp, i64, i32]),
    "slime_b200_server_take": (i64, [vp, i64, vp, i32, C.POINTER(C.c_double)]),
    "slime_b200_server_destroy": (None, [vp]),
    # biome module (the reference's mcgpu_* C ABI, MinecraftGPUNoise.cu:1076-2018)
    "mcgpu_api_version": (C.c_int, []),
    "mcgpu_build_name": (C.c_char_p, []),
    "mcgpu_modern_recommended_filter_batch": (i32, []),
    "mcgpu_xoroshiro_nextlong_batch": (C.c_int, [vp, i32, i32, vp]),
    "mcgpu_xperlin_sample_batch": (C.c_int, [vp, vp, vp, vp, i32, vp]),
    "mcgpu_xperlin_sample_fixed_seed": (C.c_int, [C.c_uint64, vp, vp, vp, i32, vp]),
    "mcgpu_continentalness_noise_fixed_seed": (C.c_int, [C.c_uint64, vp, vp, i32, vp]),
    "mcgpu_climate5_fixed_seed": (C.c_int, [C.c_uint64, vp, vp, i32, vp]),
    "mcgpu_climate5_quant_fixed_seed": (C.c_int, [C.c_uint64, vp, vp, i32, vp]),
    "mcgpu_climate5_i32_fixed_seed": (C.c_int, [C.c_uint64, vp, vp, i32, vp]),
    "mcgpu_climate_ctx_create": (vp, [C.c_uint64, i32]),
    "mcgpu_climate_ctx_query_i32": (C.c_int, [vp, vp, vp, i32, vp]),
    "mcgpu_climate_ctx_destroy": (None, [vp]),
    "mcgpu_climate6_i32_fixed_seed": (C.c_int, [C.c_uint64, vp, vp, vp, i32, vp]),
    "mcgpu_climate6_i32_fixed_seed_ex": (C.c_int, [C.c_uint64, i32, vp, vp, vp, i32, vp]),
    "mcgpu_biome20_i32_fixed_seed": (C.c_int, [C.c_uint64, vp, vp, vp, i32, vp]),
    "mcgpu_biome20_ctx_create": (vp, [C.c_uint64, i32]),
    "mcgpu_biome20_ctx_query": (C.c_int, [vp, vp, vp, vp, i32, vp]),
    "mcgpu_biome20_ctx_destroy": (None, [vp]),
    "mcgpu_modern_ctx_create": (vp, [i32, C.c_uint64, i32]),
    "mcgpu_modern_ctx_create_ex": (vp, [i32, C.c_uint64, i32, i32]),
    "mcgpu_modern_ctx_query": (C.c_int, [vp, vp, vp, vp, i32, vp]),
    "mcgpu_modern_ctx_filter_candidates": (C.c_int, [vp, vp, vp, i32, i32, vp]),
    "mcgpu_modern_ctx_destroy": (None, [vp]),
    "slime_b200_biome_last_stats": (None, [vp, C.POINTER(C.c_double), C.POINTER(i64)]),
    "slime_b200_search_biome": (i64, [i64, i64, i32, i32, i64, i32, i32, vp, i32, i32, i32, i32]),
    "slime_b200_last_biome_stats": (None, [C.POINTER(i64), C.POINTER(i64)]),
}

# SlimeBatchRequest (56 bytes): the arguments of one search of a batch.
REQUEST_DTYPE = np.dtype(
    [("seed", "<i8"), ("rd_max", "<i8"), ("rd_min", "<i8"), ("min_size", "<i4"),
     ("max_size", "<i4"), ("center_x", "<i4"), ("center_z", "<i4"), ("max_results", "<i4"),
     ("precise_afk", "<i4"), ("biome_flags", "<i4"), ("biome_version", "<i4")]
)
assert REQUEST_DTYPE.itemsize == 56


def load(path: Path | str = LIB) -> C.CDLL:
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"{path} is not built; run `python -m slime_b200.build`")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class SlimeError(RuntimeError):
    pass


TUNING = Path(__file__).with_name("tuning_b200.json")
RULE_KEYS = ("band_min_threshold", "band_min_periods", "band_fast_threshold", "band_fast_periods",
             "indep_min_threshold", "indep_min_centres", "exact_below_threshold", "exact_min_centres",
             "grouped_min_threshold", "grouped_min_width", "grouped_max_width", "exact_wide_below_threshold")


class SlimeCoreB200:
    """Pythonic view of the C ABI; every call goes through the exported C functions. The engine
    rule measured by slime_b200/autotune.py (tuning_b200.json) is applied when present."""

    def __init__(self, path: Path | str = LIB, apply_tuning: bool = True):
        self.lib = load(path)
        if apply_tuning and TUNING.exists():
            import json
            self.set_engine_rule(json.loads(TUNING.read_text())["rule"])

    def set_engine_rule(self, rule: dict):
        keys = next(RULE_KEYS[:n] for n in (12, 8, 6) if all(k in rule for k in RULE_KEYS[:n]))
        vals = np.array([int(rule[k]) for k in keys], dtype=np.int64)
        self._check(self.lib.slime_b200_set_engine_rule(_ptr(vals), len(vals)) == 0, "set_engine_rule")

    def engine_rule(self) -> dict:
        vals = np.zeros(len(RULE_KEYS), dtype=np.int64)
        self._check(self.lib.slime_b200_get_engine_rule(_ptr(vals), len(vals)) == 0, "get_engine_rule")
        return dict(zip(RULE_KEYS, (int(v) for v in vals)))

    def _check(self, ok: bool, what: str):
        if not ok:
            raise SlimeError(f"{what} failed: {self.lib.slime_b200_last_error().decode()}")

    def search(self, seed: int, rd_max: int, min_size: int, max_size: int = 221, rd_min: int = 0,
               center_x: int = 0, center_z: int = 0, max_results: int = 1000,
               precise_afk: int = 0, out: np.ndarray | None = None):
        """search_slime_clusters_gpu_v1_centered; returns (total, ranked results)."""
        buf = out if out is not None else np.zeros(max(max_results, 1), dtype=RESULT_DTYPE)
        total = self.lib.search_slime_clusters_gpu_v1_centered(
            seed, rd_max, min_size, max_size, rd_min, center_x, center_z, _ptr(buf), max_results,
            precise_afk)
        self._check(total >= 0, "search")
        return total, buf[: min(total, max_results)]

    def search_batch(self, searches):
        """slime_b200_search_batch over objects with the fields of workloads.Search; returns a
        list of (total, ranked results), one per search."""
        req = np.zeros(len(searches), dtype=REQUEST_DTYPE)
        for i, q in enumerate(searches):
            req[i] = _request(q)[0]
        offs = np.concatenate([[0], np.cumsum(req["max_results"].astype(np.int64))])
        buf = np.zeros(max(int(offs[-1]), 1), dtype=RESULT_DTYPE)
        totals = np.zeros(max(len(searches), 1), dtype=np.int64)
        rc = self.lib.slime_b200_search_batch(_ptr(req), len(searches), _ptr(buf), _ptr(totals))
        self._check(rc == 0, "search_batch")
        out = []
        for i in range(len(searches)):
            t = int(totals[i])
            n = 0 if t < 0 else min(t, int(req["max_results"][i]))
            out.append((t, passing(buf[offs[i]:offs[i] + n].copy())))
        return out

    def search_biome(self, seed: int, rd_max: int, min_size: int, max_size: int = 221, rd_min: int = 0,
                     center_x: int = 0, center_z: int = 0, max_results: int = 1000, precise_afk: int = 0,
                     biome_flags: int = 3, biome_version: int = 2602):
        """slime_b200_search_biome: the search with sites whose window holds Deep Dark (flag 1) /
        Mushroom Fields (flag 2) excluded; returns (total, ranked results)."""
        buf = np.zeros(max(max_results, 1), dtype=RESULT_DTYPE)
        total = self.lib.slime_b200_search_biome(seed, rd_max, min_size, max_size, rd_min, center_x, center_z,
                                                  _ptr(buf), max_results, precise_afk, biome_flags, biome_version)
        self._check(total >= 0, "search_biome")
        return total, passing(buf[: min(total, max_results)])

    def score_precise(self, seed: int, sites: np.ndarray, scan_xz: int = 1) -> np.ndarray:
        buf = np.ascontiguousarray(sites, dtype=RESULT_DTYPE).copy()
        self.lib.score_candidates_precise(seed, _ptr(buf), len(buf), 0, scan_xz)
        return buf

    def refine_y(self, seed: int, sites: np.ndarray) -> np.ndarray:
        buf = np.ascontiguousarray(sites, dtype=RESULT_DTYPE).copy()
        self.lib.refine_candidates_y(seed, _ptr(buf), len(buf))
        return buf

    def set_y_scan_config(self, enabled=0, platform_y=-64, y_min=-64, y_max=64, y_step=4):
        self.lib.set_y_scan_config(enabled, platform_y, y_min, y_max, y_step)

    def is_slime_batch(self, seed: int, x: np.ndarray, z: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.int64)
        z = np.ascontiguousarray(z, dtype=np.int64)
        out = np.zeros(len(x), dtype=np.uint8)
        self._check(self.lib.slime_b200_is_slime_batch(seed, _ptr(x), _ptr(z), _ptr(out), len(x)) == 0,
                    "is_slime_batch")
        return out

    def last_search_stats(self):
        ms, n = C.c_double(), C.c_int64()
        self.lib.slime_b200_last_search_stats(C.byref(ms), C.byref(n))
        return ms.value, n.value

    def microbench(self, kind: int, iters: int = 4096):
        ops, ms = C.c_double(), C.c_double()
        self._check(self.lib.slime_b200_microbench(kind, iters, C.byref(ops), C.byref(ms)) == 0,
                    "microbench")
        return ops.value, ms.value


def _request(q) -> np.ndarray:
    req = np.zeros(1, dtype=REQUEST_DTYPE)
    flags = getattr(q, "biome_flags", 0)
    req[0] = (q.seed, q.radius, q.rd_min, q.min_size, q.max_size, q.center_x, q.center_z,
              q.max_results, q.precise_afk, flags, getattr(q, "biome_version", 2602) if flags else 0)
    return req


class SlimeServer:
    """The search server of the C ABI (slime_b200_server_*): submit requests, poll or wait for
    tickets, take results with their submission-to-completion latency."""

    QUEUED, RUNNING, DONE, FAILED, UNKNOWN = 0, 1, 2, -1, -2

    def __init__(self, device_bytes: int = 8 << 30, tiles_per_step: int = 0,
                 core: SlimeCoreB200 | None = None):
        self.core = core or SlimeCoreB200()
        self.lib = self.core.lib
        self.handle = self.lib.slime_b200_server_create(device_bytes, tiles_per_step)
        if not self.handle:
            raise SlimeError("server_create failed: " + self.lib.slime_b200_last_error().decode())

    def submit(self, q) -> int:
        t = self.lib.slime_b200_server_submit(self.handle, _ptr(_request(q)))
        if t < 0:
            raise SlimeError("server_submit: invalid request")
        return t

    def poll(self, ticket: int) -> int:
        return self.lib.slime_b200_server_poll(self.handle, ticket)

    def wait(self, ticket: int, timeout_ms: int = 600_000) -> int:
        return self.lib.slime_b200_server_wait(self.handle, ticket, timeout_ms)

    def take(self, ticket: int, max_results: int):
        """(total, ranked results, latency ms) of a finished ticket; total -1 if it failed."""
        buf = np.zeros(max(max_results, 1), dtype=RESULT_DTYPE)
        lat = C.c_double()
        total = self.lib.slime_b200_server_take(self.handle, ticket, _ptr(buf), max_results,
                                                C.byref(lat))
        if total == -2:
            raise SlimeError(f"ticket {ticket} is not finished")
        n = 0 if total < 0 else min(total, max_results)
        return total, passing(buf[:n].copy()), lat.value

    def close(self):
        if self.handle:
            self.lib.slime_b200_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def passing(records: np.ndarray) -> np.ndarray:
    """The records before the first with size -1 (the end of a biome-filtered result list)."""
    end = np.flatnonzero(records["size"] < 0)
    return records[: end[0]] if len(end) else records


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


class BiomeFilter:
    """A biome context of the C ABI (mcgpu_modern_ctx_*): one world seed, Minecraft version code
    and biome size. filter() returns the Deep Dark (bit 0) / Mushroom Fields (bit 1) verdict mask
    of candidate centre chunks, query() biome ids of quarts."""

    def __init__(self, version: int, world_seed: int, capacity: int, large: int = 0,
                 core: SlimeCoreB200 | None = None):
        self.core = core or SlimeCoreB200()
        self.lib = self.core.lib
        self.capacity = capacity
        self.handle = self.lib.mcgpu_modern_ctx_create_ex(version, world_seed & (2**64 - 1), large, capacity)
        if not self.handle:
            raise SlimeError("mcgpu_modern_ctx_create_ex failed: " + self.lib.slime_b200_last_error().decode())

    def filter(self, cx, cz, flags: int = 3) -> np.ndarray:
        x, z = _i32(cx), _i32(cz)
        out = np.zeros(max(len(x), 1), dtype=np.int32)
        rc = self.lib.mcgpu_modern_ctx_filter_candidates(self.handle, _ptr(x), _ptr(z), len(x), flags, _ptr(out))
        if rc != 0:
            raise SlimeError(f"filter_candidates: {rc} {self.lib.slime_b200_last_error().decode()}")
        return out[: len(x)]

    def query(self, xs, ys, zs) -> np.ndarray:
        x, y, z = _i32(xs), _i32(ys), _i32(zs)
        out = np.zeros(max(len(x), 1), dtype=np.int32)
        rc = self.lib.mcgpu_modern_ctx_query(self.handle, _ptr(x), _ptr(y), _ptr(z), len(x), _ptr(out))
        if rc != 0:
            raise SlimeError(f"query: {rc} {self.lib.slime_b200_last_error().decode()}")
        return out[: len(x)]

    def last_stats(self):
        ms, n = C.c_double(), C.c_int64()
        self.lib.slime_b200_biome_last_stats(self.handle, C.byref(ms), C.byref(n))
        return ms.value, n.value

    def close(self):
        if self.handle:
            self.lib.mcgpu_modern_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
