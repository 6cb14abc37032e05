"""ctypes bindings for the checkers of the slime-chunk cluster search.

TEST INFRASTRUCTURE ONLY. Two checkers live here:

* ``Oracle``  -- the plain-C restatement in ``slime_oracle.c`` (built into ``_build/``);
* ``RefCpu``  -- the reference's own CPU library ``SlimeCore.cpp`` compiled from its source by
  ``Makefile`` into ``_ref/`` (only where the reference source tree was available at build time;
  the built ``.so`` travels with the repository snapshot).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use them, and only
as checkers or as the timed CPU baseline -- never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libslime_oracle.so"
REF_SO = HERE / "_ref" / "libslimecore_ref.so"
REF_GPU_SO = HERE / "_ref" / "libslimecore_gpu_ref.so"


def reference_dir(ref_dir=None):
    """The reference source tree: the argument, else $SLIME_REFERENCE_DIR, else None (no default)."""
    d = ref_dir if ref_dir is not None else os.environ.get("SLIME_REFERENCE_DIR")
    return Path(d) if d else None


class ExtChunkResult(C.Structure):
    """24-byte result record shared by the reference and this project (SlimeCore.cpp:182-189)."""

    _fields_ = [
        ("size", C.c_int32),
        ("center_x", C.c_int32),
        ("center_z", C.c_int32),
        ("obs_count", C.c_int32),
        ("afk_x", C.c_int32),
        ("afk_z", C.c_int32),
    ]


RESULT_DTYPE = np.dtype(
    [("size", "<i4"), ("center_x", "<i4"), ("center_z", "<i4"), ("obs_count", "<i4"),
     ("afk_x", "<i4"), ("afk_z", "<i4")]
)


class YConfig(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("platform_y", C.c_int32), ("y_min", C.c_int32),
                ("y_max", C.c_int32), ("y_step", C.c_int32)]


def build(ref: bool = True, ref_dir=None) -> None:
    """Build the restatement, and the reference libraries when the reference source tree is given
    (``ref_dir`` or ``$SLIME_REFERENCE_DIR``) and present."""
    subprocess.run(["make", "-C", str(HERE), "oracle"], check=True, capture_output=True)
    src = reference_dir(ref_dir)
    if ref and src is not None and (src / "SlimeCore.cpp").exists():
        subprocess.run(["make", "-C", str(HERE), "ref", "ref_gpu", "ref_biome", "ref_biome_gpu",
                        f"REF_DIR={src}"], check=True, capture_output=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def empty_results(n: int) -> np.ndarray:
    return np.zeros(max(int(n), 1), dtype=RESULT_DTYPE)


class Oracle:
    """The C restatement (slime_oracle.c)."""

    def __init__(self, path: Path = ORACLE_SO):
        if not Path(path).exists():
            build(ref=False)
        lib = C.CDLL(str(path))
        i64, i32, vp = C.c_int64, C.c_int32, C.c_void_p
        lib.oracle_is_slime.argtypes = [i64, i64, i64]
        lib.oracle_is_slime.restype = C.c_int
        lib.oracle_slime_bitmap.argtypes = [i64, i64, i64, i32, i32, vp]
        lib.oracle_window_counts.argtypes = [i64, i64, i64, i32, i32, vp]
        lib.oracle_search_centered.argtypes = [i64, i64, i32, i32, i64, i32, i32, vp, i32, i32,
                                               i32, C.POINTER(YConfig), i32]
        lib.oracle_search_centered.restype = i64
        lib.oracle_score_candidates_precise.argtypes = [i64, vp, i32, i32, C.POINTER(YConfig), i32]
        lib.oracle_refine_candidates_y.argtypes = [i64, vp, i32, C.POINTER(YConfig), i32]
        self.lib = lib

    def is_slime(self, seed: int, cx: int, cz: int) -> bool:
        return bool(self.lib.oracle_is_slime(seed, cx, cz))

    def bitmap(self, seed: int, x0: int, z0: int, w: int, h: int) -> np.ndarray:
        out = np.zeros((h, w), dtype=np.uint8)
        self.lib.oracle_slime_bitmap(seed, x0, z0, w, h, _ptr(out))
        return out

    def window_counts(self, seed: int, cx0: int, cz0: int, w: int, h: int) -> np.ndarray:
        out = np.zeros((h, w), dtype=np.int32)
        self.lib.oracle_window_counts(seed, cx0, cz0, w, h, _ptr(out))
        return out

    def search(self, seed, rd_max, min_size, max_size, rd_min=0, center_x=0, center_z=0,
               max_results=1000, precise_afk=0, precise_limit=100, ycfg=None, threads=0):
        out = empty_results(max_results)
        y = C.byref(ycfg) if ycfg is not None else None
        total = self.lib.oracle_search_centered(seed, rd_max, min_size, max_size, rd_min,
                                                center_x, center_z, _ptr(out), max_results,
                                                precise_afk, precise_limit, y,
                                                threads or os.cpu_count())
        n = 0 if total < 0 else min(total, max_results)
        return total, out[:n].copy()

    def score_precise(self, seed, results: np.ndarray, scan_xz=1, ycfg=None, threads=0):
        buf = np.ascontiguousarray(results, dtype=RESULT_DTYPE).copy()
        y = C.byref(ycfg) if ycfg is not None else None
        self.lib.oracle_score_candidates_precise(seed, _ptr(buf), len(buf), scan_xz, y,
                                                 threads or os.cpu_count())
        return buf

    def refine_y(self, seed, results: np.ndarray, ycfg=None, threads=0):
        buf = np.ascontiguousarray(results, dtype=RESULT_DTYPE).copy()
        y = C.byref(ycfg) if ycfg is not None else None
        self.lib.oracle_refine_candidates_y(seed, _ptr(buf), len(buf), y,
                                            threads or os.cpu_count())
        return buf


class RefCpu:
    """The reference's CPU library, compiled from SlimeCore.cpp (not re-implemented)."""

    def __init__(self, path: Path = REF_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} is not built (needs the reference source tree)")
        lib = C.CDLL(str(path))
        i64, i32, vp = C.c_int64, C.c_int32, C.c_void_p
        lib.search_slime_clusters_centered.argtypes = [i64, i64, i32, i32, i64, i32, i32, vp,
                                                       i32, i32, i32]
        lib.search_slime_clusters_centered.restype = i64
        lib.search_slime_clusters.argtypes = [i64, i64, i32, i32, i64, vp, i32, i32, i32]
        lib.search_slime_clusters.restype = i64
        lib.score_candidates_precise.argtypes = [i64, vp, i32, i32, i32]
        lib.refine_candidates_y.argtypes = [i64, vp, i32, i32]
        lib.set_y_scan_config.argtypes = [i32, i32, i32, i32, i32]
        lib.get_progress.restype = i32
        # build_chunk_cache(int64 seed, int64 ox, int64 oz, uint32 cache[21], int64&, int64&)
        # is an exported C++ symbol (SlimeCore.cpp:234-246): a 21x21 slime bitmap oracle.
        self._bcc = getattr(lib, "_Z17build_chunk_cachelllPjRlS0_")
        self._bcc.argtypes = [i64, i64, i64, vp, C.POINTER(i64), C.POINTER(i64)]
        self._bcc.restype = None
        self.lib = lib

    def chunk_cache(self, seed: int, ox: int, oz: int):
        """21x21 slime bits around block (ox, oz): returns (bits[i][j], base_cx, base_cz)."""
        cache = np.zeros(21, dtype=np.uint32)
        bx, bz = C.c_int64(0), C.c_int64(0)
        self._bcc(seed, ox, oz, _ptr(cache), C.byref(bx), C.byref(bz))
        bits = ((cache[:, None] >> np.arange(21, dtype=np.uint32)[None, :]) & 1).astype(np.uint8)
        return bits, bx.value, bz.value

    def set_y_scan_config(self, enabled=0, platform_y=-64, y_min=-64, y_max=64, y_step=4):
        self.lib.set_y_scan_config(enabled, platform_y, y_min, y_max, y_step)

    def search(self, seed, rd_max, min_size, max_size, rd_min=0, center_x=0, center_z=0,
               max_results=1000, threads=0, precise_afk=0):
        out = empty_results(max_results)
        total = self.lib.search_slime_clusters_centered(seed, rd_max, min_size, max_size, rd_min,
                                                        center_x, center_z, _ptr(out),
                                                        max_results, threads or os.cpu_count(),
                                                        precise_afk)
        n = 0 if total < 0 else min(total, max_results)
        return total, out[:n].copy()

    def score_precise(self, seed, results: np.ndarray, scan_xz=1, threads=0):
        buf = np.ascontiguousarray(results, dtype=RESULT_DTYPE).copy()
        self.lib.score_candidates_precise(seed, _ptr(buf), len(buf), threads or os.cpu_count(),
                                          scan_xz)
        return buf

    def refine_y(self, seed, results: np.ndarray, threads=0):
        buf = np.ascontiguousarray(results, dtype=RESULT_DTYPE).copy()
        self.lib.refine_candidates_y(seed, _ptr(buf), len(buf), threads or os.cpu_count())
        return buf


class RefGpu:
    """The reference's GPU library, compiled from SlimeCoreGPU.cu for sm_100a (a checker for
    areas too large for the CPU). Its cleanup_gpu_resources() resets the device and is never
    called."""

    def __init__(self, path: Path = REF_GPU_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} is not built (needs the reference source tree)")
        lib = C.CDLL(str(path))
        i64, i32, vp = C.c_int64, C.c_int32, C.c_void_p
        lib.search_slime_clusters_gpu_v1_centered.argtypes = [i64, i64, i32, i32, i64, i32, i32,
                                                              vp, i32, i32]
        lib.search_slime_clusters_gpu_v1_centered.restype = i64
        lib.get_processed_centers.restype = i64
        lib.reset_cancel.argtypes = []
        self.lib = lib

    def search(self, seed, rd_max, min_size, max_size, rd_min=0, center_x=0, center_z=0,
               max_results=1000, precise_afk=0):
        out = empty_results(max_results)
        self.lib.reset_cancel()
        total = self.lib.search_slime_clusters_gpu_v1_centered(seed, rd_max, min_size, max_size,
                                                               rd_min, center_x, center_z,
                                                               _ptr(out), max_results, precise_afk)
        n = 0 if total < 0 else min(total, max_results)
        return total, out[:n].copy()


def python_is_slime(seed: int, cx: int, cz: int) -> bool:
    """Pure-Python restatement of the predicate for small cases (SlimeCore.cpp:208-232)."""
    m64 = (1 << 64) - 1
    m48 = (1 << 48) - 1

    def s32(v):
        v &= 0xFFFFFFFF
        return v - (1 << 32) if v & 0x80000000 else v

    x, z = s32(cx), s32(cz)
    mix = (seed + s32(x * x * 0x4C1906) + s32(x * 0x5AC0DB) + s32(z * z) * 0x4307A7
           + s32(z * 0x5F24F)) & m64
    state = (mix ^ 0x3AD8025F ^ 0x5DEECE66D) & m48
    while True:
        state = (state * 0x5DEECE66D + 0xB) & m48
        bits = state >> 17
        val = bits % 10
        if bits - val + 9 <= 0x7FFFFFFF:
            return val == 0


# ---- biome filter checkers -----------------------------------------------------------------------

BIOME_ORACLE_SO = HERE / "_build" / "libbiome_oracle.so"
REF_BIOME_HOST_SO = HERE / "_ref" / "libmcgpu_host_ref.so"
REF_BIOME_GPU_SO = {"fmad": HERE / "_ref" / "libmcgpu_ref_fmad.so",
                    "nofmad": HERE / "_ref" / "libmcgpu_ref_nofmad.so"}


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class _BiomeCalls:
    """Shared call shapes of the biome checkers (prefix `bo_` or `refb_`)."""

    def _bind(self, lib, p):
        u64p = vp = C.c_void_p
        i32 = C.c_int32
        getattr(lib, p + "xoroshiro_nextlong").argtypes = [u64p, i32, i32, vp]
        getattr(lib, p + "xperlin_sample").argtypes = [vp, vp, vp, vp, i32, vp]
        getattr(lib, p + "climate6").argtypes = [C.c_uint64, i32, vp, vp, vp, i32, vp]
        getattr(lib, p + "depth_spline").argtypes = [vp]
        getattr(lib, p + "depth_spline").restype = C.c_float
        getattr(lib, p + "biome_at").argtypes = [i32, C.c_uint64, i32, vp, vp, vp, i32, vp]
        getattr(lib, p + "biome_at").restype = i32
        getattr(lib, p + "filter").argtypes = [i32, C.c_uint64, i32, vp, vp, i32, i32, vp]
        getattr(lib, p + "filter").restype = i32
        self.lib, self.p = lib, p

    def _f(self, name):
        return getattr(self.lib, self.p + name)

    def xoroshiro(self, seeds, steps):
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        out = np.zeros((len(s), steps), dtype=np.uint64)
        self._f("xoroshiro_nextlong")(_ptr(s), len(s), steps, _ptr(out))
        return out

    def perlin(self, seeds, xs, ys, zs):
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (xs, ys, zs))
        out = np.zeros(len(s), dtype=np.float64)
        self._f("xperlin_sample")(_ptr(s), _ptr(x), _ptr(y), _ptr(z), len(s), _ptr(out))
        return out

    def climate6(self, world_seed, xs, ys, zs, large=0):
        x, y, z = _i32(xs), _i32(ys), _i32(zs)
        out = np.zeros((len(x), 6), dtype=np.int32)
        self._f("climate6")(world_seed & (2**64 - 1), large, _ptr(x), _ptr(y), _ptr(z), len(x), _ptr(out))
        return out

    def depth_spline(self, v4):
        v = np.ascontiguousarray(v4, dtype=np.float32)
        return float(self._f("depth_spline")(_ptr(v)))

    def biome_at(self, version, world_seed, xs, ys, zs, large=0):
        x, y, z = _i32(xs), _i32(ys), _i32(zs)
        out = np.zeros(len(x), dtype=np.int32)
        rc = self._f("biome_at")(version, world_seed & (2**64 - 1), large, _ptr(x), _ptr(y), _ptr(z),
                                 len(x), _ptr(out))
        assert rc == 0
        return out

    def filter(self, version, world_seed, cx, cz, flags, large=0):
        x, z = _i32(cx), _i32(cz)
        out = np.zeros(len(x), dtype=np.int32)
        rc = self._f("filter")(version, world_seed & (2**64 - 1), large, _ptr(x), _ptr(z), len(x),
                               flags, _ptr(out))
        assert rc == 0
        return out


class BiomeOracle(_BiomeCalls):
    """The plain-C restatement of the biome filter (biome_oracle.c)."""

    def __init__(self, path: Path = BIOME_ORACLE_SO):
        if not Path(path).exists():
            build(ref=False)
        self._bind(C.CDLL(str(path)), "bo_")


class RefBiomeHost(_BiomeCalls):
    """The reference biome module's own device math compiled for the CPU (ref_biome_host.cpp)."""

    def __init__(self, path: Path = REF_BIOME_HOST_SO):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} is not built (needs the reference source tree)")
        self._bind(C.CDLL(str(path)), "refb_")


class RefBiomeGpu:
    """The reference biome module (MinecraftGPUNoise.cu) built for sm_100a, with (`fmad`) or
    without (`nofmad`) FMA contraction; its own mcgpu_* C ABI."""

    def __init__(self, kind: str = "nofmad"):
        path = REF_BIOME_GPU_SO[kind]
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (needs the reference source tree)")
        lib = C.CDLL(str(path))
        vp, i32, u64 = C.c_void_p, C.c_int32, C.c_uint64
        lib.mcgpu_modern_ctx_create.argtypes = [i32, u64, i32]
        lib.mcgpu_modern_ctx_create.restype = vp
        lib.mcgpu_modern_ctx_create_ex.argtypes = [i32, u64, i32, i32]
        lib.mcgpu_modern_ctx_create_ex.restype = vp
        lib.mcgpu_modern_ctx_filter_candidates.argtypes = [vp, vp, vp, i32, i32, vp]
        lib.mcgpu_modern_ctx_query.argtypes = [vp, vp, vp, vp, i32, vp]
        lib.mcgpu_modern_ctx_destroy.argtypes = [vp]
        lib.mcgpu_xoroshiro_nextlong_batch.argtypes = [vp, i32, i32, vp]
        lib.mcgpu_xperlin_sample_batch.argtypes = [vp, vp, vp, vp, i32, vp]
        lib.mcgpu_climate6_i32_fixed_seed.argtypes = [u64, vp, vp, vp, i32, vp]
        lib.mcgpu_climate6_i32_fixed_seed_ex.argtypes = [u64, i32, vp, vp, vp, i32, vp]
        self.lib = lib

    def filter(self, version, world_seed, cx, cz, flags, large=0):
        x, z = _i32(cx), _i32(cz)
        h = self.lib.mcgpu_modern_ctx_create_ex(version, world_seed & (2**64 - 1), large, len(x))
        assert h
        try:
            out = np.zeros(len(x), dtype=np.int32)
            assert self.lib.mcgpu_modern_ctx_filter_candidates(h, _ptr(x), _ptr(z), len(x), flags, _ptr(out)) == 0
            return out
        finally:
            self.lib.mcgpu_modern_ctx_destroy(h)

    def biome_at(self, version, world_seed, xs, ys, zs, large=0):
        x, y, z = _i32(xs), _i32(ys), _i32(zs)
        h = self.lib.mcgpu_modern_ctx_create_ex(version, world_seed & (2**64 - 1), large, len(x))
        assert h
        try:
            out = np.zeros(len(x), dtype=np.int32)
            assert self.lib.mcgpu_modern_ctx_query(h, _ptr(x), _ptr(y), _ptr(z), len(x), _ptr(out)) == 0
            return out
        finally:
            self.lib.mcgpu_modern_ctx_destroy(h)

    def climate6(self, world_seed, xs, ys, zs, large=0):
        x, y, z = _i32(xs), _i32(ys), _i32(zs)
        out = np.zeros((len(x), 6), dtype=np.int32)
        assert self.lib.mcgpu_climate6_i32_fixed_seed_ex(world_seed & (2**64 - 1), large, _ptr(x), _ptr(y),
                                                         _ptr(z), len(x), _ptr(out)) == 0
        return out

    def xoroshiro(self, seeds, steps):
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        out = np.zeros((len(s), steps), dtype=np.uint64)
        assert self.lib.mcgpu_xoroshiro_nextlong_batch(_ptr(s), len(s), steps, _ptr(out)) == 0
        return out

    def perlin(self, seeds, xs, ys, zs):
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (xs, ys, zs))
        out = np.zeros(len(s), dtype=np.float64)
        assert self.lib.mcgpu_xperlin_sample_batch(_ptr(s), _ptr(x), _ptr(y), _ptr(z), len(s), _ptr(out)) == 0
        return out
