"""GPU parity of the FP64 biome filter (mcgpu_* C ABI of libslime_b200.so).

Bit-exact, no tolerance, against
  * the golden vectors made by the reference's own code compiled for the CPU (tests/golden/biome.npz);
  * the oracle's C restatement on fresh inputs: quarts, real threshold-50 survivors of a search;
  * the reference biome module itself built for sm_100a (oracle/_ref/libmcgpu_ref_{nofmad,fmad}.so)
    on the same survivors and candidates. The --fmad=false build is the reference's arithmetic
    operation by operation; the default (--fmad=true) build lets the compiler fuse multiply-adds,
    which can move a quantised climate parameter by one unit, so against it the verdict masks are
    compared (they agree unless a contraction moves a quart across a biome border) and any
    differing climate parameters are counted, not asserted.
"""
import numpy as np
import pytest

from oracle.oracle import REF_BIOME_GPU_SO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def core():
    from slime_b200 import build
    from slime_b200.lib import SlimeCoreB200
    build.build()
    c = SlimeCoreB200()
    c.set_y_scan_config(0, -64, -64, 64, 4)
    return c


@pytest.fixture(scope="module")
def g():
    from pathlib import Path
    return np.load(Path(__file__).resolve().parent / "golden" / "biome.npz")


def _p(a):
    import ctypes
    return a.ctypes.data_as(ctypes.c_void_p)


def test_abi_basics(core):
    lib = core.lib
    assert lib.mcgpu_api_version() == 1
    assert 32 <= lib.mcgpu_modern_recommended_filter_batch() <= 1024
    assert lib.mcgpu_modern_ctx_create(1179, 1, 16) is None          # before 1.18: no tree
    assert lib.mcgpu_modern_ctx_create(2602, 1, 0) is None           # capacity
    assert lib.mcgpu_modern_ctx_create_ex(2602, 1, 2, 16) is None    # unknown flag
    h = lib.mcgpu_modern_ctx_create(2602, 1, 4)
    assert h
    x = np.zeros(8, dtype=np.int32)
    m = np.zeros(8, dtype=np.int32)
    assert lib.mcgpu_modern_ctx_filter_candidates(h, _p(x), _p(x), 4, 0, _p(m)) == -1   # flags 0
    assert lib.mcgpu_modern_ctx_filter_candidates(h, _p(x), _p(x), 5, 3, _p(m)) == -1   # > capacity
    assert lib.mcgpu_modern_ctx_filter_candidates(h, _p(x), _p(x), 4, 4, _p(m)) == -1   # bad flag
    assert lib.mcgpu_modern_ctx_filter_candidates(h, _p(x), _p(x), 4, 3, _p(m)) == 0
    lib.mcgpu_modern_ctx_destroy(h)


def test_primitives_golden(core, g):
    lib = core.lib
    s = np.ascontiguousarray(g["xr_seeds"])
    out = np.zeros((len(s), 8), dtype=np.uint64)
    assert lib.mcgpu_xoroshiro_nextlong_batch(_p(s), len(s), 8, _p(out)) == 0
    assert np.array_equal(out, g["xr_out"])
    ps = np.ascontiguousarray(g["perlin_seeds"])
    px, py, pz = (np.ascontiguousarray(g[k]) for k in ("perlin_x", "perlin_y", "perlin_z"))
    po = np.zeros(len(ps))
    assert lib.mcgpu_xperlin_sample_batch(_p(ps), _p(px), _p(py), _p(pz), len(ps), _p(po)) == 0
    assert np.array_equal(po.view(np.uint64), g["perlin_out"].view(np.uint64))
    ws = int(g["world_seed"][0])
    for tag, large in (("", 0), ("_large", 1)):
        xyz = np.ascontiguousarray(g[f"c6{tag}_xyz"])
        x, y, z = (np.ascontiguousarray(xyz[:, i]) for i in range(3))
        o6 = np.zeros((len(x), 6), dtype=np.int32)
        assert lib.mcgpu_climate6_i32_fixed_seed_ex(ws, large, _p(x), _p(y), _p(z), len(x), _p(o6)) == 0
        assert np.array_equal(o6, g[f"c6{tag}_out"]), tag
        if not large:
            o5 = np.zeros((len(x), 5), dtype=np.int32)
            assert lib.mcgpu_climate5_i32_fixed_seed(ws, _p(x), _p(z), len(x), _p(o5)) == 0
            assert np.array_equal(o5, g["c6_out"][:, [0, 1, 2, 3, 5]])


def test_fixed_seed_perlin_matches_per_seed_perlin(core, g):
    lib = core.lib
    px, py, pz = (np.ascontiguousarray(g[k]) for k in ("perlin_x", "perlin_y", "perlin_z"))
    seed = int(g["perlin_seeds"][0])
    ps = np.full(len(px), seed, dtype=np.uint64)
    a, b = np.zeros(len(px)), np.zeros(len(px))
    assert lib.mcgpu_xperlin_sample_batch(_p(ps), _p(px), _p(py), _p(pz), len(px), _p(a)) == 0
    assert lib.mcgpu_xperlin_sample_fixed_seed(seed, _p(px), _p(py), _p(pz), len(px), _p(b)) == 0
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_biome_query_golden(core, g):
    from slime_b200.lib import BiomeFilter
    xyz = g["bio_xyz"]
    ws = int(g["world_seed"][0])
    with BiomeFilter(2602, ws, len(xyz), core=core) as f:
        assert np.array_equal(f.query(xyz[:, 0], xyz[:, 1], xyz[:, 2]), g["bio_out"])
    with BiomeFilter(2602, ws, len(xyz), large=1, core=core) as f:
        assert np.array_equal(f.query(xyz[:, 0], xyz[:, 1], xyz[:, 2]), g["bio_large_out"])
    for v, want in zip(g["bio_versions"], g["bio_versions_out"]):
        with BiomeFilter(int(v), ws, 2048, core=core) as f:
            assert np.array_equal(f.query(xyz[:2048, 0], xyz[:2048, 1], xyz[:2048, 2]), want), v
    # The biome20 entry points use the 1.20.6 tree.
    x, y, z = (np.ascontiguousarray(xyz[:2048, i]) for i in range(3))
    out = np.zeros(2048, dtype=np.int32)
    assert core.lib.mcgpu_biome20_i32_fixed_seed(ws, _p(x), _p(y), _p(z), 2048, _p(out)) == 0
    assert np.array_equal(out, g["bio_versions_out"][list(g["bio_versions"]).index(1206)])


@pytest.mark.parametrize("flags,key", [(3, "flt_mask"), (1, "flt_mask_deep"), (2, "flt_mask_mush")])
def test_filter_golden(core, g, flags, key):
    from slime_b200.lib import BiomeFilter
    ws = int(g["world_seed"][0])
    with BiomeFilter(2602, ws, 1024, core=core) as f:
        got = f.filter(g["flt_cx"], g["flt_cz"], flags)
        again = f.filter(g["flt_cx"], g["flt_cz"], flags)
    assert np.array_equal(got, g[key])
    assert np.array_equal(again, got)


def survivors(core, seed, radius=150_000, thr=50, cx=0, cz=0, n=400):
    total, res = core.search(seed, radius, thr, 221, 0, cx, cz, n)
    assert total > 0
    return (res["center_x"] - 8) // 16, (res["center_z"] - 8) // 16


@pytest.fixture(scope="module")
def config4_survivors(core):
    from slime_b200 import workloads
    seeds = workloads.precise_biome_seeds()
    out = []
    for k, (cx, cz) in enumerate([(0, 0), (900_000, -1_200_000), (-1_500_000, 400_000)]):
        s = seeds[k].seed
        x, z = survivors(core, s, cx=cx, cz=cz)
        out.append((s, x, z))
    return out


def test_filter_survivors_vs_oracle(core, config4_survivors):
    from oracle.oracle import BiomeOracle
    from slime_b200.lib import BiomeFilter
    o = BiomeOracle()
    for s, x, z in config4_survivors:
        with BiomeFilter(2602, s, len(x), core=core) as f:
            got = f.filter(x, z, 3)
        want = o.filter(2602, s, x[:160], z[:160], 3)
        assert np.array_equal(got[:160], want), s
        assert (got & 1).any() or (got == 0).all()


@pytest.mark.skipif(not REF_BIOME_GPU_SO["nofmad"].exists(), reason="reference biome build absent")
def test_filter_survivors_vs_reference_gpu(core, config4_survivors, g):
    from oracle.oracle import RefBiomeGpu
    from slime_b200.lib import BiomeFilter
    ref = {k: RefBiomeGpu(k) for k in ("nofmad", "fmad")}
    cases = [(int(g["world_seed"][0]), g["flt_cx"], g["flt_cz"])] + list(config4_survivors)
    differ_fmad = 0
    for s, x, z in cases:
        with BiomeFilter(2602, s, len(x), core=core) as f:
            got = f.filter(x, z, 3)
        assert np.array_equal(got, ref["nofmad"].filter(2602, s, x, z, 3)), s
        differ_fmad += int((got != ref["fmad"].filter(2602, s, x, z, 3)).sum())
    # Masks of the shipped (contracting) build: equal on these candidates.
    assert differ_fmad == 0


@pytest.mark.skipif(not REF_BIOME_GPU_SO["nofmad"].exists(), reason="reference biome build absent")
def test_query_and_climate_vs_reference_gpu(core, g):
    from oracle.oracle import RefBiomeGpu
    from slime_b200.lib import BiomeFilter
    rng = np.random.default_rng(5)
    ws = int(rng.integers(-2**63, 2**63, dtype=np.int64)) & (2**64 - 1)
    n = 20000
    qx = rng.integers(-7_500_000, 7_500_000, n).astype(np.int32)
    qz = rng.integers(-7_500_000, 7_500_000, n).astype(np.int32)
    qy = rng.integers(-16, 17, n).astype(np.int32)
    exact = RefBiomeGpu("nofmad")
    with BiomeFilter(2602, ws, n, core=core) as f:
        ours = f.query(qx, qy, qz)
    assert np.array_equal(ours, exact.biome_at(2602, ws, qx, qy, qz))
    o6 = np.zeros((n, 6), dtype=np.int32)
    assert core.lib.mcgpu_climate6_i32_fixed_seed(ws, _p(qx), _p(qy), _p(qz), n, _p(o6)) == 0
    assert np.array_equal(o6, exact.climate6(ws, qx, qy, qz))
    fm = RefBiomeGpu("fmad")
    c_f = fm.climate6(ws, qx, qy, qz)
    b_f = fm.biome_at(2602, ws, qx, qy, qz)
    print(f"fmad build: {(c_f != o6).any(axis=1).sum()} of {n} quarts differ in a climate parameter, "
          f"{(b_f != ours).sum()} in the biome")
    assert (b_f != ours).sum() <= n // 1000


def reference_filtered(q, ref_gpu_filter, pool=4000):
    """The reference's answer to a biome-filtered search: its own search (reference CPU library up
    to radius 20k, its GPU library above) keeping `pool` ranked sites, the reference biome filter
    (sm_100a build, no contraction) on them, and the first max_results that pass."""
    from dataclasses import replace
    from tests.refcheck import reference_search
    t, recs = reference_search(replace(q, max_results=pool, precise_afk=0))
    cx = (recs["center_x"] - 8) // 16
    cz = (recs["center_z"] - 8) // 16
    mask = ref_gpu_filter.filter(q.biome_version, q.seed, cx, cz, q.biome_flags & 3, (q.biome_flags >> 2) & 1)
    keep = recs[(mask & q.biome_flags & 3) == 0]
    assert len(keep) >= min(q.max_results, t) or len(recs) == t
    return t, keep[: q.max_results]


def biome_searches():
    from slime_b200.workloads import Search
    return [
        Search(seed=-7_123_456_789, center_x=0, center_z=0, radius=20_000, min_size=46, max_results=60, biome_flags=3),
        Search(seed=424242, center_x=-600_000, center_z=350_000, radius=90_000, min_size=52, max_results=40,
               biome_flags=1),
        Search(seed=99, center_x=1_200_000, center_z=-10_000, radius=4_000, min_size=40, max_results=80,
               biome_flags=2),
        Search(seed=-31, center_x=5_000, center_z=5_000, radius=3_000, min_size=38, max_results=50,
               biome_flags=3 | 4),
        Search(seed=2024, center_x=0, center_z=0, radius=150_000, min_size=50, max_results=100, biome_flags=3,
               biome_version=1215),
    ]


@pytest.mark.skipif(not REF_BIOME_GPU_SO["nofmad"].exists(), reason="reference biome build absent")
def test_search_biome_vs_reference(core):
    from oracle.oracle import RefBiomeGpu
    ref = RefBiomeGpu("nofmad")
    for q in biome_searches():
        t, res = core.search_biome(q.seed, q.radius, q.min_size, q.max_size, q.rd_min, q.center_x, q.center_z,
                                   q.max_results, 0, q.biome_flags, q.biome_version)
        t_r, keep = reference_filtered(q, ref)
        assert t == t_r, q
        assert np.array_equal(res, keep), q
    # Without flags it is the plain search.
    q = biome_searches()[0]
    a = core.search_biome(q.seed, q.radius, q.min_size, 221, 0, 0, 0, 500, 0, 0, 0)
    b = core.search(q.seed, q.radius, q.min_size, 221, 0, 0, 0, 500, 0)
    assert a[0] == b[0] and np.array_equal(a[1], b[1])


def test_search_biome_precise_scores(core):
    from tests.refcheck import ref_cpu
    q = biome_searches()[0]
    t, plain = core.search_biome(q.seed, q.radius, q.min_size, 221, 0, 0, 0, q.max_results, 0, 3, 2602)
    t2, scored = core.search_biome(q.seed, q.radius, q.min_size, 221, 0, 0, 0, q.max_results, 1, 3, 2602)
    assert t == t2 and np.array_equal(plain[["size", "center_x", "center_z"]], scored[["size", "center_x", "center_z"]])
    assert np.array_equal(scored, ref_cpu().score_precise(q.seed, plain, scan_xz=1))


def test_batch_and_server_biome_equal_single(core):
    from slime_b200.lib import SlimeServer
    qs = biome_searches()
    singles = [core.search_biome(q.seed, q.radius, q.min_size, q.max_size, q.rd_min, q.center_x, q.center_z,
                                 q.max_results, q.precise_afk, q.biome_flags, q.biome_version) for q in qs]
    batch = core.search_batch(qs)
    for (t, r), (tb, rb) in zip(singles, batch):
        assert t == tb and np.array_equal(r, rb)
    with SlimeServer(core=core) as server:
        tickets = [server.submit(q) for q in qs]
        for tk, q, (t, r) in zip(tickets, qs, singles):
            assert server.wait(tk) == server.DONE
            ts, rs, _ = server.take(tk, q.max_results)
            assert ts == t and np.array_equal(rs, r)


def test_search_biome_rejects_bad_flags(core):
    from slime_b200.lib import RESULT_DTYPE
    buf = np.zeros(4, dtype=RESULT_DTYPE)
    assert core.lib.slime_b200_search_biome(1, 100, 40, 221, 0, 0, 0, _p(buf), 4, 0, 8, 2602) == -1
    assert core.lib.slime_b200_search_biome(1, 100, 40, 221, 0, 0, 0, _p(buf), 4, 0, 3, 1100) == -1
