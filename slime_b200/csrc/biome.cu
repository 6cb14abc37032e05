// biome.cu -- the FP64 biome filter (Deep Dark / Mushroom Fields exclusion) and the reference's
// biome-module C ABI (mcgpu_*, gpu_noise/MinecraftGPUNoise.cu:1076-2018, mcgpu.h).
//
// Compiled with --fmad=false (slime_b200/build.py): every floating-point operation is one IEEE
// operation in source order, as in the reference's source text, so climate parameters and biome
// ids are bit-exact with the reference's arithmetic (the noise math is in biome_math.cuh).
//
// The filter of a set of candidate centres (B200 layout, results identical to the reference's
// block-per-candidate kernel, MinecraftGPUNoise.cu:978-1074):
//   1. count_kernel / insert_kernel -- one warp per candidate tests the 221 cells of its window
//      for slime chunks and inserts every slime chunk into a device hash set, so a chunk shared by
//      neighbouring candidates is evaluated once (high-count sites come in clusters);
//   2. chunk_kernel -- one thread per (unique chunk, quart): the column's climate noise once
//      (FP64, 46 octaves in shared memory), then one multi-query tree traversal answers the 17
//      Deep Dark layers (quart Y -16..0) and the Mushroom Fields layer (quart Y 16) together,
//      since they differ only in the depth parameter; verdict bits are OR-ed per chunk;
//   3. verdict_kernel -- one warp per candidate ORs the verdicts of its window's slime chunks.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "biome_math.cuh"
#include "driver.h"

namespace slime {
namespace biome {

// ---- host-side set-up -----------------------------------------------------------------------

// Improved-noise octave from its Xoroshiro state: offsets, the permutation (Fisher-Yates with
// nextInt) and the y = 0 cell, fraction and fade (MinecraftGPUNoise.cu:80-105).
__host__ __device__ inline void perlin_init(Octave& p, Xr xr) {
    p.ox = xr_next_double(xr) * 256.0;
    p.oy = xr_next_double(xr) * 256.0;
    p.oz = xr_next_double(xr) * 256.0;
    for (int i = 0; i < 256; ++i) p.perm[i] = (uint8_t)i;
    for (int i = 0; i < 256; ++i) {
        const int j = (int)xr_next_int(xr, (uint32_t)(256 - i)) + i;
        const uint8_t t = p.perm[i];
        p.perm[i] = p.perm[j];
        p.perm[j] = t;
    }
    p.perm[256] = p.perm[0];
    const double cell = floor(p.oy);
    p.y_cell = (uint8_t)(int)cell;
    p.y_frac = p.oy - cell;
    p.y_fade = fade(p.y_frac);
    p.amp = 1.0;
    p.lac = 1.0;
}

// One octave set (MinecraftGPUNoise.cu:255-282): lacunarity 2^first doubling per octave,
// amplitude amp_i * 2^(n-1-i) / (2^n - 1); octave k seeded with the hash of "octave_<k>".
void octave_set_init(Octave* out, Xr& parent, const double* amp, int first, int n, int* count) {
    double lac = std::ldexp(1.0, first);
    double persist = std::ldexp(1.0, n - 1) / (std::ldexp(1.0, n) - 1.0);
    const uint64_t lo = xr_next(parent), hi = xr_next(parent);
    int m = 0;
    for (int i = 0; i < n; ++i, lac *= 2.0, persist *= 0.5) {
        if (amp[i] == 0.0) continue;
        const int k = 16 + first + i;
        perlin_init(out[m], Xr{lo ^ BD_OCTAVE_HASH[k][0], hi ^ BD_OCTAVE_HASH[k][1]});
        out[m].amp = amp[i] * persist;
        out[m].lac = lac;
        ++m;
    }
    *count = m;
}

// The six climate noises of a world seed (MinecraftGPUNoise.cu:324-405): each a double-Perlin
// noise (two octave sets from one parent seeded by the hash of its name) with amplitude factor
// 5n / (3(n+1)) over the n octaves between its first and last non-zero amplitude.
void climate_init(Climate& c, uint64_t world_seed, bool large) {
    std::memset(&c, 0, sizeof(c));
    Xr base = xr_seed(world_seed);
    const uint64_t lo = xr_next(base), hi = xr_next(base);
    int off = 0;
    for (int s = 0; s < 6; ++s) {
        const BdClimateNoise& d = BD_CLIMATE[s];
        const int li = large ? 1 : 0;
        Xr xr{lo ^ d.hash[li][0], hi ^ d.hash[li][1]};
        int na = 0, nb = 0;
        octave_set_init(c.oct + off, xr, d.amp, d.first_octave[li], d.octaves, &na);
        octave_set_init(c.oct + off + na, xr, d.amp, d.first_octave[li], d.octaves, &nb);
        c.noise[s] = Noise{off, na, nb, 0, 0.0};
        off += na + nb;
        int lead = 0, last = d.octaves;
        while (last > 0 && d.amp[last - 1] == 0.0) --last;
        while (lead < last && d.amp[lead] == 0.0) ++lead;
        const int span = last - lead;
        c.noise[s].amp = (double)(5 * span) / (double)(3 * (span + 1));
    }
}

namespace {

constexpr int kThreads = 128;
constexpr int kParamSlots = 256;  // node words index parameter ranges with 8 bits
constexpr uint64_t kEmptyKey = ~0ull;
constexpr int kDeepLayers = 17;   // quart Y -16..0
constexpr int32_t kDeepDark = 183, kMushroom = 14;

// Per-device tables: the depth spline and every vendored biome tree (nodes with patches
// applied, parameter ranges), uploaded once.
struct Tables {
    bool ready = false;
    SplineHead* heads = nullptr;
    SplinePt* pts = nullptr;
    uint64_t* nodes[BD_TREES] = {};
    int2* params[BD_TREES] = {};
    TreeGeom geom[BD_TREES] = {};
};

Tables& tables() {
    static Tables t;
    return t;
}

float bits_to_float(int32_t b) {
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

}  // namespace

int tree_index(int32_t version) {
    int k = -1;
    for (int i = 0; i < BD_TREES; ++i)
        if (version >= BD_TREE[i].version_from) k = i;
    return k;
}

namespace {

// Under the library lock, with the library's stream.
bool ensure_tables() {
    Tables& t = tables();
    if (t.ready) return true;
    Context& c = ctx();
    if (!c.ensure_device()) return false;
    std::vector<SplineHead> heads(BD_SPLINES);
    std::vector<SplinePt> pts(BD_SPLINE_POINTS);
    for (int s = 0; s < BD_SPLINES; ++s)
        heads[s] = SplineHead{BD_SPLINE_HEAD[s][0], BD_SPLINE_HEAD[s][1], BD_SPLINE_HEAD[s][2], 0};
    for (int i = 0; i < BD_SPLINE_POINTS; ++i)
        pts[i] = SplinePt{bits_to_float(BD_SPLINE_PTS[i][0]), bits_to_float(BD_SPLINE_PTS[i][1]),
                          bits_to_float(BD_SPLINE_PTS[i][2]), BD_SPLINE_PTS[i][3]};
    cudaError_t e;
    if ((e = cudaMalloc(&t.heads, sizeof(SplineHead) * heads.size())) != cudaSuccess ||
        (e = cudaMalloc(&t.pts, sizeof(SplinePt) * pts.size())) != cudaSuccess ||
        (e = cudaMemcpy(t.heads, heads.data(), sizeof(SplineHead) * heads.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(t.pts, pts.data(), sizeof(SplinePt) * pts.size(), cudaMemcpyHostToDevice)) != cudaSuccess) {
        c.set_error("biome tables", e);
        return false;
    }
    for (int k = 0; k < BD_TREES; ++k) {
        const BdTree& b = BD_TREE[k];
        // The tree search packs a node index (16 bits), a child count (8) and a depth (8) per
        // stack level.
        if (b.depth > 8 || b.nparams > kParamSlots || b.order > 255 || b.nnodes + b.steps[0] > 65535) {
            c.set_error_text("biome tables: tree shape out of range");
            return false;
        }
        std::vector<uint64_t> nodes(b.node, b.node + b.nnodes);
        for (int i = 0; i < b.npatch; ++i) nodes[(size_t)b.patch[i][0]] = b.patch[i][1];
        std::vector<int2> param(kParamSlots, make_int2(0, 0));
        for (int i = 0; i < b.nparams; ++i) param[i] = make_int2(b.param[i][0], b.param[i][1]);
        TreeGeom g{};
        g.order = b.order;
        g.depth = b.depth;
        g.nnodes = b.nnodes;
        g.nparams = b.nparams;
        for (int d = 0; d < b.depth; ++d) g.steps[d] = b.steps[d];
        t.geom[k] = g;
        if ((e = cudaMalloc(&t.nodes[k], 8 * nodes.size())) != cudaSuccess ||
            (e = cudaMalloc(&t.params[k], sizeof(int2) * param.size())) != cudaSuccess ||
            (e = cudaMemcpy(t.nodes[k], nodes.data(), 8 * nodes.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
            (e = cudaMemcpy(t.params[k], param.data(), sizeof(int2) * param.size(), cudaMemcpyHostToDevice)) != cudaSuccess) {
            c.set_error("biome tables", e);
            return false;
        }
    }
    t.ready = true;
    return true;
}

// ---- kernels --------------------------------------------------------------------------------

// Shared-memory copy of what every thread samples: the climate octaves, the spline and the tree's
// parameter ranges (node words stay in global memory, read through L1).
struct __align__(16) Shared {
    Climate cl;
    SplineHead heads[BD_SPLINES];
    SplinePt pts[BD_SPLINE_POINTS];
    int2 param[kParamSlots];
};

__device__ __forceinline__ void load_shared(Shared& sh, const Climate* cl, const SplineHead* heads,
                                            const SplinePt* pts, const int2* param) {
    {
        const uint4* src = reinterpret_cast<const uint4*>(cl);
        uint4* dst = reinterpret_cast<uint4*>(&sh.cl);
        for (int i = threadIdx.x; i < (int)(sizeof(Climate) / 16); i += blockDim.x) dst[i] = src[i];
    }
    for (int i = threadIdx.x; i < BD_SPLINES; i += blockDim.x) sh.heads[i] = heads[i];
    for (int i = threadIdx.x; i < BD_SPLINE_POINTS; i += blockDim.x) sh.pts[i] = pts[i];
    if (param)
        for (int i = threadIdx.x; i < kParamSlots; i += blockDim.x) sh.param[i] = param[i];
    __syncthreads();
}

// The 221 cells of the AFK window (dx^2 + dz^2 <= 68), as (dx + 8) * 17 + (dz + 8).
__constant__ uint16_t c_window[221];

__device__ __forceinline__ int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }

__device__ __forceinline__ uint64_t chunk_key(int32_t x, int32_t z) {
    return ((uint64_t)(uint32_t)x << 32) | (uint32_t)z;
}

__device__ __forceinline__ uint32_t key_hash(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (uint32_t)k;
}

// Number of slime chunks in the windows of all candidates (an upper bound of the unique ones).
__global__ void __launch_bounds__(kThreads) count_kernel(int64_t seed, const int32_t* __restrict__ cx,
                                                         const int32_t* __restrict__ cz, int32_t n,
                                                         unsigned long long* total) {
    const int warp = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int32_t x0 = cx[warp], z0 = cz[warp];
    uint32_t m = 0;
    for (int i = lane; i < 221; i += 32) {
        const int c = c_window[i];
        m += is_slime(seed, wrap_add(x0, c / 17 - 8), wrap_add(z0, c % 17 - 8)) ? 1u : 0u;
    }
    m = __reduce_add_sync(0xffffffffu, m);
    if (lane == 0 && m) atomicAdd(total, (unsigned long long)m);
}

struct HashSet {
    uint64_t* keys;         // cap slots, kEmptyKey when free
    int32_t* vals;          // unique index of the key in the slot
    uint32_t mask;          // cap - 1 (cap a power of two, at least twice the insertions)
    int2* uniq;             // unique chunks in insertion order
    unsigned int* nuniq;
    int32_t* special;       // unique index of the one key equal to kEmptyKey (-1 if none)
    unsigned int* error;    // set when a probe sequence runs past the table size
};

__device__ __forceinline__ void hash_insert(const HashSet& h, int32_t x, int32_t z) {
    const uint64_t key = chunk_key(x, z);
    if (key == kEmptyKey) {
        if (atomicCAS(h.special, -1, -2) == -1) {
            const unsigned u = atomicAdd(h.nuniq, 1u);
            h.uniq[u] = make_int2(x, z);
            atomicExch(h.special, (int32_t)u);
        }
        return;
    }
    uint32_t s = key_hash(key) & h.mask;
    for (uint32_t probe = 0; probe <= h.mask; ++probe, s = (s + 1) & h.mask) {
        const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(&h.keys[s]),
                                                  (unsigned long long)kEmptyKey, (unsigned long long)key);
        if (prev == kEmptyKey) {
            const unsigned u = atomicAdd(h.nuniq, 1u);
            h.uniq[u] = make_int2(x, z);
            h.vals[s] = (int32_t)u;
            return;
        }
        if (prev == key) return;
    }
    atomicOr(h.error, 1u);
}

__device__ __forceinline__ int32_t hash_find(const HashSet& h, int32_t x, int32_t z) {
    const uint64_t key = chunk_key(x, z);
    if (key == kEmptyKey) return *h.special;
    uint32_t s = key_hash(key) & h.mask;
    for (uint32_t probe = 0; probe <= h.mask; ++probe, s = (s + 1) & h.mask) {
        const uint64_t k = h.keys[s];
        if (k == key) return h.vals[s];
        if (k == kEmptyKey) break;
    }
    return -1;
}

__global__ void __launch_bounds__(kThreads) insert_kernel(int64_t seed, const int32_t* __restrict__ cx,
                                                          const int32_t* __restrict__ cz, int32_t n, HashSet h) {
    const int warp = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int32_t x0 = cx[warp], z0 = cz[warp];
    for (int i = lane; i < 221; i += 32) {
        const int c = c_window[i];
        const int32_t x = wrap_add(x0, c / 17 - 8), z = wrap_add(z0, c % 17 - 8);
        if (is_slime(seed, x, z)) hash_insert(h, x, z);
    }
}

// Verdict bits of the quart columns of unique chunks: bit 0 Deep Dark at some quart Y -16..0,
// bit 1 Mushroom Fields at quart Y 16. NQ queries: 18 (both), 17 (Deep Dark), 1 (Mushroom).
// Four CTAs per SM (128 registers, no spills): the traversal is latency-bound; twice the warps of
// the register-limited default (200 registers) ran 23 % more quart columns per second on B200 in a
// back-to-back comparison on one GPU.
template <int NQ>
__global__ void __launch_bounds__(kThreads, 4) chunk_kernel(const Climate* __restrict__ cl, const SplineHead* heads,
                                                         const SplinePt* pts, const uint64_t* __restrict__ nodes,
                                                         const int2* __restrict__ param, TreeGeom g,
                                                         const int2* __restrict__ chunks, int32_t nchunks,
                                                         unsigned int* chunk_bits, uint32_t want) {
    __shared__ Shared sh;
    load_shared(sh, cl, heads, pts, param);
    const int64_t items = (int64_t)nchunks * 16;
    for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < items;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = (int32_t)(it >> 4), q = (int32_t)(it & 15);
        if ((*(volatile unsigned int*)&chunk_bits[u] & want) == want) continue;
        const int2 ch = chunks[u];
        const int32_t qx = (int32_t)((uint32_t)ch.x * 4u + (uint32_t)(q >> 2));
        const int32_t qz = (int32_t)((uint32_t)ch.y * 4u + (uint32_t)(q & 3));
        const Column col = column_climate<BD_SPLINE_LEVELS>(sh.cl, sh.heads, sh.pts, qx, qz);
        const int32_t base[5] = {col.t, col.h, col.c, col.e, col.w};
        int32_t depth[NQ], biome[NQ];
        if constexpr (NQ == 1) {
            depth[0] = depth_at(col.off, 16);
        } else {
#pragma unroll
            for (int i = 0; i < kDeepLayers; ++i) depth[i] = depth_at(col.off, -16 + i);
            if constexpr (NQ == kDeepLayers + 1) depth[kDeepLayers] = depth_at(col.off, 16);
        }
        tree_nearest<NQ>(nodes, sh.param, g, base, depth, biome);
        uint32_t bits = 0;
        if constexpr (NQ == 1) {
            bits = biome[0] == kMushroom ? 2u : 0u;
        } else {
#pragma unroll
            for (int i = 0; i < kDeepLayers; ++i) bits |= biome[i] == kDeepDark ? 1u : 0u;
            if constexpr (NQ == kDeepLayers + 1) bits |= biome[kDeepLayers] == kMushroom ? 2u : 0u;
        }
        if (bits) atomicOr(&chunk_bits[u], bits);
    }
}

__global__ void __launch_bounds__(kThreads) verdict_kernel(int64_t seed, const int32_t* __restrict__ cx,
                                                           const int32_t* __restrict__ cz, int32_t n, HashSet h,
                                                           const unsigned int* __restrict__ chunk_bits,
                                                           uint32_t want, int32_t* mask) {
    const int warp = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int32_t x0 = cx[warp], z0 = cz[warp];
    uint32_t m = 0;
    for (int i = lane; i < 221; i += 32) {
        const int c = c_window[i];
        const int32_t x = wrap_add(x0, c / 17 - 8), z = wrap_add(z0, c % 17 - 8);
        if (!is_slime(seed, x, z)) continue;
        const int32_t u = hash_find(h, x, z);
        if (u < 0) atomicOr(h.error, 2u);
        else m |= chunk_bits[u];
    }
    m = __reduce_or_sync(0xffffffffu, m);
    if (lane == 0) mask[warp] = (int32_t)(m & want);
}

// Biome ids of single quarts (x, y, z).
__global__ void __launch_bounds__(kThreads) query_kernel(const Climate* __restrict__ cl, const SplineHead* heads,
                                                         const SplinePt* pts, const uint64_t* __restrict__ nodes,
                                                         const int2* __restrict__ param, TreeGeom g,
                                                         const int32_t* __restrict__ xs, const int32_t* __restrict__ ys,
                                                         const int32_t* __restrict__ zs, int32_t n, int32_t* out) {
    __shared__ Shared sh;
    load_shared(sh, cl, heads, pts, param);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const Column col = column_climate<BD_SPLINE_LEVELS>(sh.cl, sh.heads, sh.pts, xs[i], zs[i]);
        const int32_t base[5] = {col.t, col.h, col.c, col.e, col.w};
        const int32_t depth[1] = {depth_at(col.off, ys[i])};
        int32_t biome[1];
        tree_nearest<1>(nodes, sh.param, g, base, depth, biome);
        out[i] = biome[0];
    }
}

// Climate parameters of points. mode 0: 6 quantised {T, H, C, E, depth, W} of int quarts
// (climate6, MinecraftGPUNoise.cu:811-866); 1: 5 quantised {T, H, C, E, W} of int quarts
// (climate5_i32, :616-642); 2: 5 quantised of double points (climate5_quant, :588-614);
// 3: 5 doubles of double points (climate5, :532-558); 4: continentalness noise of double
// points (continentalness_sample_kernel, :498-516).
__global__ void __launch_bounds__(kThreads) climate_kernel(const Climate* __restrict__ cl, const SplineHead* heads,
                                                           const SplinePt* pts, int mode, const void* xs_, const void* ys_,
                                                           const void* zs_, int32_t n, void* out_) {
    __shared__ Shared sh;
    load_shared(sh, cl, heads, pts, nullptr);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double x, z;
        if (mode <= 1) {
            x = (double)static_cast<const int32_t*>(xs_)[i];
            z = (double)static_cast<const int32_t*>(zs_)[i];
        } else {
            x = static_cast<const double*>(xs_)[i];
            z = static_cast<const double*>(zs_)[i];
        }
        if (mode == 4) {
            static_cast<double*>(out_)[i] = noise_sample(sh.cl, kCont, x, 0.0, z);
            continue;
        }
        const double px = x + noise_sample(sh.cl, kShift, x, 0.0, z) * 4.0;
        const double pz = z + noise_sample(sh.cl, kShift, z, x, 0.0) * 4.0;
        const double c = noise_sample(sh.cl, kCont, px, 0.0, pz);
        const double e = noise_sample(sh.cl, kEros, px, 0.0, pz);
        const double w = noise_sample(sh.cl, kWeird, px, 0.0, pz);
        const double t = noise_sample(sh.cl, kTemp, px, 0.0, pz);
        const double h = noise_sample(sh.cl, kHumid, px, 0.0, pz);
        if (mode == 3) {
            double* o = static_cast<double*>(out_) + i * 5;
            o[0] = t; o[1] = h; o[2] = c; o[3] = e; o[4] = w;
            continue;
        }
        const float cf = (float)c, ef = (float)e, wf = (float)w, tf = (float)t, hf = (float)h;
        if (mode == 0) {
            const float in[4] = {cf, ef, peaks_valleys(wf), wf};
            const float off = spline_eval<BD_SPLINE_LEVELS>(sh.heads, sh.pts, 0, in) + 0.015f;
            int32_t* o = static_cast<int32_t*>(out_) + i * 6;
            o[0] = (int32_t)(10000.0f * tf);
            o[1] = (int32_t)(10000.0f * hf);
            o[2] = (int32_t)(10000.0f * cf);
            o[3] = (int32_t)(10000.0f * ef);
            o[4] = depth_at(off, static_cast<const int32_t*>(ys_)[i]);
            o[5] = (int32_t)(10000.0f * wf);
        } else {
            int32_t* o = static_cast<int32_t*>(out_) + i * 5;
            o[0] = (int32_t)(10000.0f * tf);
            o[1] = (int32_t)(10000.0f * hf);
            o[2] = (int32_t)(10000.0f * cf);
            o[3] = (int32_t)(10000.0f * ef);
            o[4] = (int32_t)(10000.0f * wf);
        }
    }
}

// Xoroshiro128++ draws: steps nextLong values per seed (xoroshiro_batch_kernel, :424-442).
__global__ void xoroshiro_kernel(const uint64_t* __restrict__ seeds, int32_t n, int32_t steps, uint64_t* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Xr s = xr_seed(seeds[i]);
    for (int32_t j = 0; j < steps; ++j) out[i * steps + j] = xr_next(s);
}

// One improved-noise sample per (seed, point): the octave is initialised per thread
// (xperlin_sample_batch_kernel, :444-459), or shared by all points (fixed seed, :466-496).
__global__ void perlin_kernel(const uint64_t* __restrict__ seeds, const Octave* fixed, const double* __restrict__ xs,
                              const double* __restrict__ ys, const double* __restrict__ zs, int32_t n, double* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (fixed) {
        out[i] = perlin_sample(*fixed, xs[i], ys[i], zs[i]);
        return;
    }
    Octave p;
    perlin_init(p, xr_seed(seeds[i]));
    out[i] = perlin_sample(p, xs[i], ys[i], zs[i]);
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t reserve(size_t want, cudaStream_t s) {
        if (want <= n) return cudaSuccess;
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
        const cudaError_t e = cudaMallocAsync(&p, want * sizeof(T), s);
        if (e == cudaSuccess) n = want;
        return e;
    }
    void release(cudaStream_t s) {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
};

bool window_table_ready = false;

}  // namespace

// ---- the filter ---------------------------------------------------------------------------------

// A biome context: one world seed, version and biome size; the climate octaves on the device and
// the work buffers of the filter (grown on demand).
struct BiomeContext {
    int32_t version = 0, tree = -1, large = 0, capacity = 0;
    uint64_t world_seed = 0;
    Climate* d_climate = nullptr;
    DevBuf<int32_t> x, y, z, out;
    DevBuf<uint64_t> keys;
    DevBuf<int32_t> vals;
    DevBuf<int2> uniq;
    DevBuf<unsigned int> chunk_bits, counters;  // counters: [0..1] total (u64), [2] nuniq, [3] error, [4] special
    double last_ms = 0.0;
    int64_t last_unique = 0;
};

namespace {

bool ensure_window_table() {
    if (window_table_ready) return true;
    uint16_t w[221];
    int k = 0;
    for (int dx = -8; dx <= 8; ++dx)
        for (int dz = -8; dz <= 8; ++dz)
            if (dx * dx + dz * dz <= 68) w[k++] = (uint16_t)((dx + 8) * 17 + (dz + 8));
    const cudaError_t e = cudaMemcpyToSymbol(c_window, w, sizeof(w));
    if (e != cudaSuccess) {
        ctx().set_error("biome window table", e);
        return false;
    }
    window_table_ready = true;
    return true;
}

int grid_for(int64_t items, int per_block) {
    const int64_t blocks = (items + per_block - 1) / per_block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(blocks, (int64_t)ctx().sm_count * 16));
}

}  // namespace

BiomeContext* context_create(int32_t version, uint64_t world_seed, int32_t large, int32_t capacity) {
    if (capacity <= 0 || tree_index(version) < 0) return nullptr;
    Context& c = ctx();
    if (!c.ensure_device() || !ensure_tables() || !ensure_window_table()) return nullptr;
    BiomeContext* b = new BiomeContext();
    b->version = version;
    b->tree = tree_index(version);
    b->large = large ? 1 : 0;
    b->capacity = capacity;
    b->world_seed = world_seed;
    std::vector<Climate> host(1);
    climate_init(host[0], world_seed, large != 0);
    cudaError_t e;
    if ((e = cudaMalloc(&b->d_climate, sizeof(Climate))) != cudaSuccess ||
        (e = cudaMemcpy(b->d_climate, host.data(), sizeof(Climate), cudaMemcpyHostToDevice)) != cudaSuccess) {
        c.set_error("biome context", e);
        if (b->d_climate) cudaFree(b->d_climate);
        delete b;
        return nullptr;
    }
    return b;
}

void context_destroy(BiomeContext* b) {
    if (!b) return;
    cudaStream_t s = ctx().stream;
    b->x.release(s);
    b->y.release(s);
    b->z.release(s);
    b->out.release(s);
    b->keys.release(s);
    b->vals.release(s);
    b->uniq.release(s);
    b->chunk_bits.release(s);
    b->counters.release(s);
    if (s) cudaStreamSynchronize(s);
    if (b->d_climate) cudaFree(b->d_climate);
    delete b;
}

// Verdict masks of n candidates whose chunk coordinates are already on the device (dcx, dcz);
// writes dmask (device). flags: bit 0 Deep Dark, bit 1 Mushroom Fields. Returns false on a CUDA
// failure (error text set).
bool filter_device(BiomeContext* b, const int32_t* dcx, const int32_t* dcz, int32_t n, int32_t flags,
                   int32_t* dmask) {
    Context& c = ctx();
    cudaStream_t s = c.stream;
    const Tables& t = tables();
    cudaError_t e;
    if (n <= 0) return true;
    unsigned int* pin = static_cast<unsigned int*>(c.pinned);
    const int warps_grid = (int)(((int64_t)n * 32 + kThreads - 1) / kThreads);
    if ((e = b->counters.reserve(8, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(b->counters.p, 0, 8 * sizeof(unsigned int), s)) != cudaSuccess ||
        (e = cudaMemsetAsync(b->counters.p + 4, 0xff, sizeof(unsigned int), s)) != cudaSuccess) {
        c.set_error("biome filter", e);
        return false;
    }
    unsigned long long* total = reinterpret_cast<unsigned long long*>(b->counters.p);
    count_kernel<<<warps_grid, kThreads, 0, s>>>((int64_t)b->world_seed, dcx, dcz, n, total);
    ++c.last_launches;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(pin, b->counters.p, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        c.set_error("biome filter: count", e);
        return false;
    }
    const uint64_t slime = *reinterpret_cast<unsigned long long*>(pin);
    uint64_t cap = 1024;
    while (cap < 2 * slime) cap <<= 1;
    if (cap > (1ull << 31)) {
        c.set_error_text("biome filter: too many candidates in one call");
        return false;
    }
    if ((e = b->keys.reserve(cap, s)) != cudaSuccess || (e = b->vals.reserve(cap, s)) != cudaSuccess ||
        (e = b->uniq.reserve(std::max<uint64_t>(slime, 1), s)) != cudaSuccess ||
        (e = b->chunk_bits.reserve(std::max<uint64_t>(slime, 1), s)) != cudaSuccess ||
        (e = cudaMemsetAsync(b->keys.p, 0xff, cap * 8, s)) != cudaSuccess) {
        c.set_error("biome filter: hash set", e);
        return false;
    }
    HashSet h{b->keys.p, b->vals.p, (uint32_t)(cap - 1), b->uniq.p, b->counters.p + 2,
              reinterpret_cast<int32_t*>(b->counters.p + 4), b->counters.p + 3};
    insert_kernel<<<warps_grid, kThreads, 0, s>>>((int64_t)b->world_seed, dcx, dcz, n, h);
    ++c.last_launches;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(pin, b->counters.p + 2, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        c.set_error("biome filter: insert", e);
        return false;
    }
    const uint32_t nuniq = pin[0];
    if (pin[1]) {
        c.set_error_text("biome filter: hash set overflow");
        return false;
    }
    b->last_unique = nuniq;
    const uint32_t want = (uint32_t)flags & 3u;
    if (nuniq > 0) {
        if ((e = cudaMemsetAsync(b->chunk_bits.p, 0, (size_t)nuniq * 4, s)) != cudaSuccess) {
            c.set_error("biome filter", e);
            return false;
        }
        const int grid = grid_for((int64_t)nuniq * 16, kThreads);
        const TreeGeom& g = t.geom[b->tree];
        if (want == 3)
            chunk_kernel<kDeepLayers + 1><<<grid, kThreads, 0, s>>>(b->d_climate, t.heads, t.pts, t.nodes[b->tree],
                                                                     t.params[b->tree], g, b->uniq.p, (int32_t)nuniq,
                                                                     b->chunk_bits.p, want);
        else if (want == 1)
            chunk_kernel<kDeepLayers><<<grid, kThreads, 0, s>>>(b->d_climate, t.heads, t.pts, t.nodes[b->tree],
                                                                 t.params[b->tree], g, b->uniq.p, (int32_t)nuniq,
                                                                 b->chunk_bits.p, want);
        else
            chunk_kernel<1><<<grid, kThreads, 0, s>>>(b->d_climate, t.heads, t.pts, t.nodes[b->tree],
                                                      t.params[b->tree], g, b->uniq.p, (int32_t)nuniq,
                                                      b->chunk_bits.p, want);
        ++c.last_launches;
        if ((e = cudaGetLastError()) != cudaSuccess) {
            c.set_error("biome filter: chunks", e);
            return false;
        }
    }
    verdict_kernel<<<warps_grid, kThreads, 0, s>>>((int64_t)b->world_seed, dcx, dcz, n, h, b->chunk_bits.p, want,
                                                   dmask);
    ++c.last_launches;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(pin, b->counters.p + 3, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        c.set_error("biome filter: verdicts", e);
        return false;
    }
    if (pin[0]) {
        c.set_error_text("biome filter: chunk missing from the hash set");
        return false;
    }
    return true;
}

// Host arrays in and out; at most `capacity` candidates per device batch.
bool filter_host(BiomeContext* b, const int32_t* cx, const int32_t* cz, int64_t n, int32_t flags, int32_t* mask) {
    Context& c = ctx();
    cudaStream_t s = c.stream;
    const int64_t batch = std::max<int64_t>(1, std::min<int64_t>(b->capacity, 1 << 18));
    cudaError_t e;
    if ((e = b->x.reserve(batch, s)) != cudaSuccess || (e = b->z.reserve(batch, s)) != cudaSuccess ||
        (e = b->out.reserve(batch, s)) != cudaSuccess) {
        c.set_error("biome filter", e);
        return false;
    }
    cudaEvent_t e0 = c.ev_a, e1 = c.ev_b;
    b->last_ms = 0.0;
    for (int64_t off = 0; off < n; off += batch) {
        const int32_t m = (int32_t)std::min<int64_t>(batch, n - off);
        if ((e = cudaMemcpyAsync(b->x.p, cx + off, (size_t)m * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(b->z.p, cz + off, (size_t)m * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaEventRecord(e0, s)) != cudaSuccess) {
            c.set_error("biome filter: copy", e);
            return false;
        }
        if (!filter_device(b, b->x.p, b->z.p, m, flags, b->out.p)) return false;
        float ms = 0.f;
        if ((e = cudaEventRecord(e1, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(mask + off, b->out.p, (size_t)m * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess) {
            c.set_error("biome filter: copy", e);
            return false;
        }
        cudaEventElapsedTime(&ms, e0, e1);
        b->last_ms += ms;
    }
    return true;
}

bool query_host(BiomeContext* b, const int32_t* xs, const int32_t* ys, const int32_t* zs, int32_t n, int32_t* out) {
    Context& c = ctx();
    cudaStream_t s = c.stream;
    const Tables& t = tables();
    cudaError_t e;
    if ((e = b->x.reserve(n, s)) != cudaSuccess || (e = b->y.reserve(n, s)) != cudaSuccess ||
        (e = b->z.reserve(n, s)) != cudaSuccess || (e = b->out.reserve(n, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b->x.p, xs, (size_t)n * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b->y.p, ys, (size_t)n * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b->z.p, zs, (size_t)n * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
        c.set_error("biome query", e);
        return false;
    }
    query_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(b->d_climate, t.heads, t.pts, t.nodes[b->tree],
                                                              t.params[b->tree], t.geom[b->tree], b->x.p, b->y.p,
                                                              b->z.p, n, b->out.p);
    ++c.last_launches;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(out, b->out.p, (size_t)n * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        c.set_error("biome query", e);
        return false;
    }
    return true;
}

// Climate sampling of host points (see climate_kernel for the modes); element sizes: 4 bytes for
// int inputs (modes 0, 1), 8 for double inputs; out_per_point values of out_size bytes.
int climate_host(uint64_t world_seed, int32_t large, int mode, const void* xs, const void* ys, const void* zs,
                 int32_t n, void* out) {
    Context& c = ctx();
    if (!c.ensure_device() || !ensure_tables()) return -2;
    cudaStream_t s = c.stream;
    const size_t in_sz = mode <= 1 ? 4 : 8;
    const size_t out_sz = mode == 0 ? 24 : mode == 1 || mode == 2 ? 20 : mode == 3 ? 40 : 8;
    std::vector<Climate> host(1);
    climate_init(host[0], world_seed, large != 0);
    void *dcl = nullptr, *dx = nullptr, *dy = nullptr, *dz = nullptr, *dout = nullptr;
    cudaError_t e;
    int rc = 0;
    if ((e = cudaMallocAsync(&dcl, sizeof(Climate), s)) != cudaSuccess ||
        (e = cudaMallocAsync(&dx, n * in_sz, s)) != cudaSuccess ||
        (e = cudaMallocAsync(&dz, n * in_sz, s)) != cudaSuccess ||
        (mode == 0 && (e = cudaMallocAsync(&dy, n * 4, s)) != cudaSuccess) ||
        (e = cudaMallocAsync(&dout, n * out_sz, s)) != cudaSuccess) {
        rc = -3;
    } else if ((e = cudaMemcpyAsync(dcl, host.data(), sizeof(Climate), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
               (e = cudaMemcpyAsync(dx, xs, n * in_sz, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
               (e = cudaMemcpyAsync(dz, zs, n * in_sz, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
               (mode == 0 && (e = cudaMemcpyAsync(dy, ys, n * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess)) {
        rc = -2;
    } else {
        const Tables& t = tables();
        climate_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(static_cast<Climate*>(dcl), t.heads, t.pts, mode,
                                                                    dx, dy, dz, n, dout);
        ++c.last_launches;
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpyAsync(out, dout, n * out_sz, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            rc = -2;
    }
    if (rc) c.set_error("biome climate", e);
    for (void* p : {dcl, dx, dy, dz, dout})
        if (p) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
    return rc;
}

int xoroshiro_host(const uint64_t* seeds, int32_t n, int32_t steps, uint64_t* out) {
    Context& c = ctx();
    if (!c.ensure_device()) return -2;
    cudaStream_t s = c.stream;
    uint64_t *ds = nullptr, *dout = nullptr;
    cudaError_t e;
    int rc = 0;
    if ((e = cudaMallocAsync(&ds, (size_t)n * 8, s)) != cudaSuccess ||
        (e = cudaMallocAsync(&dout, (size_t)n * steps * 8, s)) != cudaSuccess) {
        rc = -3;
    } else if ((e = cudaMemcpyAsync(ds, seeds, (size_t)n * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
        rc = -2;
    } else {
        xoroshiro_kernel<<<(n + 255) / 256, 256, 0, s>>>(ds, n, steps, dout);
        ++c.last_launches;
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpyAsync(out, dout, (size_t)n * steps * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            rc = -2;
    }
    if (rc) c.set_error("xoroshiro", e);
    if (ds) cudaFreeAsync(ds, s);
    if (dout) cudaFreeAsync(dout, s);
    cudaStreamSynchronize(s);
    return rc;
}

int perlin_host(const uint64_t* seeds, uint64_t fixed_seed, bool fixed, const double* xs, const double* ys,
                const double* zs, int32_t n, double* out) {
    Context& c = ctx();
    if (!c.ensure_device()) return -2;
    cudaStream_t s = c.stream;
    void *ds = nullptr, *dfix = nullptr, *dx = nullptr, *dy = nullptr, *dz = nullptr, *dout = nullptr;
    cudaError_t e;
    int rc = 0;
    Octave oct;
    if (fixed) perlin_init(oct, xr_seed(fixed_seed));
    if ((!fixed && (e = cudaMallocAsync(&ds, (size_t)n * 8, s)) != cudaSuccess) ||
        (fixed && (e = cudaMallocAsync(&dfix, sizeof(Octave), s)) != cudaSuccess) ||
        (e = cudaMallocAsync(&dx, (size_t)n * 8, s)) != cudaSuccess ||
        (e = cudaMallocAsync(&dy, (size_t)n * 8, s)) != cudaSuccess ||
        (e = cudaMallocAsync(&dz, (size_t)n * 8, s)) != cudaSuccess ||
        (e = cudaMallocAsync(&dout, (size_t)n * 8, s)) != cudaSuccess) {
        rc = -3;
    } else if ((!fixed && (e = cudaMemcpyAsync(ds, seeds, (size_t)n * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess) ||
               (fixed && (e = cudaMemcpyAsync(dfix, &oct, sizeof(Octave), cudaMemcpyHostToDevice, s)) != cudaSuccess) ||
               (e = cudaMemcpyAsync(dx, xs, (size_t)n * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
               (e = cudaMemcpyAsync(dy, ys, (size_t)n * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
               (e = cudaMemcpyAsync(dz, zs, (size_t)n * 8, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
        rc = -2;
    } else {
        perlin_kernel<<<(n + 127) / 128, 128, 0, s>>>(static_cast<uint64_t*>(ds), static_cast<Octave*>(dfix),
                                                      static_cast<double*>(dx), static_cast<double*>(dy),
                                                      static_cast<double*>(dz), n, static_cast<double*>(dout));
        ++c.last_launches;
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpyAsync(out, dout, (size_t)n * 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            rc = -2;
    }
    if (rc) c.set_error("perlin", e);
    for (void* p : {ds, dfix, dx, dy, dz, dout})
        if (p) cudaFreeAsync(p, s);
    cudaStreamSynchronize(s);
    return rc;
}

}  // namespace biome

namespace {
biome::BiomeContext* g_search_ctx = nullptr;  // biome context of the last filtered search
}

bool biome_masks(int64_t world_seed, int32_t version, int32_t large, int32_t flags, const int32_t* cx,
                 const int32_t* cz, int64_t n, int32_t* mask) {
    if (n <= 0) return true;
    biome::BiomeContext*& b = g_search_ctx;
    if (!b || b->world_seed != (uint64_t)world_seed || b->version != version || b->large != (large ? 1 : 0)) {
        biome::context_destroy(b);
        b = biome::context_create(version, (uint64_t)world_seed, large, 1 << 18);
        if (!b) {
            if (biome::tree_index(version) < 0) ctx().set_error_text("biome filter: unsupported version code");
            return false;
        }
    }
    return biome::filter_host(b, cx, cz, n, flags, mask);
}

void release_biome() {
    biome::context_destroy(g_search_ctx);
    g_search_ctx = nullptr;
}

}  // namespace slime

// ---- C ABI: the reference's biome module (MinecraftGPUNoise.cu:1076-2018) --------------------------

using slime::ctx;
namespace bm = slime::biome;

namespace {
enum { MC_OK = 0, MC_ERR_ARG = -1, MC_ERR_CUDA = -2, MC_ERR_ALLOC = -3 };

// A ctx of the climate-only and biome20 entry points is a BiomeContext of a fixed version.
constexpr int32_t kBiome20Version = 1206;

int query_impl(void* handle, const int32_t* xs, const int32_t* ys, const int32_t* zs, int32_t count,
               int32_t* out) {
    auto* b = static_cast<bm::BiomeContext*>(handle);
    if (!b || !xs || !ys || !zs || !out || count <= 0 || count > b->capacity) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::query_host(b, xs, ys, zs, count, out) ? MC_OK : MC_ERR_CUDA;
}
}  // namespace

extern "C" {

int mcgpu_api_version(void) { return 1; }

const char* mcgpu_build_name(void) { return "slime_b200 biome filter (sm_100a, FP64, xoroshiro128++)"; }

// One wave of filter work (MinecraftGPUNoise.cu:1081-1100): here the batch that fills every SM with
// chunk_kernel blocks at ~22 slime chunks x 16 quarts per candidate, rounded to 32, in [32, 1024].
int32_t mcgpu_modern_recommended_filter_batch(void) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 128;
    }
    int32_t wave = sms * 4;
    wave = ((wave + 31) / 32) * 32;
    return std::min<int32_t>(1024, std::max<int32_t>(32, wave));
}

int mcgpu_xoroshiro_nextlong_batch(const uint64_t* seeds, int32_t count, int32_t steps, uint64_t* out) {
    if (!seeds || !out || count <= 0 || steps <= 0 || (int64_t)count * steps > (int64_t)1 << 40) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::xoroshiro_host(seeds, count, steps, out);
}

int mcgpu_xperlin_sample_batch(const uint64_t* seeds, const double* xs, const double* ys, const double* zs,
                               int32_t count, double* out) {
    if (!seeds || !xs || !ys || !zs || !out || count <= 0) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::perlin_host(seeds, 0, false, xs, ys, zs, count, out);
}

int mcgpu_xperlin_sample_fixed_seed(uint64_t seed, const double* xs, const double* ys, const double* zs,
                                    int32_t count, double* out) {
    if (!xs || !ys || !zs || !out || count <= 0) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::perlin_host(nullptr, seed, true, xs, ys, zs, count, out);
}

int mcgpu_continentalness_noise_fixed_seed(uint64_t world_seed, const double* xs, const double* zs, int32_t count,
                                           double* out) {
    if (!xs || !zs || !out || count <= 0) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::climate_host(world_seed, 0, 4, xs, nullptr, zs, count, out);
}

int mcgpu_climate5_fixed_seed(uint64_t world_seed, const double* xs, const double* zs, int32_t count, double* out5) {
    if (!xs || !zs || !out5 || count <= 0) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::climate_host(world_seed, 0, 3, xs, nullptr, zs, count, out5);
}

int mcgpu_climate5_quant_fixed_seed(uint64_t world_seed, const double* xs, const double* zs, int32_t count,
                                    int32_t* out5) {
    if (!xs || !zs || !out5 || count <= 0) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::climate_host(world_seed, 0, 2, xs, nullptr, zs, count, out5);
}

int mcgpu_climate5_i32_fixed_seed(uint64_t world_seed, const int32_t* xs, const int32_t* zs, int32_t count,
                                  int32_t* out5) {
    if (!xs || !zs || !out5 || count <= 0) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::climate_host(world_seed, 0, 1, xs, nullptr, zs, count, out5);
}

int mcgpu_climate6_i32_fixed_seed(uint64_t world_seed, const int32_t* xs, const int32_t* ys, const int32_t* zs,
                                  int32_t count, int32_t* out6) {
    if (!xs || !ys || !zs || !out6 || count <= 0) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::climate_host(world_seed, 0, 0, xs, ys, zs, count, out6);
}

int mcgpu_climate6_i32_fixed_seed_ex(uint64_t world_seed, int32_t large, const int32_t* xs, const int32_t* ys,
                                     const int32_t* zs, int32_t count, int32_t* out6) {
    if (!xs || !ys || !zs || !out6 || count <= 0) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::climate_host(world_seed, large != 0, 0, xs, ys, zs, count, out6);
}

// Climate context (MinecraftGPUNoise.cu:1461-1542): climate5_i32 of a fixed world seed.
void* mcgpu_climate_ctx_create(uint64_t world_seed, int32_t capacity) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::context_create(kBiome20Version, world_seed, 0, capacity);
}

int mcgpu_climate_ctx_query_i32(void* handle, const int32_t* xs, const int32_t* zs, int32_t count, int32_t* out5) {
    auto* b = static_cast<bm::BiomeContext*>(handle);
    if (!b || !xs || !zs || !out5 || count <= 0 || count > b->capacity) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::climate_host(b->world_seed, b->large, 1, xs, nullptr, zs, count, out5);
}

void mcgpu_climate_ctx_destroy(void* handle) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    bm::context_destroy(static_cast<bm::BiomeContext*>(handle));
}

// Biome ids with the 1.20.6 tree (MinecraftGPUNoise.cu:1597-1775).
int mcgpu_biome20_i32_fixed_seed(uint64_t world_seed, const int32_t* xs, const int32_t* ys, const int32_t* zs,
                                 int32_t count, int32_t* biome_out) {
    if (!xs || !ys || !zs || !biome_out || count <= 0) return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    bm::BiomeContext* b = bm::context_create(kBiome20Version, world_seed, 0, count);
    if (!b) return MC_ERR_ALLOC;
    const bool ok = bm::query_host(b, xs, ys, zs, count, biome_out);
    bm::context_destroy(b);
    return ok ? MC_OK : MC_ERR_CUDA;
}

void* mcgpu_biome20_ctx_create(uint64_t world_seed, int32_t capacity) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::context_create(kBiome20Version, world_seed, 0, capacity);
}

int mcgpu_biome20_ctx_query(void* handle, const int32_t* xs, const int32_t* ys, const int32_t* zs, int32_t count,
                            int32_t* biome_out) {
    return query_impl(handle, xs, ys, zs, count, biome_out);
}

void mcgpu_biome20_ctx_destroy(void* handle) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    bm::context_destroy(static_cast<bm::BiomeContext*>(handle));
}

// Modern biome context (MinecraftGPUNoise.cu:1837-1990): NULL for a version whose tree is not
// vendored (below 1180, as in the reference), a non-positive capacity or no usable device.
void* mcgpu_modern_ctx_create(int32_t version_code, uint64_t world_seed, int32_t capacity) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::context_create(version_code, world_seed, 0, capacity);
}

void* mcgpu_modern_ctx_create_ex(int32_t version_code, uint64_t world_seed, int32_t flags, int32_t capacity) {
    if ((flags & ~1) != 0) return nullptr;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::context_create(version_code, world_seed, flags & 1, capacity);
}

int mcgpu_modern_ctx_query(void* handle, const int32_t* xs, const int32_t* ys, const int32_t* zs, int32_t count,
                           int32_t* biome_out) {
    return query_impl(handle, xs, ys, zs, count, biome_out);
}

int mcgpu_modern_ctx_filter_candidates(void* handle, const int32_t* center_chunk_x, const int32_t* center_chunk_z,
                                       int32_t count, int32_t flags, int32_t* mask_out) {
    auto* b = static_cast<bm::BiomeContext*>(handle);
    if (!b || !center_chunk_x || !center_chunk_z || !mask_out || count <= 0 || count > b->capacity ||
        (flags & ~3) != 0 || flags == 0)
        return MC_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx().mu);
    return bm::filter_host(b, center_chunk_x, center_chunk_z, count, flags, mask_out) ? MC_OK : MC_ERR_CUDA;
}

void mcgpu_modern_ctx_destroy(void* handle) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    bm::context_destroy(static_cast<bm::BiomeContext*>(handle));
}

// Timing of the last filter call on a context: device time of its kernels (CUDA events on the
// library's stream) and the number of unique slime chunks it evaluated. No reference counterpart.
void slime_b200_biome_last_stats(void* handle, double* kernel_ms, int64_t* unique_chunks) {
    auto* b = static_cast<bm::BiomeContext*>(handle);
    if (!b) return;
    if (kernel_ms) *kernel_ms = b->last_ms;
    if (unique_chunks) *unique_chunks = b->last_unique;
}

}  // extern "C"
