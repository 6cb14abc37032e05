// biome_math.cuh -- FP64 climate noise, depth spline and biome-tree search of the biome filter.
//
// Bit-exact restatement of the reference's biome module (gpu_noise/MinecraftGPUNoise.cu) with its
// floating-point operations in source order and no contraction: the file that includes this
// header is compiled with --fmad=false, so every double/float operation is one IEEE operation, as
// in the reference's source text (and as Minecraft's Java code computes them).
//
//   Xoroshiro128++ seeding and draws ........ MinecraftGPUNoise.cu:15-73
//   improved Perlin noise .................... :75-190
//   octave sets and double-Perlin climate .... :196-422
//   depth spline ............................. spline_generated.cuh (control points in biome_data.h)
//   parameter-tree nearest leaf .............. :650-809
//   quart climate and biome .................. :868-913
#pragma once

#include <cstdint>

#include "biome_data.h"

namespace slime {
namespace biome {

// ---- Xoroshiro128++ -------------------------------------------------------------------------

struct Xr {
    uint64_t lo, hi;
};

__host__ __device__ inline uint64_t rotl64(uint64_t x, unsigned b) { return (x << b) | (x >> (64u - b)); }

__host__ __device__ inline uint64_t mix13(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// 64-bit seed to the 128-bit state (Java RandomSupport.upgradeSeedTo128bit).
__host__ __device__ inline Xr xr_seed(uint64_t seed) {
    const uint64_t lo = seed ^ 0x6a09e667f3bcc909ull;
    return Xr{mix13(lo), mix13(lo + 0x9e3779b97f4a7c15ull)};
}

__host__ __device__ inline uint64_t xr_next(Xr& s) {
    const uint64_t l = s.lo;
    uint64_t h = s.hi;
    const uint64_t out = rotl64(l + h, 17) + l;
    h ^= l;
    s.lo = rotl64(l, 49) ^ h ^ (h << 21);
    s.hi = rotl64(h, 28);
    return out;
}

// Java nextInt(bound): multiply-high of the low word, rejecting the biased low products.
__host__ __device__ inline uint32_t xr_next_int(Xr& s, uint32_t n) {
    uint64_t r = (xr_next(s) & 0xffffffffull) * (uint64_t)n;
    if ((uint32_t)r < n) {
        const uint32_t bound = (0u - n) % n;
        while ((uint32_t)r < bound) r = (xr_next(s) & 0xffffffffull) * (uint64_t)n;
    }
    return (uint32_t)(r >> 32);
}

__host__ __device__ inline double xr_next_double(Xr& s) { return (double)(xr_next(s) >> 11) * 0x1.0p-53; }

// ---- improved Perlin noise --------------------------------------------------------------------

// One octave of a noise: offsets, permutation, the y cell/fraction/fade for samples at y = 0,
// amplitude and lacunarity. 320 bytes; the 46 octaves of the six climate noises stay in shared
// memory during sampling.
struct Octave {
    double ox, oy, oz;
    double y_frac, y_fade;
    double amp, lac;
    uint8_t perm[257];
    uint8_t y_cell;
    uint8_t pad[6];
};

struct Noise {
    int32_t first, na, nb, pad;
    double amp;
};

// The six climate noises of a world seed (shift, temperature, humidity, continentalness,
// erosion, weirdness): 14.8 KB.
struct Climate {
    Noise noise[6];
    Octave oct[46];
};

enum { kShift = 0, kTemp = 1, kHumid = 2, kCont = 3, kEros = 4, kWeird = 5 };

__host__ __device__ inline double fade(double t) { return t * t * t * (t * (t * 6.0 - 15.0) + 10.0); }
__host__ __device__ inline double lerp(double t, double a, double b) { return a + t * (b - a); }

// Gradient dot product of improved noise for hash h: x, y or z (a), with a sign, plus another
// (b) with a sign: the 12 cube edges, 4 of them repeated.
__host__ __device__ inline double grad(uint32_t h, double x, double y, double z) {
    switch (h & 15u) {
    case 0: case 12: return x + y;
    case 1: case 14: return -x + y;
    case 2: return x - y;
    case 3: return -x - y;
    case 4: return x + z;
    case 5: return -x + z;
    case 6: return x - z;
    case 7: return -x - z;
    case 8: return y + z;
    case 9: case 13: return -y + z;
    case 10: return y - z;
    default: return -y - z;  // 11, 15
    }
}

// Octave set initialisation on the host (the permutation shuffle is serial): two seeds from the
// parent, then per non-zero amplitude an octave seeded with the hash of "octave_<k>".
void octave_set_init(Octave* out, Xr& parent, const double* amp, int first, int n, int* count);

__device__ __forceinline__ double perlin_sample(const Octave& p, double x, double y, double z) {
    uint32_t hy;
    double ty;
    if (y == 0.0) {
        y = p.y_frac;
        hy = p.y_cell;
        ty = p.y_fade;
    } else {
        y += p.oy;
        const double cy = floor(y);
        y -= cy;
        hy = (uint8_t)(int)cy;
        ty = fade(y);
    }
    x += p.ox;
    z += p.oz;
    const double cx = floor(x), cz = floor(z);
    x -= cx;
    z -= cz;
    const uint32_t hx = (uint8_t)(int)cx, hz = (uint8_t)(int)cz;
    const double tx = fade(x), tz = fade(z);
    const uint8_t* d = p.perm;
    const uint32_t a1 = (uint8_t)(d[hx] + hy), b1 = (uint8_t)(d[hx + 1] + hy);
    const uint32_t a2 = (uint8_t)(d[a1] + hz), b2 = (uint8_t)(d[b1] + hz);
    const uint32_t a3 = (uint8_t)(d[a1 + 1] + hz), b3 = (uint8_t)(d[b1 + 1] + hz);
    const double x1 = x - 1.0, y1 = y - 1.0, z1 = z - 1.0;
    double l1 = grad(d[a2], x, y, z), l2 = grad(d[b2], x1, y, z);
    double l3 = grad(d[a3], x, y1, z), l4 = grad(d[b3], x1, y1, z);
    double l5 = grad(d[a2 + 1], x, y, z1), l6 = grad(d[b2 + 1], x1, y, z1);
    double l7 = grad(d[a3 + 1], x, y1, z1), l8 = grad(d[b3 + 1], x1, y1, z1);
    l1 = lerp(tx, l1, l2);
    l3 = lerp(tx, l3, l4);
    l5 = lerp(tx, l5, l6);
    l7 = lerp(tx, l7, l8);
    l1 = lerp(ty, l1, l3);
    l5 = lerp(ty, l5, l7);
    return lerp(tz, l1, l5);
}

__device__ __forceinline__ double octaves_sample(const Octave* o, int n, double x, double y, double z) {
    double v = 0.0;
    for (int i = 0; i < n; ++i) {
        const double f = o[i].lac;
        const double s = perlin_sample(o[i], x * f, y * f, z * f);
        v += o[i].amp * s;
    }
    return v;
}

__device__ __forceinline__ double noise_sample(const Climate& c, int s, double x, double y, double z) {
    const Noise& n = c.noise[s];
    const double f = 337.0 / 331.0;
    double v = octaves_sample(c.oct + n.first, n.na, x, y, z);
    v += octaves_sample(c.oct + n.first + n.na, n.nb, x * f, y * f, z * f);
    return v * n.amp;
}

// ---- depth spline ---------------------------------------------------------------------------

struct SplinePt {
    float loc, der, val;
    int32_t child;  // -1: constant value
};

struct SplineHead {
    int32_t coord, first, count, pad;
};

// Cubic Hermite segments between control points, linear outside (cubiomes getSpline); values of
// points may be child splines, evaluated to depth LEVEL.
template <int LEVEL>
__device__ __forceinline__ float spline_eval(const SplineHead* heads, const SplinePt* pts, int s, const float* v);

template <int LEVEL>
__device__ __forceinline__ float spline_value(const SplineHead* heads, const SplinePt* pts, const SplinePt& p,
                                              const float* v) {
    if constexpr (LEVEL <= 0) {
        return p.val;
    } else {
        return p.child < 0 ? p.val : spline_eval<LEVEL - 1>(heads, pts, p.child, v);
    }
}

template <int LEVEL>
__device__ __forceinline__ float spline_eval(const SplineHead* heads, const SplinePt* pts, int s, const float* v) {
    const SplineHead hd = heads[s];
    const SplinePt* p = pts + hd.first;
    const float f = v[hd.coord];
    if (f <= p[0].loc) return spline_value<LEVEL>(heads, pts, p[0], v) + p[0].der * (f - p[0].loc);
    for (int i = 1; i < hd.count; ++i) {
        const float h = p[i].loc;
        if (f > h) continue;
        const float g = p[i - 1].loc;
        const float k = (f - g) / (h - g);
        const float l = p[i - 1].der, m = p[i].der;
        const float v0 = spline_value<LEVEL>(heads, pts, p[i - 1], v);
        const float v1 = spline_value<LEVEL>(heads, pts, p[i], v);
        const float pp = l * (h - g) - (v1 - v0);
        const float q = -m * (h - g) + (v1 - v0);
        const double a = lerp((double)k, (double)v0, (double)v1);
        const float kk = k * (1.0f - k);
        const double b = lerp((double)k, (double)pp, (double)q);
        return (float)(a + (double)kk * b);
    }
    const SplinePt& last = p[hd.count - 1];
    return spline_value<LEVEL>(heads, pts, last, v) + last.der * (f - last.loc);
}

__device__ __forceinline__ float peaks_valleys(float w) {
    return -(fabsf(fabsf(w) - 0.6666667f) - 0.33333334f) * 3.0f;
}

// Climate of quart column (x, z): the quantised {T, H, C, E, W} (x 1e4, truncated) and the float
// depth offset of the spline; the depth parameter of quart Y y is depth_at(offset, y).
struct Column {
    int32_t t, h, c, e, w;
    float off;
};

template <int SPLINE_LEVELS>
__device__ __forceinline__ Column column_climate(const Climate& cl, const SplineHead* heads, const SplinePt* pts,
                                                 int32_t xi, int32_t zi) {
    const double x = (double)xi, z = (double)zi;
    const double px = x + noise_sample(cl, kShift, x, 0.0, z) * 4.0;
    const double pz = z + noise_sample(cl, kShift, z, x, 0.0) * 4.0;
    const float c = (float)noise_sample(cl, kCont, px, 0.0, pz);
    const float e = (float)noise_sample(cl, kEros, px, 0.0, pz);
    const float w = (float)noise_sample(cl, kWeird, px, 0.0, pz);
    const float in[4] = {c, e, peaks_valleys(w), w};
    Column col;
    col.off = spline_eval<SPLINE_LEVELS>(heads, pts, 0, in) + 0.015f;
    const float t = (float)noise_sample(cl, kTemp, px, 0.0, pz);
    const float h = (float)noise_sample(cl, kHumid, px, 0.0, pz);
    col.t = (int32_t)(10000.0f * t);
    col.h = (int32_t)(10000.0f * h);
    col.c = (int32_t)(10000.0f * c);
    col.e = (int32_t)(10000.0f * e);
    col.w = (int32_t)(10000.0f * w);
    return col;
}

__device__ __forceinline__ int32_t depth_at(float off, int32_t y) {
    const double d0 = 1.0 - ((double)(y * 4)) / 128.0 - 83.0 / 160.0 + (double)off;
    const float d = (float)d0;
    return (int32_t)(10000.0f * d);
}

// ---- biome parameter tree -------------------------------------------------------------------

// Tree geometry (device copy of a BdTree's scalars); nodes and parameter ranges live in device
// memory / shared memory.
struct TreeGeom {
    int32_t order, depth, nnodes, nparams;
    int32_t steps[8];
};

__device__ __forceinline__ int64_t axis_d2(int32_t v, int2 r) {
    const int64_t d = v > r.y ? (int64_t)v - r.y : v < r.x ? (int64_t)r.x - v : 0;
    return d * d;
}

// Distance of v to the range r along one axis. kWide: exact for every int32 v (64-bit
// differences); otherwise 32-bit differences, exact while |v| <= 2^30 (range bounds are within
// +-12,000, so no difference overflows).
template <bool kWide>
__device__ __forceinline__ uint32_t axis_gap(int32_t v, int2 r) {
    if constexpr (kWide) {
        return (uint32_t)(v > r.y ? (int64_t)v - r.y : v < r.x ? (int64_t)r.x - v : 0);
    } else {
        return (uint32_t)max(max(r.x - v, v - r.y), 0);
    }
}

// The squared distance sum of one node's box plus g^2 (squares of 32-bit gaps, summed in 64 bits,
// as the reference's int64 / uint64 arithmetic gives for these magnitudes).
__device__ __forceinline__ uint64_t add_sq(uint64_t acc, uint32_t g) { return acc + (uint64_t)g * g; }

// Nearest leaves of NQ queries that differ only in the depth axis (axis 4), in one traversal.
// Each query follows exactly the reference's branch and bound (MinecraftGPUNoise.cu:686-809):
// children of a node at tree depth d are `order` nodes steps[d] apart (a node whose subtree would
// run past the end descends in place), a child is entered when its box is strictly closer than
// the query's best leaf, and a leaf replaces the best only when strictly closer. Per stack level
// a bit mask keeps the queries that entered the subtree; the other queries neither descend nor
// update there, so every query visits and decides exactly as a search of its own would.
// Returns the biome ids (link byte of the best leaf) in biome[].
template <int NQ, bool kWide>
__device__ __forceinline__ void tree_nearest_impl(const uint64_t* __restrict__ nodes, const int2* __restrict__ param,
                                                  const TreeGeom& g, const int32_t base[5],
                                                  const int32_t (&depth)[NQ], int32_t (&biome)[NQ]) {
    constexpr int kMaxDepth = 8;
    static_assert(NQ <= 32, "query mask is 32 bits");
    uint64_t ds[NQ];
    int32_t best[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        ds[q] = ~0ull;
        best[q] = 0;
    }
    // Stack level: next child (bits 0-15), children left (16-23), tree depth (24-31); query mask.
    uint32_t st_node[kMaxDepth], st_mask[kMaxDepth];
    int sp = 0;
    // Root: node 0 at depth 0, every query active.
    {
        int d = 0;
        while (d < g.depth && 0 + g.steps[d] >= g.nnodes) ++d;
        st_node[0] = (uint32_t)((nodes[0] >> 48) & 0xffff) | ((uint32_t)g.order << 16) | ((uint32_t)d << 24);
        st_mask[0] = NQ == 32 ? 0xffffffffu : ((1u << NQ) - 1u);
    }
    while (sp >= 0) {
        const uint32_t top = st_node[sp];
        const int32_t child = (int32_t)(top & 0xffff);
        const int left = (int)((top >> 16) & 0xff), d = (int)(top >> 24);
        if (left <= 0 || child >= g.nnodes) {
            --sp;
            continue;
        }
        st_node[sp] = (uint32_t)(child + g.steps[d]) | ((uint32_t)(left - 1) << 16) | ((uint32_t)d << 24);
        const uint32_t active = st_mask[sp];
        const uint64_t node = nodes[child];
        // The five depth-independent axes once, then the depth axis per query.
        uint64_t b5 = add_sq(0, axis_gap<kWide>(base[0], param[node & 0xff]));
        b5 = add_sq(b5, axis_gap<kWide>(base[1], param[(node >> 8) & 0xff]));
        b5 = add_sq(b5, axis_gap<kWide>(base[2], param[(node >> 16) & 0xff]));
        b5 = add_sq(b5, axis_gap<kWide>(base[3], param[(node >> 24) & 0xff]));
        b5 = add_sq(b5, axis_gap<kWide>(base[4], param[(node >> 40) & 0xff]));
        const int2 rd = param[(node >> 32) & 0xff];
        uint32_t enter = 0;
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            if (((active >> q) & 1u) && add_sq(b5, axis_gap<kWide>(depth[q], rd)) < ds[q]) enter |= 1u << q;
        if (!enter) continue;
        // The child sits at depth d + 1; a subtree that would run past the end descends in place.
        int cd = d + 1;
        while (cd < g.depth && child + g.steps[cd] >= g.nnodes) ++cd;
        if (cd >= g.depth) {
            // A leaf: each entering query takes it (its distance is below the query's best).
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                if ((enter >> q) & 1u) {
                    ds[q] = add_sq(b5, axis_gap<kWide>(depth[q], rd));
                    best[q] = child;
                }
            continue;
        }
        ++sp;
        st_node[sp] = (uint32_t)((node >> 48) & 0xffff) | ((uint32_t)g.order << 16) | ((uint32_t)cd << 24);
        st_mask[sp] = enter;
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) biome[q] = (int32_t)((nodes[best[q]] >> 48) & 0xff);
}

// The 32-bit-gap traversal when every coordinate is within +-2^30 (always, for climate values and
// the depths of quart Y within the world), else the 64-bit one; both give the same leaves.
template <int NQ>
__device__ __forceinline__ void tree_nearest(const uint64_t* __restrict__ nodes, const int2* __restrict__ param,
                                             const TreeGeom& g, const int32_t base[5], const int32_t (&depth)[NQ],
                                             int32_t (&biome)[NQ]) {
    constexpr int32_t kLim = 1 << 30;
    bool wide = false;
#pragma unroll
    for (int i = 0; i < 5; ++i) wide |= base[i] > kLim || base[i] < -kLim;
#pragma unroll
    for (int q = 0; q < NQ; ++q) wide |= depth[q] > kLim || depth[q] < -kLim;
    if (wide)
        tree_nearest_impl<NQ, true>(nodes, param, g, base, depth, biome);
    else
        tree_nearest_impl<NQ, false>(nodes, param, g, base, depth, biome);
}

}  // namespace biome
}  // namespace slime
