// ref_biome_host.cpp -- host build of the reference biome module's device math.
//
// TEST INFRASTRUCTURE ONLY (a checker, never the product). The reference's own code is compiled
// here for the CPU: ref_noise_host.inc is MinecraftGPUNoise.cu up to its first extern "C"
// function, with the __global__ kernels removed (oracle/ref_biome_extract.py), and this file
// defines the CUDA qualifiers away so that g++ compiles it with IEEE float/double arithmetic and
// no contraction (-ffp-contract=off, SSE2). The entry points below are thin loops over the
// reference's device functions; the bodies of the removed kernels they stand in for are restated
// from MinecraftGPUNoise.cu (cited per function).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <cmath>

#define __device__
#define __host__
#define __forceinline__ inline
#define __constant__
#define __restrict__

#include "ref_noise_host.inc"

namespace {

struct TreeView {
    const uint64_t* nodes;
    const int32_t* param;
    int32_t len;
    int32_t family;
};

// mcgpu_select_modern_tree (MinecraftGPUNoise.cu:1785-1820).
bool select_tree(int32_t v, TreeView* t) {
#define SEL(N, F)                                                             \
    do {                                                                      \
        t->nodes = N##_nodes;                                                 \
        t->param = &N##_param[0][0];                                          \
        t->len = (int32_t)(sizeof(N##_nodes) / sizeof(N##_nodes[0]));        \
        t->family = F;                                                        \
    } while (0)
    if (v < 1180) return false;
    if (v >= 2602) SEL(btree262, 1);
    else if (v >= 1215) SEL(btree215, 1);
    else if (v >= 1214) SEL(btree21wd, 1);
    else if (v >= 1206) SEL(btree20, 1);
    else if (v >= 1194) SEL(btree19, 1);
    else if (v >= 1192) SEL(btree192, 0);
    else SEL(btree18, 0);
#undef SEL
    return true;
}

}  // namespace

extern "C" {

// xoroshiro_batch_kernel (MinecraftGPUNoise.cu:424-442).
void refb_xoroshiro_nextlong(const uint64_t* seeds, int32_t n, int32_t steps, uint64_t* out) {
    for (int32_t i = 0; i < n; ++i) {
        Xoroshiro128PP s = xoroshiro_from_seed(seeds[i]);
        for (int32_t j = 0; j < steps; ++j) out[(size_t)i * steps + j] = xoroshiro_next_long(s);
    }
}

// xperlin_sample_batch_kernel (MinecraftGPUNoise.cu:444-459).
void refb_xperlin_sample(const uint64_t* seeds, const double* xs, const double* ys, const double* zs,
                         int32_t n, double* out) {
    for (int32_t i = 0; i < n; ++i) {
        PerlinState p;
        xperlin_init(p, seeds[i]);
        out[i] = xperlin_sample(p, xs[i], ys[i], zs[i]);
    }
}

// climate6_i32_kernel (MinecraftGPUNoise.cu:811-866): {T, H, C, E, depth, W} per point.
void refb_climate6(uint64_t world_seed, int32_t large, const int32_t* xs, const int32_t* ys,
                   const int32_t* zs, int32_t n, int32_t* out6) {
    static ClimateState st;
    init_climate_state_mode(st, world_seed, large != 0);
    for (int32_t i = 0; i < n; ++i) {
        const double x = (double)xs[i];
        const double z = (double)zs[i];
        const double px = x + sample_compact_dp(st, C_SHIFT, x, 0.0, z) * 4.0;
        const double pz = z + sample_compact_dp(st, C_SHIFT, z, x, 0.0) * 4.0;
        int32_t* o = out6 + (size_t)i * 6;
        const float c = (float)sample_compact_dp(st, C_CONTINENTALNESS, px, 0.0, pz);
        o[2] = (int32_t)(10000.0F * c);
        const float e = (float)sample_compact_dp(st, C_EROSION, px, 0.0, pz);
        o[3] = (int32_t)(10000.0F * e);
        const float w = (float)sample_compact_dp(st, C_WEIRDNESS, px, 0.0, pz);
        o[5] = (int32_t)(10000.0F * w);
        const float vals[4] = {c, e, mcgpu_peaks_and_valleys(w), w};
        const float off_f = mcgpu_depth_spline(vals) + 0.015F;
        const double d0 = 1.0 - ((double)(ys[i] * 4)) / 128.0 - 83.0 / 160.0 + (double)off_f;
        const float d = (float)d0;
        o[4] = (int32_t)(10000.0F * d);
        const float t = (float)sample_compact_dp(st, C_TEMPERATURE, px, 0.0, pz);
        o[0] = (int32_t)(10000.0F * t);
        const float h = (float)sample_compact_dp(st, C_HUMIDITY, px, 0.0, pz);
        o[1] = (int32_t)(10000.0F * h);
    }
}

// mcgpu_depth_spline (spline_generated.cuh) on {continentalness, erosion, pv, weirdness}.
float refb_depth_spline(const float* v4) { return mcgpu_depth_spline(v4); }

// biome_modern_i32_kernel (MinecraftGPUNoise.cu:915-940): biome ids; -1 for an unknown version.
int32_t refb_biome_at(int32_t version, uint64_t world_seed, int32_t large, const int32_t* xs,
                      const int32_t* ys, const int32_t* zs, int32_t n, int32_t* out) {
    TreeView t;
    if (!select_tree(version, &t)) return -1;
    static ClimateState st;
    init_climate_state_mode(st, world_seed, large != 0);
    for (int32_t i = 0; i < n; ++i)
        out[i] = biome_modern_at(st, t.nodes, t.param, t.len, t.family, xs[i], ys[i], zs[i]);
    return 0;
}

// biome_filter_candidates_kernel (MinecraftGPUNoise.cu:978-1074) as CPU loops: the slime chunks
// of the 221-cell window; per chunk its 16 quarts over quart Y -16..0 (Deep Dark, 183, bit 0) and
// quart Y 16 (Mushroom Fields, 14, bit 1). Candidates are spread over OpenMP threads.
int32_t refb_filter(int32_t version, uint64_t world_seed, int32_t large, const int32_t* ccx,
                    const int32_t* ccz, int32_t n, int32_t flags, int32_t* mask) {
    TreeView t;
    if (!select_tree(version, &t)) return -1;
    static ClimateState st;
    init_climate_state_mode(st, world_seed, large != 0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t i = 0; i < n; ++i) {
        int32_t m = 0;
        for (int ci = 0; ci < 17 * 17; ++ci) {
            const int dx = ci / 17 - 8, dz = ci % 17 - 8;
            if (dx * dx + dz * dz > 68 || !slime_chunk_exact(world_seed, ccx[i] + dx, ccz[i] + dz)) continue;
            for (int q = 0; q < 16; ++q) {
                const int qx = (ccx[i] + dx) * 4 + q / 4, qz = (ccz[i] + dz) * 4 + q % 4;
                if ((flags & 1) && !(m & 1))
                    for (int yi = 0; yi < 17; ++yi)
                        if (biome_modern_at(st, t.nodes, t.param, t.len, t.family, qx, -16 + yi, qz) == 183) {
                            m |= 1;
                            break;
                        }
                if ((flags & 2) && !(m & 2) &&
                    biome_modern_at(st, t.nodes, t.param, t.len, t.family, qx, 16, qz) == 14)
                    m |= 2;
            }
        }
        mask[i] = m;
    }
    return 0;
}

}  // extern "C"
