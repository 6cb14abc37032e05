// precise.cu -- precise AFK scoring of ranked sites.
//
// Semantics of score_candidates_precise (SlimeCore.cpp:654-726): for each site and each offset
// (dx, dz) in {-16..16 step 4}^2 (or only (0,0) without the XZ scan) and each Y level, count the
// block columns of slime chunks inside the annulus 24^2 < dx^2 + dy^2 + dz^2 <= 128^2 around the
// offset position (count_spawnable_cached_table, SlimeCore.cpp:291-331); keep the strict maximum,
// first in (dx, dz, Y) order, starting from 0 at the site centre.
//
// B200 design: one CTA per site builds a 23 x 23 chunk bitmap covering all 81 windows once; a
// precomputed table gives each slime chunk's block-column count for the window alignment
// (o mod 16 on each axis), the chunk's place in the 21 x 21 window and the Y level, so a score is
// a sum of table entries over the window's slime chunks. Threads split the (offset, Y) pairs and
// a block reduction picks (max obs, first order).
#include "engine.h"

namespace slime {
namespace {

constexpr int kPreciseTpb = 128;
constexpr int kDxMin = -128, kDxCount = 257;

__device__ __forceinline__ int64_t floor_div16(int64_t v) { return v >> 4; }

__device__ __forceinline__ int interval_len(int a, int b) { return b >= a ? b - a + 1 : 0; }

// weights[(((ax * 16 + az) * 21 + i) * 21 + j) * y_count + yi]
__global__ void weight_table_kernel(uint16_t* weights, const int16_t* outer, const int16_t* inner,
                                    int32_t y_count) {
    const int64_t total = 16LL * 16 * 21 * 21 * y_count;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int yi = (int)(e % y_count);
        int64_t rest = e / y_count;
        const int j = (int)(rest % 21); rest /= 21;
        const int i = (int)(rest % 21); rest /= 21;
        const int az = (int)(rest % 16);
        const int ax = (int)(rest / 16);
        // Block offsets of the chunk relative to the scored position.
        const int rx0 = (i - 10) * 16 - ax, rz0 = (j - 10) * 16 - az;
        const int x0 = max(-128, rx0), x1 = min(128, rx0 + 15);
        const int z0 = max(-128, rz0), z1 = min(128, rz0 + 15);
        const int16_t* o = outer + (int64_t)yi * kDxCount;
        const int16_t* n = inner + (int64_t)yi * kDxCount;
        int total_cols = 0;
        if (z0 <= z1) {
            for (int dx = x0; dx <= x1; ++dx) {
                const int ro = o[dx - kDxMin];
                if (ro < 0) continue;
                const int zl = max(z0, -ro), zr = min(z1, ro);
                int add = interval_len(zl, zr);
                if (!add) continue;
                const int ri = n[dx - kDxMin];
                if (ri >= 0) add -= interval_len(max(zl, -ri), min(zr, ri));
                total_cols += add;
            }
        }
        weights[e] = (uint16_t)total_cols;
    }
}

__global__ void __launch_bounds__(kPreciseTpb) precise_kernel(const PreciseArgs a) {
    __shared__ uint32_t bits[24];
    __shared__ int s_obs[kPreciseTpb];
    __shared__ int s_ord[kPreciseTpb];
    const int tid = threadIdx.x;
    const int lo = a.scan_xz ? -16 : 0, hi = a.scan_xz ? 16 : 0;
    const int side = a.scan_xz ? 9 : 1;
    const int pairs = side * side * a.y_count;

    for (int site = blockIdx.x; site < a.n; site += gridDim.x) {
        const int64_t bx = a.sites[site].center_x, bz = a.sites[site].center_z;
        const int64_t ux0 = floor_div16(bx + lo) - 10, uz0 = floor_div16(bz + lo) - 10;
        const int nx = (int)(floor_div16(bx + hi) + 10 - ux0 + 1);
        const int nz = (int)(floor_div16(bz + hi) + 10 - uz0 + 1);
        if (tid < 24) bits[tid] = 0;
        __syncthreads();
        for (int e = tid; e < nx * nz; e += kPreciseTpb) {
            const int i = e / nz, j = e % nz;
            if (is_slime(a.seed, ux0 + i, uz0 + j)) atomicOr(&bits[i], 1u << j);
        }
        __syncthreads();

        int best = -1, best_ord = 0x7FFFFFFF;
        for (int p = tid; p < pairs; p += kPreciseTpb) {
            const int off = p / a.y_count, yi = p % a.y_count;
            const int64_t ox = bx + lo + (off / side) * 4, oz = bz + lo + (off % side) * 4;
            const int wx = (int)(floor_div16(ox) - 10 - ux0), wz = (int)(floor_div16(oz) - 10 - uz0);
            const uint16_t* w = a.weights +
                (int64_t)(((int)(ox & 15) * 16 + (int)(oz & 15)) * 441) * a.y_count + yi;
            int obs = 0;
            for (int i = 0; i < 21; ++i) {
                uint32_t row = (bits[wx + i] >> wz) & 0x1FFFFFu;
                while (row) {
                    const int j = __ffs(row) - 1;
                    row &= row - 1;
                    obs += w[(int64_t)(i * 21 + j) * a.y_count];
                }
            }
            if (obs > best) { best = obs; best_ord = p; }  // p ascends: first maximum wins
        }
        s_obs[tid] = best;
        s_ord[tid] = best_ord;
        __syncthreads();
        for (int stride = kPreciseTpb / 2; stride > 0; stride >>= 1) {
            if (tid < stride) {
                const int ob = s_obs[tid + stride], od = s_ord[tid + stride];
                if (ob > s_obs[tid] || (ob == s_obs[tid] && od < s_ord[tid])) {
                    s_obs[tid] = ob;
                    s_ord[tid] = od;
                }
            }
            __syncthreads();
        }
        if (tid == 0) {
            int obs = s_obs[0];
            int64_t ax = bx, az = bz;
            int y = a.platform_y;
            if (obs > 0) {
                const int off = s_ord[0] / a.y_count, yi = s_ord[0] % a.y_count;
                ax = bx + lo + (off / side) * 4;
                az = bz + lo + (off % side) * 4;
                y = a.y_values[yi];
            } else {
                obs = 0;
            }
            ExtChunkResult& r = a.sites[site];
            r.obs_count = a.pack_y ? (int32_t)((uint32_t)obs | ((uint32_t)(y + 1024) << 20)) : obs;
            r.afk_x = (int32_t)ax;
            r.afk_z = (int32_t)az;
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_weight_table(uint16_t* weights, const int16_t* outer, const int16_t* inner,
                                int32_t y_count, cudaStream_t s) {
    const int64_t total = 16LL * 16 * 21 * 21 * y_count;
    const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
    weight_table_kernel<<<blocks, 256, 0, s>>>(weights, outer, inner, y_count);
    return cudaGetLastError();
}

cudaError_t launch_precise(const PreciseArgs& a, cudaStream_t s) {
    if (a.n <= 0) return cudaSuccess;
    const int grid = a.n < 148 * 16 ? a.n : 148 * 16;
    precise_kernel<<<grid, kPreciseTpb, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace slime
