// slime_core.cuh -- shared definitions of the B200 slime-chunk cluster search.
//
// A chunk (x, z) is a slime chunk when Java's
//   new Random(seed + (int)(x*x*0x4c1906) + (int)(x*0x5ac0db) + (int)(z*z)*0x4307a7L
//              + (int)(z*0x5f24f) ^ 0x3ad8025fL).nextInt(10) == 0
// (SlimeCore.cpp:208-232). The cluster size of a centre chunk is the number of slime chunks in
// the 221-cell AFK window dx^2 + dz^2 <= 68 (SlimeCore.cpp:399-404).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace slime {

constexpr uint64_t kLcgMult = 0x5DEECE66DULL;
constexpr uint64_t kLcgAdd = 0xBULL;
constexpr uint64_t kMask48 = 0xFFFFFFFFFFFFULL;
// java.util.Random(long) XORs the multiplier into the seed; the slime formula XORs 0x3ad8025f.
constexpr uint64_t kSeedXor = 0x3AD8025FULL ^ kLcgMult;
// next(31) values at or above this are redrawn by nextInt(10) (Java's bound check).
constexpr uint32_t kRejectFrom = 2147483640u;

// Result record of the reference C ABI (SlimeCoreGPU.cu:198-205), 24 bytes.
struct ExtChunkResult {
    int32_t size;
    int32_t center_x;
    int32_t center_z;
    int32_t obs_count;
    int32_t afk_x;
    int32_t afk_z;
};
static_assert(sizeof(ExtChunkResult) == 24, "ABI record size");

// What a scan kernel writes for each centre it keeps: the exact count and chunk coordinates.
struct Hit {
    int32_t count;
    int32_t cx;
    int32_t cz;
};

// Half-widths of the 17 window rows (dz = -8..8): largest k with dz^2 + k^2 <= 68.
__host__ __device__ constexpr int window_half_width(int i) {
    return i == 0 || i == 16 ? 2 : i == 1 || i == 15 ? 4 : i == 2 || i == 14 ? 5
         : i == 3 || i == 13 ? 6 : i == 4 || i == 5 || i == 11 || i == 12 ? 7 : 8;
}

// 17-bit mask of the cells of window row i inside the circle, bit k = column offset k - 8.
__host__ __device__ constexpr uint32_t window_row_mask(int i) {
    return ((1u << (2 * window_half_width(i) + 1)) - 1u) << (8 - window_half_width(i));
}

// x and z parts of the Java seed mix with 32-bit wrap and sign extension (SlimeCore.cpp:209-214).
__host__ __device__ __forceinline__ uint64_t x_term(int32_t x) {
    const uint32_t u = (uint32_t)x;
    return (uint64_t)(int64_t)(int32_t)(u * u * 0x4c1906u) +
           (uint64_t)(int64_t)(int32_t)(u * 0x5ac0dbu);
}
__host__ __device__ __forceinline__ uint64_t z_term(int32_t z) {
    const uint32_t u = (uint32_t)z;
    return (uint64_t)(int64_t)(int32_t)(u * u) * 0x4307a7ULL +
           (uint64_t)(int64_t)(int32_t)(u * 0x5f24fu);
}

// Exact divisibility of a 31-bit value by 10: multiply by the inverse of 5 modulo 2^32 and
// rotate the parity bit to the top (a multiple of 10 maps below 2^32 / 10).
__host__ __device__ __forceinline__ bool divisible_by_10(uint32_t v) {
    const uint32_t q = v * 0xCCCCCCCDu;
    return ((q >> 1) | (q << 31)) <= 0x19999999u;
}

// Java's nextInt(10) redraw loop from a first LCG state that was rejected.
__host__ __device__ __noinline__ inline bool slime_redraw(uint64_t state) {
    for (;;) {
        state = (state * kLcgMult + kLcgAdd) & kMask48;
        const uint32_t bits = (uint32_t)(state >> 17);
        const uint32_t val = bits % 10u;
        if (bits - val + 9u <= 0x7FFFFFFFu) return val == 0;
    }
}

// Exact predicate from the two precomputed parts (the seed is folded into the z part).
// The state is only reduced mod 2^48 where it matters: the low 48 bits of a product depend
// only on the low 48 bits of its factors.
__host__ __device__ __forceinline__ bool slime_from_terms(uint64_t xt, uint64_t zt_seeded) {
    const uint64_t state = ((xt + zt_seeded) ^ kSeedXor) * kLcgMult + kLcgAdd;
    const uint32_t bits = (uint32_t)(state >> 17) & 0x7FFFFFFFu;
    if (bits < kRejectFrom) return divisible_by_10(bits);
    return slime_redraw(state & kMask48);
}

// True when every centre of the rectangle [x0, x1] x [z0, z1] (chunk coordinates) lies strictly
// inside the rd_min disc about (cx, cz), i.e. its farthest corner is closer than rd_min: an annulus
// search keeps none of them.
__host__ __device__ __forceinline__ bool rect_inside_disc(int64_t x0, int64_t x1, int64_t z0, int64_t z1, int64_t cx,
                                                          int64_t cz, int64_t rd_min_sq) {
    const int64_t dx = cx - x0 > x1 - cx ? cx - x0 : x1 - cx;
    const int64_t dz = cz - z0 > z1 - cz ? cz - z0 : z1 - cz;
    return dx * dx + dz * dz < rd_min_sq;
}

__host__ __device__ __forceinline__ bool is_slime(int64_t seed, int64_t x, int64_t z) {
    return slime_from_terms(x_term((int32_t)x), z_term((int32_t)z) + (uint64_t)seed);
}

}  // namespace slime
