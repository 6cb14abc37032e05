// band_math.cuh -- the first-draw slime test split at bit 17, shared across period-2^17 bands.
//
// Java's first draw is bits = state1 >> 17 with state1 = state0 * A + 11 (mod 2^48) and
// state0 = (mix ^ 0x5DEECE66D ^ 0x3ad8025f) mod 2^48, mix = X(x) + Z(z) + seed. Split state0
// at bit 17, state0 = L + 2^17 * H:
//     bits = (Q(L) + H * A) mod 2^31,   Q(L) = (L * A + 11) >> 17.
// A first draw is a slime chunk iff bits < 2^31 - 8 and bits % 10 == 0. With
//     y = 2 * bits * inv5 (mod 2^32) = 2*Q*inv5 + H * (2*A*inv5)   (one multiply-add per chunk)
// an even `bits` is a multiple of 10 below the rejection bound iff y < 858993456, and the parity
// of `bits` is bit 0 of Q xor bit 0 of H (A is odd).
//
// Period structure: X(x + 2^17) = X(x) (mod 2^17) and Z(z + 2^17) = Z(z) (mod 2^17), and bit 17
// flips in both. So chunks (x0 + i*2^17, z0 + j*2^17) share L, Q, the carry out of the low 17
// bits and hence D = 2*Q*inv5; their H differ only through the high parts of X and Z; and their
// parity alternates with i + j. Of the two X phases i0, i0+1 exactly one has an even first draw
// in every band, and only that one can be a first-draw slime chunk.
//
// Rejected first draws (bits >= 2^31 - 8, 8 / 2^31 of all chunks) are reported as "not slime"
// here; the rare-state pass adds back the ones that Java's redraw makes slime chunks.
#pragma once

#include <cstdint>

namespace slime {
namespace band {

constexpr int kPeriodBits = 17;
constexpr int64_t kPeriod = 1LL << kPeriodBits;
constexpr uint32_t kA32 = 0xDEECE66Du;                 // low 32 bits of the LCG multiplier
constexpr uint64_t kSeedXor = 0x5E434E432ULL;          // 0x5DEECE66D ^ 0x3ad8025f
constexpr uint32_t kXorLo = (uint32_t)(kSeedXor & 0x1FFFF);
constexpr uint32_t kXorHi = (uint32_t)(kSeedXor >> kPeriodBits);
constexpr uint32_t kInv5 = 0xCCCCCCCDu;
constexpr uint32_t kTwoInv5 = 2u * kInv5;                         // mod 2^32
constexpr uint32_t kMulH = (uint32_t)((2ULL * 0x5DEECE66DULL * kInv5) & 0xFFFFFFFFULL);
constexpr uint32_t kHitBelow = 858993456u;                        // 4 * floor((2^30 - 1) / 5)
constexpr uint32_t kQLimbMul = 5u << 15;                          // (L * 5 * 2^32) >> 17

// Per-(column, row) shared part: D and the parity seed from the low 17 bits of X and Z.
struct Shared {
    uint32_t carry;   // carry out of the low 17 bits of X + Z
    uint32_t d;       // 2 * Q * inv5
    uint32_t q0;      // bit 0 of Q (parity contribution)
};

__host__ __device__ __forceinline__ Shared shared_part(uint32_t x_lo17, uint32_t z_lo17) {
    const uint32_t s = x_lo17 + z_lo17;
    const uint32_t l = (s & 0x1FFFFu) ^ kXorLo;
    const uint64_t prod = (uint64_t)l * kA32 + 11u;
    const uint32_t q = (uint32_t)(prod >> kPeriodBits) + l * kQLimbMul;
    return Shared{s >> kPeriodBits, q * kTwoInv5, q & 1u};
}

// Exact first-draw test of one chunk from full 64-bit terms (used by checks and fix-ups).
__host__ __device__ __forceinline__ bool first_draw_slime(uint64_t xt, uint64_t zt_seeded) {
    const uint64_t state = ((xt + zt_seeded) ^ kSeedXor) * 0x5DEECE66DULL + 0xBULL;
    const uint32_t bits = (uint32_t)(state >> 17) & 0x7FFFFFFFu;
    if (bits >= 2147483640u) return false;
    const uint32_t q = bits * 0xCCCCCCCDu;
    return ((q >> 1) | (q << 31)) <= 0x19999999u;
}

}  // namespace band
}  // namespace slime
