// rare_fix.cu -- exact correction of the first-draw bitmap for Java's nextInt(10) redraws.
//
// The band engine tests only the first draw; a chunk whose first draw is rejected (bits >=
// 2^31 - 8, i.e. LCG state1 in the top 2^20 of the 48-bit ring) is reported as "not slime",
// which is wrong for the ~1/10 of those states that Java's redraw turns into slime chunks
// (SlimeCore.cpp:221-231). There are exactly 104,848 such initial states. This file finds every
// chunk of a search area whose state is one of them and recomputes the affected centres.
//
// Finding them (no scan of the area): a chunk's seed mix is M = X(x) + Z(z) + seed with
// X(x) = sext(x*x*0x4c1906) + sext(x*0x5ac0db) in [-2^32, 2^32). So for a row z the target value
// tau = state0 ^ 0x5E434E432 can only match if tau - (Z(z) + seed) lies within 2^32 of 0 mod 2^48:
// about 3 * 104,848 / 2^16 ~ 5 candidate targets per row (three 2^32-wide buckets of the sorted
// target table). And x -> x*x*0x4c1906 + x*0x5ac0db is a permutation of Z/2^32 (odd linear,
// even quadratic coefficient), so each candidate gives exactly one x: it is recovered bit by bit
// (flipping bit k of x flips bit k of the polynomial and no lower bit), then checked in full.
#include <algorithm>
#include <vector>

#include "band_math.cuh"
#include "engine.h"

namespace slime {
namespace {

constexpr uint64_t kM48 = 0xFFFFFFFFFFFFULL;
constexpr uint32_t kBuckets = 1u << 16;

// Recovers x (mod 2^32) with x*x*0x4c1906 + x*0x5ac0db == d (mod 2^32).
__device__ __forceinline__ uint32_t invert_x_poly(uint32_t d) {
    uint32_t x = 0;
#pragma unroll 4
    for (int k = 0; k < 32; ++k) {
        const uint32_t f = x * x * 0x4c1906u + x * 0x5ac0dbu;
        x |= (f ^ d) & (1u << k);
    }
    return x;
}

__global__ void rare_scan_kernel(const uint64_t* targets, const uint32_t* offsets, int64_t seed,
                                 int32_t z_first, int32_t nz, int32_t x_first, int32_t nx,
                                 int2* out, uint32_t cap, unsigned int* count) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nz) return;
    const int32_t z = (int32_t)((int64_t)z_first + i);
    const uint64_t zz = (z_term(z) + (uint64_t)seed) & kM48;
    const uint32_t b0 = (uint32_t)(zz >> 32);
    for (int db = -1; db <= 1; ++db) {
        const uint32_t b = (b0 + kBuckets + db) & (kBuckets - 1);
        // Bucket -1 of bucket 0 (and +1 of the last) wrap around the 48-bit ring.
        for (uint32_t t = offsets[b]; t < offsets[b + 1]; ++t) {
            const uint64_t d = (targets[t] - zz) & kM48;
            if (d >= (1ULL << 32) && d < kM48 + 1 - (1ULL << 32)) continue;
            const int32_t x = (int32_t)invert_x_poly((uint32_t)d);
            if ((int64_t)x < (int64_t)x_first || (int64_t)x >= (int64_t)x_first + nx) continue;
            if ((x_term(x) & kM48) != d) continue;
            const unsigned int k = atomicAdd(count, 1u);
            if (k < cap) out[k] = make_int2(x, z);
        }
    }
}

// One CTA per rare chunk: the exact bitmap of the 33 x 33 chunks around it, then the exact counts
// of the (up to) 221 centres whose window holds it. A centre shared with an earlier rare chunk of
// the list is left to that one.
__global__ void __launch_bounds__(256) fixup_kernel(const int2* rare, int32_t nrare, int64_t seed,
                                                    FixArgs f) {
    __shared__ uint64_t ex_rows[33];
    __shared__ uint64_t fd_rows[33];  // first-draw bitmap: what the band scan counted
    __shared__ int near_n;
    __shared__ int2 near[32];
    const int r = blockIdx.x;
    if (r >= nrare) return;
    const int2 rc = rare[r];
    const int tid = threadIdx.x;
    if (tid < 33) ex_rows[tid] = fd_rows[tid] = 0;
    if (tid == 0) near_n = 0;
    __syncthreads();
    // Earlier rare chunks close enough to share centres: those centres belong to them.
    for (int k = tid; k < r; k += blockDim.x) {
        const int2 o = rare[k];
        if (abs(o.x - rc.x) <= 16 && abs(o.y - rc.y) <= 16) {
            const int slot = atomicAdd(&near_n, 1);
            if (slot < 32) near[slot] = o;
        }
    }
    for (int e = tid; e < 33 * 33; e += blockDim.x) {
        const int i = e / 33, j = e % 33;  // i: x offset, j: z offset
        const int32_t x = rc.x - 16 + i, z = rc.y - 16 + j;
        const uint64_t xt = x_term(x), zt = z_term(z) + (uint64_t)seed;
        if (slime_from_terms(xt, zt)) atomicOr((unsigned long long*)&ex_rows[j], 1ULL << i);
        if (f.hist_delta && band::first_draw_slime(xt, zt)) atomicOr((unsigned long long*)&fd_rows[j], 1ULL << i);
    }
    __syncthreads();
    if (near_n > 32) {
        if (tid == 0) atomicOr(f.error, 2u);
        return;
    }
    for (int e = tid; e < 17 * 17; e += blockDim.x) {
        const int dx = e % 17 - 8, dz = e / 17 - 8;
        if (dx * dx + dz * dz > 68) continue;
        const int32_t cx = rc.x + dx, cz = rc.y + dz;
        bool owned = true;
        for (int k = 0; k < near_n; ++k) {
            const int64_t ox = (int64_t)cx - near[k].x, oz = (int64_t)cz - near[k].y;
            if (ox * ox + oz * oz <= 68) owned = false;
        }
        if (!owned) continue;
        if ((int64_t)cx < f.area_x0 || (int64_t)cx >= (int64_t)f.area_x0 + f.width ||
            (int64_t)cz < f.area_z0 || (int64_t)cz >= (int64_t)f.area_z0 + f.height)
            continue;
        if (f.rd_min_sq) {
            const int64_t ddx = (int64_t)cx - f.center_x, ddz = (int64_t)cz - f.center_z;
            if (ddx * ddx + ddz * ddz < f.rd_min_sq) continue;
        }
        int ex = 0, fd = 0;
        for (int i = 0; i < 17; ++i) {  // region row dz + 8 + i holds window row i
            ex += __popc((uint32_t)(ex_rows[dz + 8 + i] >> (dx + 8)) & window_row_mask(i));
            fd += __popc((uint32_t)(fd_rows[dz + 8 + i] >> (dx + 8)) & window_row_mask(i));
        }
        if (f.hist_delta) {
            if (fd >= f.min_size && fd <= f.max_size) atomicAdd(&f.hist_delta[fd], -1);
            if (ex >= f.min_size && ex <= f.max_size) atomicAdd(&f.hist_delta[ex], 1);
        }
        if (ex >= f.min_size && ex <= f.max_size) {
            const unsigned long long k = atomicAdd(f.fixed_count, 1ULL);
            if (k < f.cap) f.fixed[k] = Hit{ex, cx, cz};
        }
    }
}

// Marks main-scan hits whose window holds a rare chunk (their first-draw count may be short).
// With the rare list sorted by x, only the entries with |x - hit x| <= 8 are tested (binary search
// for the first one); otherwise all are.
__global__ void filter_hits_kernel(Hit* hits, int64_t n, const int2* rs, int32_t nrare, int sorted) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const Hit h = hits[i];
        int first = 0, last = nrare;
        if (sorted) {
            int lo = 0, hi = nrare;  // first entry with x >= hit x - 8
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if ((int64_t)rs[mid].x < (int64_t)h.cx - 8) lo = mid + 1; else hi = mid;
            }
            first = lo;
        }
        for (int k = first; k < last; ++k) {
            if (sorted && (int64_t)rs[k].x > (int64_t)h.cx + 8) break;
            // 64-bit: centres and rare chunks can lie millions of chunks apart.
            const int64_t dx = (int64_t)h.cx - rs[k].x, dz = (int64_t)h.cz - rs[k].y;
            if (dx * dx + dz * dz <= 68) {
                hits[i].count = -1;
                break;
            }
        }
    }
}

}  // namespace

// The sorted table of the 104,848 seed-mix values (mod 2^48) whose first draw is rejected and
// whose redraw is a slime chunk, with offsets of the 2^16 buckets of their top 16 bits.
void rare_target_table(std::vector<uint64_t>& targets, std::vector<uint32_t>& offsets) {
    const uint64_t mul = 0x5DEECE66DULL;
    // Inverse of the multiplier mod 2^48 (Newton iteration on odd numbers).
    uint64_t inv = mul;
    for (int i = 0; i < 6; ++i) inv = (inv * (2 - mul * inv)) & kM48;
    targets.clear();
    for (uint64_t s1 = kM48 + 1 - (1ULL << 20); s1 <= kM48; ++s1) {
        uint64_t st = s1;
        uint32_t bits;
        do {
            st = (st * mul + 0xB) & kM48;
            bits = (uint32_t)(st >> 17);
        } while (bits >= 2147483640u);
        if (bits % 10 == 0) targets.push_back((((s1 - 0xB) * inv) & kM48) ^ band::kSeedXor);
    }
    std::sort(targets.begin(), targets.end());
    offsets.assign(kBuckets + 1, 0);
    size_t t = 0;
    for (uint32_t b = 0; b <= kBuckets; ++b) {
        while (t < targets.size() && (targets[t] >> 32) < b) ++t;
        offsets[b] = (uint32_t)t;
    }
}

cudaError_t launch_rare_scan(const uint64_t* targets, const uint32_t* offsets, int64_t seed,
                             int32_t z_first, int32_t nz, int32_t x_first, int32_t nx, int2* out,
                             uint32_t cap, unsigned int* count, cudaStream_t s) {
    if (nz <= 0) return cudaSuccess;
    rare_scan_kernel<<<(nz + 255) / 256, 256, 0, s>>>(targets, offsets, seed, z_first, nz, x_first,
                                                      nx, out, cap, count);
    return cudaGetLastError();
}

cudaError_t launch_fixup(const int2* rare, int32_t nrare, int64_t seed, const FixArgs& f,
                         cudaStream_t s) {
    if (nrare <= 0) return cudaSuccess;
    fixup_kernel<<<nrare, 256, 0, s>>>(rare, nrare, seed, f);
    return cudaGetLastError();
}

cudaError_t launch_filter_hits(Hit* hits, int64_t n, const int2* rare, int32_t nrare, bool sorted_by_x,
                               cudaStream_t s) {
    if (n <= 0 || nrare <= 0) return cudaSuccess;
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    filter_hits_kernel<<<grid, 256, 0, s>>>(hits, n, rare, nrare, sorted_by_x ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace slime
