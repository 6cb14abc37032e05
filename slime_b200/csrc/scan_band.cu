// scan_band.cu -- the band engine: large searches with a shared-LCG bitmap generator.
//
// Behaviour: the same kept set as the general scan (SlimeCoreGPU.cu:501-610 semantics) for
// first-draw slime chunks; the rare Java redraws are added back by rare_fix.cu.
//
// B200 design (see band_math.cuh for the arithmetic):
//  * A CTA owns one base tile -- 1,024 base columns x (band_h + 16) base rows -- and evaluates it
//    for two X phases (x and x + 2^17) and up to 32 Z bands (z + j * 2^17) at once. Per chunk
//    position the low-17-bit work (carry, Q, D, parity) is done once; per band it costs one add,
//    one xor, one multiply-add, one compare and one ballot for the two phases together, because
//    the parity tells which of the two phases can be a first-draw slime chunk.
//  * Ballots land in a 20-row shared ring (one plane per band plus the phase-swap plane).
//  * Counting is SWAR in byte lanes on 4x4 centre groups: nibble popcounts of 4 rows give 4x4
//    block counts, three funnel shifts and two adds give the 20-column sums of 8 groups per word,
//    and a rolling sum over 5 row batches gives the 20x20 box that bounds the 16 circles. Groups
//    whose box reaches the threshold get exact 221-cell counts from the ring (one popcount per
//    window row, spread over the whole CTA), and those in range are appended to the hit list.
#include "band_math.cuh"
#include "engine.h"

namespace slime {
namespace {

using namespace band;

constexpr int kTpb = 512;
constexpr int kWords = 32;                  // words per ring row: 1,024 base columns
constexpr int kOutW = kWords * 32 - 16;     // 1,008 centres per tile row
constexpr int kMaxBands = 32;
constexpr int kSwPlane = kMaxBands;         // plane of the phase-swap ballot
constexpr int kPlanes = kMaxBands + 4;      // 16-byte aligned rows of planes
constexpr int kRing = 20;                   // rows in the ring (5 batches of 4)
constexpr int kMaxCombos = 2 * kMaxBands;
constexpr int kMaxPairs = kMaxCombos * kWords;
constexpr int kSlots = kMaxPairs / kTpb;    // (combo, word) pairs per thread
constexpr int kSurvCap = 192;               // survivor groups processed per round
constexpr unsigned kFull = 0xFFFFFFFFu;

struct __align__(16) BandSmem {
    uint32_t ring[kRing][kWords + 1][kPlanes];   // word kWords is a zero pad
    uint32_t hist_e[5][kMaxPairs];
    uint32_t hist_o[5][kMaxPairs];
    uint32_t eo_e[kMaxCombos][kWords + 1];
    uint32_t eo_o[kMaxCombos][kWords + 1];
    uint32_t rows[4][kMaxBands + 1];             // batch row terms: [0] low 17 bits, [1+m] high
    uint32_t surv[kSurvCap];                     // (pair << 3) | group
    int cnt[kSurvCap * 16];
    int nsurv;
    int any;
};

__device__ __forceinline__ uint32_t nibble_counts(uint32_t r) {
    const uint32_t a = r - ((r >> 1) & 0x55555555u);
    return (a & 0x33333333u) + ((a >> 2) & 0x33333333u);
}

// Maps the per-byte "reached" bits of the even (te) and odd (to) group sums to an 8-bit mask.
__device__ __forceinline__ uint32_t group_mask(uint32_t te, uint32_t to) {
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        m |= ((te >> (8 * k + 7)) & 1u) << (2 * k);
        m |= ((to >> (8 * k + 7)) & 1u) << (2 * k + 1);
    }
    return m;
}

__global__ void __launch_bounds__(kTpb, 1) band_scan_kernel(const BandArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BandSmem& S = *reinterpret_cast<BandSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nb = a.nb, ncombo = 2 * nb, npairs = ncombo * kWords;
    const uint32_t bias = (uint32_t)(128 - a.min_size) * 0x01010101u;
    const bool no_upper = a.max_size >= 221;
    uint32_t guard = 0;

    // Zero pads that are never written: ring word kWords and the E/O pad word.
    for (int i = tid; i < kRing * kPlanes; i += kTpb) S.ring[i / kPlanes][kWords][i % kPlanes] = 0;
    for (int i = tid; i < kMaxCombos; i += kTpb) {
        S.eo_e[i][kWords] = 0;
        S.eo_o[i][kWords] = 0;
    }

    for (int64_t tile = a.tile_begin + blockIdx.x; tile < a.tile_end; tile += gridDim.x) {
        const int ut = (int)(tile % a.u_tiles);
        const int64_t rest = tile / a.u_tiles;
        const int vt = (int)(rest % a.v_tiles);
        const int pp = (int)(rest / a.v_tiles);
        const int i0 = 2 * pp;
        const int u0 = ut * kOutW;
        const int v0 = vt * a.band_h;
        const int out_h = min(a.band_h, a.vbase - v0);
        const int batches = (out_h + 16 + 3) / 4;

        // Column terms of this thread's two generator words, for phases i0 and i0 + 1.
        uint32_t lox[2], xh0[2], xh1[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int64_t idx0 = (int64_t)u0 + (warp * 2 + k) * 32 + lane + (int64_t)i0 * kPeriod;
            const uint64_t x0 = idx0 < a.ncols ? a.ct[idx0] : 0;
            const uint64_t x1 = idx0 + kPeriod < a.ncols ? a.ct[idx0 + kPeriod] : 0;
            lox[k] = (uint32_t)x0 & 0x1FFFFu;
            xh0[k] = (uint32_t)(x0 >> kPeriodBits);
            xh1[k] = (uint32_t)(x1 >> kPeriodBits);
        }
        uint32_t re[kSlots], ro[kSlots];
#pragma unroll
        for (int k = 0; k < kSlots; ++k) re[k] = ro[k] = 0;
        for (int i = tid; i < 5 * kMaxPairs; i += kTpb) {
            (&S.hist_e[0][0])[i] = 0;
            (&S.hist_o[0][0])[i] = 0;
        }
        __syncthreads();

        for (int b = 0; b < batches; ++b) {
            // (1) Row terms of the batch's 4 input rows (low 17 bits and the band high parts).
            for (int i = tid; i < 4 * (nb + 1); i += kTpb) {
                const int q = i / (nb + 1), e = i % (nb + 1);
                const int vi = v0 + 4 * b + q;
                S.rows[q][e] = vi < a.vrows ? a.rt[(int64_t)vi * a.rstride + (e == 0 ? 0 : a.j0 + e)] : 0u;
            }
            __syncthreads();

            // (2) Generator: 4 rows x 2 words per warp.
#pragma unroll 1
            for (int q = 0; q < 4; ++q) {
                const int slot = (4 * b + q) % kRing;
                const uint32_t zlo = S.rows[q][0];
                const uint32_t zpar = (S.rows[q][1] ^ kXorHi) & 1u;
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const int word = warp * 2 + k;
                    const Shared sh = shared_part(lox[k], zlo);
                    const uint32_t pi = (sh.q0 ^ xh0[k] ^ sh.carry ^ zpar) & 1u;
                    const uint32_t xa = (pi ? xh1[k] : xh0[k]) + sh.carry;
                    const uint32_t xb = (pi ? xh0[k] : xh1[k]) + sh.carry;
                    const uint32_t sw = __ballot_sync(kFull, pi != 0);
                    uint32_t* dst = &S.ring[slot][word][0];
                    int m = 0;
                    for (; m + 1 < nb; m += 2) {
                        const uint32_t ha = ((xa + S.rows[q][1 + m]) ^ kXorHi) * kMulH + sh.d;
                        const uint32_t hb = ((xb + S.rows[q][2 + m]) ^ kXorHi) * kMulH + sh.d;
                        const uint32_t wa = __ballot_sync(kFull, ha < kHitBelow);
                        const uint32_t wb = __ballot_sync(kFull, hb < kHitBelow);
                        if (lane == 0) *reinterpret_cast<uint2*>(dst + m) = make_uint2(wa, wb);
                    }
                    if (m < nb) {
                        const uint32_t ha = ((xa + S.rows[q][1 + m]) ^ kXorHi) * kMulH + sh.d;
                        const uint32_t wa = __ballot_sync(kFull, ha < kHitBelow);
                        if (lane == 0) dst[m] = wa;
                    }
                    if (lane == 0) dst[kSwPlane] = sw;
                }
            }
            __syncthreads();

            // (3) 4x4 block counts of the batch, per (combo, word): E = even nibbles, O = odd.
#pragma unroll
            for (int k = 0; k < kSlots; ++k) {
                const int p = tid + k * kTpb;
                if (p < npairs) {
                    const int combo = p % ncombo, word = p / ncombo;
                    const int m = combo >> 1;
                    const uint32_t flip = (uint32_t)((combo ^ m) & 1);  // phase ^ band parity
                    uint32_t n[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const uint32_t* row = &S.ring[(4 * b + q) % kRing][word][0];
                        const uint32_t sw = row[kSwPlane];
                        n[q] = nibble_counts(row[m] & (flip ? sw : ~sw));
                    }
                    const uint32_t n01 = n[0] + n[1], n23 = n[2] + n[3];
                    S.eo_e[combo][word] = (n01 & 0x0F0F0F0Fu) + (n23 & 0x0F0F0F0Fu);
                    S.eo_o[combo][word] = ((n01 >> 4) & 0x0F0F0F0Fu) + ((n23 >> 4) & 0x0F0F0F0Fu);
                }
            }
            if (tid == 0) { S.any = 0; S.nsurv = 0; }
            __syncthreads();

            // (4) 20-column group sums, rolling 20x20 boxes, threshold test.
            const int hs = b % 5;
            uint32_t pend[kSlots];
#pragma unroll
            for (int k = 0; k < kSlots; ++k) {
                pend[k] = 0;
                const int p = tid + k * kTpb;
                if (p < npairs) {
                    const int combo = p % ncombo, word = p / ncombo;
                    const uint32_t e = S.eo_e[combo][word], en = S.eo_e[combo][word + 1];
                    const uint32_t o = S.eo_o[combo][word], on = S.eo_o[combo][word + 1];
                    const uint32_t s = e + o, sn = en + on;
                    const uint32_t s1 = __funnelshift_r(s, sn, 8);
                    const uint32_t ge = s + s1 + __funnelshift_r(e, en, 16);
                    const uint32_t go = o + s1 + __funnelshift_r(s, sn, 16);
                    guard |= ge | go;
                    re[k] += ge - S.hist_e[hs][p];
                    ro[k] += go - S.hist_o[hs][p];
                    S.hist_e[hs][p] = ge;
                    S.hist_o[hs][p] = go;
                    if (b >= 4) {
                        const uint32_t te = (re[k] + bias) & 0x80808080u;
                        const uint32_t to = (ro[k] + bias) & 0x80808080u;
                        if (te | to) {
                            uint32_t gm = group_mask(te, to);
                            if (word == kWords - 1) gm &= 0x0Fu;  // centres 1,008.. do not exist
                            pend[k] = gm;
                            if (gm) S.any = 1;
                        }
                    }
                }
            }
            __syncthreads();

            // (5) Exact 221-cell counts of surviving groups, in rounds of kSurvCap groups.
            if (S.any) {
                for (;;) {
#pragma unroll
                    for (int k = 0; k < kSlots; ++k) {
                        while (pend[k]) {
                            const int g = __ffs(pend[k]) - 1;
                            const int idx = atomicAdd(&S.nsurv, 1);
                            if (idx >= kSurvCap) break;
                            S.surv[idx] = ((uint32_t)(tid + k * kTpb) << 3) | (uint32_t)g;
                            pend[k] &= pend[k] - 1;
                        }
                    }
                    __syncthreads();
                    const int n = min(S.nsurv, kSurvCap);
                    for (int i = tid; i < n * 16; i += kTpb) S.cnt[i] = 0;
                    __syncthreads();
                    for (int it = tid; it < n * 16 * 17; it += kTpb) {
                        const int s = it / (16 * 17), rem = it % (16 * 17);
                        const int d = rem / 17, i = rem % 17;
                        const uint32_t rec = S.surv[s];
                        const int p = (int)(rec >> 3), g = (int)(rec & 7);
                        const int combo = p % ncombo, word = p / ncombo, m = combo >> 1;
                        const uint32_t flip = (uint32_t)((combo ^ m) & 1);
                        const int c = word * 32 + 4 * g + (d & 3);
                        const int rr = 4 * (b - 4) + (d >> 2);
                        const uint32_t* row = &S.ring[(rr + i) % kRing][0][0];
                        const int w0 = c >> 5;
                        const uint32_t sw0 = row[w0 * kPlanes + kSwPlane], sw1 = row[(w0 + 1) * kPlanes + kSwPlane];
                        const uint32_t lo = row[w0 * kPlanes + m] & (flip ? sw0 : ~sw0);
                        const uint32_t hi = row[(w0 + 1) * kPlanes + m] & (flip ? sw1 : ~sw1);
                        const uint32_t bits = __funnelshift_r(lo, hi, c & 31) & window_row_mask(i);
                        if (bits) atomicAdd(&S.cnt[s * 16 + d], __popc(bits));
                    }
                    __syncthreads();
                    for (int e = tid; e < n * 16; e += kTpb) {
                        const int s = e >> 4, d = e & 15;
                        const int count = S.cnt[e];
                        if (count < a.min_size || (!no_upper && count > a.max_size)) continue;
                        const uint32_t rec = S.surv[s];
                        const int p = (int)(rec >> 3), g = (int)(rec & 7);
                        const int combo = p % ncombo, word = p / ncombo;
                        const int c = word * 32 + 4 * g + (d & 3);
                        const int rr = 4 * (b - 4) + (d >> 2);
                        const int64_t u = (int64_t)u0 + c, v = (int64_t)v0 + rr;
                        if (c >= kOutW || u >= a.ubase || rr >= out_h) continue;
                        const int64_t cu = u + (int64_t)(i0 + (combo & 1)) * kPeriod;
                        const int64_t cv = v + (int64_t)(a.j0 + (combo >> 1)) * kPeriod;
                        if (cu >= a.width_u || cv >= a.height_v) continue;
                        const int32_t cx = (int32_t)(a.transposed ? a.area_x0 + cv : a.area_x0 + cu);
                        const int32_t cz = (int32_t)(a.transposed ? a.area_z0 + cu : a.area_z0 + cv);
                        if (a.rd_min_sq) {
                            const int64_t dx = (int64_t)cx - a.center_x, dz = (int64_t)cz - a.center_z;
                            if (dx * dx + dz * dz < a.rd_min_sq) continue;
                        }
                        const unsigned long long idx = atomicAdd(a.emitted, 1ULL);
                        if (idx < a.cap) a.out[idx] = Hit{count, cx, cz};
                    }
                    const int more = __syncthreads_or((pend[0] | pend[1] | pend[2] | pend[3]) != 0);
                    if (!more) break;
                    if (tid == 0) S.nsurv = 0;
                    __syncthreads();
                }
            }
        }
        __syncthreads();
    }
    // A 4-row strip with 32+ hits among 80 cells could carry a box past a byte lane.
    if (guard & 0xE0E0E0E0u) atomicOr(a.overflow, 1u);
}

// rt[v * stride + 0] = low 17 bits of the row term of base row v; rt[v * stride + 1 + j] = its
// high part (>> 17) in band j, for base rows v < vrows and bands j < nj (0 outside the area).
__global__ void row_terms_kernel(uint32_t* rt, int32_t stride, int32_t vrows, int32_t nj,
                                 int32_t first, int64_t limit, int64_t seed, int32_t use_x_term) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)vrows * nj) return;
    const int32_t v = (int32_t)(e / nj), j = (int32_t)(e % nj);
    const int64_t off = (int64_t)v + (int64_t)j * kPeriod;
    uint64_t t = 0;
    if (off < limit) {
        const int32_t c = (int32_t)((int64_t)first + off);
        t = use_x_term ? x_term(c) + (uint64_t)seed : z_term(c) + (uint64_t)seed;
    }
    if (j == 0) rt[(int64_t)v * stride] = (uint32_t)t & 0x1FFFFu;
    rt[(int64_t)v * stride + 1 + j] = (uint32_t)(t >> kPeriodBits);
}

__global__ void col_terms_kernel(uint64_t* ct, int32_t first, int32_t n, int32_t use_x_term) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t c = (int32_t)((int64_t)first + i);
    ct[i] = use_x_term ? x_term(c) : z_term(c);
}

}  // namespace

size_t band_smem_bytes() { return sizeof(BandSmem); }
int band_tile_out_w() { return kOutW; }
int band_max_bands() { return kMaxBands; }

cudaError_t band_prepare() {
    return cudaFuncSetAttribute(band_scan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(BandSmem));
}

cudaError_t launch_band_scan(const BandArgs& a, int grid, cudaStream_t s) {
    band_scan_kernel<<<grid, kTpb, sizeof(BandSmem), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_band_terms(uint64_t* ct, int32_t col_first, int32_t ncols, uint32_t* rt,
                              int32_t rstride, int32_t vrows, int32_t nj, int32_t row_first,
                              int64_t row_limit, int64_t seed, bool transposed, cudaStream_t s) {
    // Columns carry no seed; rows carry it. Transposed searches swap which axis is x.
    col_terms_kernel<<<(ncols + 255) / 256, 256, 0, s>>>(ct, col_first, ncols, transposed ? 0 : 1);
    const int64_t n = (int64_t)vrows * nj;
    row_terms_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(rt, rstride, vrows, nj, row_first,
                                                                row_limit, seed, transposed ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace slime
