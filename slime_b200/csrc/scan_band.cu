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
//  * Rows advance in batches of 4. Ballots of a batch go to one of two 4-row buffers, so one
//    barrier per batch separates the generator (batch b+1) from the counter (batch b).
//  * Counting is SWAR in byte lanes on 4x4 centre groups. A warp owns a combo (phase, band) row
//    with one lane per 32-column word: nibble popcounts of the 4 rows give 4x4 block counts,
//    the neighbour word comes by shuffle, three funnel shifts and two adds give the 20-column
//    strip sums of the word's 8 groups, and a rolling sum over 5 batches gives the 20x20 box of
//    each group, which bounds its 16 windows. A flagged group is re-tested in registers with
//    the 32 cells of rows 0, 1, 18 and 19 that lie outside every window removed (368 cells).
//  * Groups that pass both go to a queue; the CTA re-evaluates queued groups from the term
//    tables (one warp per group: 20 x 20 first-draw bits, 16 exact window counts) and appends
//    the centres in range to the hit list.
#include "band_math.cuh"
#include "engine.h"

namespace slime {
namespace {

using namespace band;

constexpr int kTpb = 512;
constexpr int kWarps = kTpb / 32;
constexpr int kWords = 32;                  // words per ring row: 1,024 base columns
constexpr int kOutW = kWords * 32 - 16;     // 1,008 centres per tile row
constexpr int kMaxBands = 32;
constexpr int kSwPlane = kMaxBands;         // plane of the phase-swap ballot
constexpr int kPlanes = kMaxBands + 4;      // 16-byte aligned word records
constexpr int kMaxCombos = 2 * kMaxBands;
constexpr int kSlots = kMaxCombos / kWarps; // combo rows counted per warp
constexpr int kQueueCap = 1024;
constexpr int kQueueFlush = 512;
constexpr unsigned kFull = 0xFFFFFFFFu;

struct __align__(16) BandSmem {
    uint32_t ring[2][4][kWords][kPlanes];     // [buffer][row][word][band planes | swap plane]
    uint32_t hist_e[5][kMaxCombos][kWords];   // strip sums of the last 5 batches (even groups)
    uint32_t hist_o[5][kMaxCombos][kWords];   // (odd groups)
    uint32_t hist_n[5][kMaxCombos][kWords];   // nibble counts of rows 0+1 of the last 5 batches
    uint32_t rows[3][4][kMaxBands + 4];       // row terms of 3 batches: [m] high part in band m,
                                              // [kMaxBands] low 17 bits (16-byte aligned rows)
    uint32_t rvalid[3][4];                    // bit m: the row exists in band m
    uint32_t queue[kQueueCap];                // combo << 24 | word << 19 | group << 16 | batch
    uint32_t scratch[kWarps][20];             // re-evaluation rows, one block per warp
    int qcount;
    int qover;
};

__device__ __forceinline__ uint32_t nibble_counts(uint32_t r) {
    const uint32_t a = r - ((r >> 1) & 0x55555555u);
    return (a & 0x33333333u) + ((a >> 2) & 0x33333333u);
}

// Per byte: high bit set where v >= t (v, t < 256; borrow-free because v | 0x80 >= 128 >= t').
// Bytes >= 128 always report (a superset is safe: flagged groups are re-tested).
__device__ __forceinline__ uint32_t bytes_at_least(uint32_t v, uint32_t t4) {
    return (((v | 0x80808080u) - t4) | v) & 0x80808080u;
}

// Appends the groups of `gm` to the queue; returns those that did not fit (kept pending).
__device__ __forceinline__ uint32_t push_groups(BandSmem& S, int combo, int word, uint32_t gm, int b) {
    while (gm) {
        const int g = __ffs(gm) - 1;
        const int idx = atomicAdd(&S.qcount, 1);
        if (idx >= kQueueCap) {
            S.qover = 1;
            return gm;
        }
        S.queue[idx] = ((uint32_t)combo << 24) | ((uint32_t)word << 19) | ((uint32_t)g << 16) | (uint32_t)b;
        gm &= gm - 1;
    }
    return 0;
}

struct Tile {
    int u0, v0, i0, out_h;
};

// Re-evaluates the queued groups from the term tables and appends the centres in range.
__device__ void flush_queue(BandSmem& S, const BandArgs& a, const Tile& T, int warp, int lane) {
    const int n = min(S.qcount, kQueueCap);
    const bool no_upper = a.max_size >= 221;
    for (int s = warp; s < n; s += kWarps) {
        const uint32_t rec = S.queue[s];
        const int combo = (int)(rec >> 24), word = (int)((rec >> 19) & 31);
        const int g = (int)((rec >> 16) & 7), b = (int)(rec & 0xFFFF);
        const int ph = combo & 1, m = combo >> 1;
        const int c0 = word * 32 + 4 * g;       // first window column (tile-relative input col)
        const int r0 = 4 * (b - 4);             // first window row (tile-relative input row)
        uint64_t xt = 0;
        if (lane < 20) {
            const int64_t idx = (int64_t)T.u0 + c0 + lane + (int64_t)(T.i0 + ph) * kPeriod;
            xt = idx < a.ncols ? a.ct[idx] : 0;
        }
        for (int t = 0; t < 20; ++t) {
            const int vi = T.v0 + r0 + t;
            uint64_t zt = 0;
            if (vi < a.vrows) {
                const uint32_t* row = a.rt + (int64_t)vi * a.rstride;
                zt = (uint64_t)row[0] | ((uint64_t)row[1 + a.j0 + m] << kPeriodBits);
            }
            const uint32_t bits = __ballot_sync(kFull, lane < 20 && first_draw_slime(xt, zt));
            if (lane == 0) S.scratch[warp][t] = bits;
        }
        __syncwarp();
        bool keep = false;
        int count = 0, cx = 0, cz = 0;
        if (lane < 16) {
            const int dx = lane & 3, dz = lane >> 2;
#pragma unroll
            for (int i = 0; i < 17; ++i)
                count += __popc((S.scratch[warp][dz + i] >> dx) & window_row_mask(i));
            const int c = c0 + dx, rr = r0 + dz;
            const int64_t u = (int64_t)T.u0 + c, v = (int64_t)T.v0 + rr;
            const int64_t cu = u + (int64_t)(T.i0 + ph) * kPeriod;
            const int64_t cv = v + (int64_t)(a.j0 + m) * kPeriod;
            keep = count >= a.min_size && (no_upper || count <= a.max_size) && c < kOutW &&
                   u < a.ubase && rr < T.out_h && cu < a.width_u && cv < a.height_v;
            if (keep) {
                cx = (int32_t)(a.transposed ? a.area_x0 + cv : a.area_x0 + cu);
                cz = (int32_t)(a.transposed ? a.area_z0 + cu : a.area_z0 + cv);
                if (a.rd_min_sq) {
                    const int64_t ddx = (int64_t)cx - a.center_x, ddz = (int64_t)cz - a.center_z;
                    keep = ddx * ddx + ddz * ddz >= a.rd_min_sq;
                }
            }
        }
        const unsigned mk = __ballot_sync(kFull, keep);
        if (mk) {
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(a.emitted, (unsigned long long)__popc(mk));
            base = __shfl_sync(kFull, base, 0);
            if (keep) {
                const unsigned long long idx = base + __popc(mk & ((1u << lane) - 1u));
                if (idx < a.cap) a.out[idx] = Hit{count, cx, cz};
            }
        }
        __syncwarp();
    }
}

// Processes the queue (all threads; block-uniform entry) and re-pushes pending groups. With
// `final` it repeats until queue and pending groups are empty; otherwise it may return with a
// partial queue (fewer than kQueueFlush groups) and no pending groups.
__device__ void drain_queue(BandSmem& S, const BandArgs& a, const Tile& T, int tid, int warp,
                            int lane, uint32_t (&pend)[kSlots], int (&pend_b)[kSlots], bool final) {
    for (;;) {
        flush_queue(S, a, T, warp, lane);
        __syncthreads();
        if (tid == 0) { S.qcount = 0; S.qover = 0; }
        __syncthreads();
        bool left = false;
#pragma unroll
        for (int k = 0; k < kSlots; ++k) {
            if (pend[k]) pend[k] = push_groups(S, warp + kWarps * k, lane, pend[k], pend_b[k]);
            left |= pend[k] != 0;
        }
        const bool more = __syncthreads_or(left);
        const int queued = S.qcount;  // stable: every push precedes the barrier above
        if (more) continue;
        if (queued == 0 || (!final && queued < kQueueFlush)) break;
    }
}

template <bool kMadAdd>
__global__ void __launch_bounds__(kTpb, 1) band_scan_kernel(const BandArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BandSmem& S = *reinterpret_cast<BandSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nb = a.nb, ncombo = 2 * nb;
    const uint32_t thr4 = (uint32_t)min(a.min_size, 128) * 0x01010101u;
    const uint32_t one = a.one;  // 1 at run time: keeps the band add on the multiply pipe
    uint32_t guard = 0;
    if (tid == 0) { S.qcount = 0; S.qover = 0; }

    for (int64_t tile = a.tile_begin + blockIdx.x; tile < a.tile_end; tile += gridDim.x) {
        Tile T;
        const int ut = (int)(tile % a.u_tiles);
        const int64_t rest = tile / a.u_tiles;
        const int vt = (int)(rest % a.v_tiles);
        T.i0 = 2 * (int)(rest / a.v_tiles);
        T.u0 = ut * kOutW;
        T.v0 = vt * a.band_h;
        // Tiles with no centre of the area in any of their combos are skipped (block-uniform).
        if ((int64_t)T.u0 + (int64_t)T.i0 * kPeriod >= a.width_u ||
            (int64_t)T.v0 + (int64_t)a.j0 * kPeriod >= a.height_v)
            continue;
        T.out_h = min(a.band_h, a.vbase - T.v0);
        const int batches = (T.out_h + 16 + 3) / 4;

        // Generator columns of this thread: words 2*warp and 2*warp+1, lane = bit.
        uint32_t lox[2], xh0[2], xh1[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int64_t idx0 = (int64_t)T.u0 + (warp * 2 + k) * 32 + lane + (int64_t)T.i0 * kPeriod;
            const uint64_t x0 = idx0 < a.ncols ? a.ct[idx0] : 0;
            const uint64_t x1 = idx0 + kPeriod < a.ncols ? a.ct[idx0 + kPeriod] : 0;
            lox[k] = (uint32_t)x0 & 0x1FFFFu;
            xh0[k] = (uint32_t)(x0 >> kPeriodBits);
            xh1[k] = (uint32_t)(x1 >> kPeriodBits);
        }
        // Counter slots of this warp: combo rows warp + 16*k; lane = word. Columns of the word
        // that exist for the slot's phase (bits beyond are masked to zero before counting).
        uint32_t cm[kSlots], fx[kSlots], re[kSlots], ro[kSlots], pend[kSlots];
        int pend_b[kSlots];
#pragma unroll
        for (int k = 0; k < kSlots; ++k) {
            const int combo = warp + kWarps * k;
            const int64_t first = (int64_t)T.u0 + lane * 32 + (int64_t)(T.i0 + (combo & 1)) * kPeriod;
            const int64_t nvalid = a.ncols - first;
            cm[k] = nvalid >= 32 ? ~0u : nvalid <= 0 ? 0u : (1u << nvalid) - 1u;
            fx[k] = ((combo ^ (combo >> 1)) & 1) ? 0u : ~0u;
            re[k] = ro[k] = 0;
            pend[k] = 0;
            pend_b[k] = 0;
        }
        for (int i = tid; i < 5 * kMaxCombos * kWords; i += kTpb) {
            (&S.hist_e[0][0][0])[i] = 0;
            (&S.hist_o[0][0][0])[i] = 0;
            (&S.hist_n[0][0][0])[i] = 0;
        }
        // Row terms of batches 0 and 1.
        for (int i = tid; i < 2 * 4 * (nb + 1); i += kTpb) {
            const int bb = i / (4 * (nb + 1)), q = (i / (nb + 1)) % 4, e = i % (nb + 1);
            const int vi = T.v0 + 4 * bb + q;
            S.rows[bb][q][e == 0 ? kMaxBands : e - 1] =
                vi < a.vrows ? a.rt[(int64_t)vi * a.rstride + (e == 0 ? 0 : a.j0 + e)] : 0u;
        }
        if (tid < 8) {
            const int bb = tid >> 2, q = tid & 3, vi = T.v0 + 4 * bb + q;
            const int64_t room = a.height_v + 16 - ((int64_t)vi + (int64_t)a.j0 * kPeriod);
            uint32_t mask = 0;
            if (vi < a.vrows)
                for (int m = 0; m < nb; ++m)
                    if (room - (int64_t)m * kPeriod > 0) mask |= 1u << m;
            S.rvalid[bb][q] = mask;
        }
        __syncthreads();

        for (int b = 0; b < batches; ++b) {
            const int rb = b % 3, buf = b & 1;
            // ---- generator: batch b into ring[buf] ------------------------------------------
#pragma unroll 1
            for (int q = 0; q < 4; ++q) {
                const uint32_t* zr = &S.rows[rb][q][0];
                const uint32_t zlo = zr[kMaxBands];
                const uint32_t zpar = (zr[0] ^ kXorHi) & 1u;
                uint32_t xa[2], xb[2], dd[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const Shared sh = shared_part(lox[k], zlo);
                    const uint32_t pi = (sh.q0 ^ xh0[k] ^ sh.carry ^ zpar) & 1u;
                    xa[k] = (pi ? xh1[k] : xh0[k]) + sh.carry;
                    xb[k] = (pi ? xh0[k] : xh1[k]) + sh.carry;
                    dd[k] = sh.d;
                    const uint32_t sw = __ballot_sync(kFull, pi != 0);
                    if (lane == 0) S.ring[buf][q][warp * 2 + k][kSwPlane] = sw;
                }
                uint32_t* dst0 = &S.ring[buf][q][warp * 2][0];
                uint32_t* dst1 = &S.ring[buf][q][warp * 2 + 1][0];
                auto hit = [&](uint32_t x, uint32_t z, uint32_t d) {
                    const uint32_t t = kMadAdd ? z * one + x : z + x;
                    return ((t ^ kXorHi) * kMulH + d) < kHitBelow;
                };
                int m = 0;
                for (; m + 3 < nb; m += 4) {
                    const uint4 z4 = *reinterpret_cast<const uint4*>(zr + m);  // m % 4 == 0: aligned
                    const uint32_t z0 = z4.x, z1 = z4.y, z2 = z4.z, z3 = z4.w;
                    const uint32_t a0 = __ballot_sync(kFull, hit(xa[0], z0, dd[0]));
                    const uint32_t a1 = __ballot_sync(kFull, hit(xa[1], z0, dd[1]));
                    const uint32_t b0 = __ballot_sync(kFull, hit(xb[0], z1, dd[0]));
                    const uint32_t b1 = __ballot_sync(kFull, hit(xb[1], z1, dd[1]));
                    const uint32_t c0 = __ballot_sync(kFull, hit(xa[0], z2, dd[0]));
                    const uint32_t c1 = __ballot_sync(kFull, hit(xa[1], z2, dd[1]));
                    const uint32_t e0 = __ballot_sync(kFull, hit(xb[0], z3, dd[0]));
                    const uint32_t e1 = __ballot_sync(kFull, hit(xb[1], z3, dd[1]));
                    if (lane == 0) {
                        *reinterpret_cast<uint4*>(dst0 + m) = make_uint4(a0, b0, c0, e0);
                        *reinterpret_cast<uint4*>(dst1 + m) = make_uint4(a1, b1, c1, e1);
                    }
                }
                for (; m < nb; ++m) {
                    const uint32_t z0 = zr[m];
                    const uint32_t w0 = __ballot_sync(kFull, hit((m & 1) ? xb[0] : xa[0], z0, dd[0]));
                    const uint32_t w1 = __ballot_sync(kFull, hit((m & 1) ? xb[1] : xa[1], z0, dd[1]));
                    if (lane == 0) {
                        dst0[m] = w0;
                        dst1[m] = w1;
                    }
                }
            }
            __syncthreads();

            // ---- survivor queue: flush when half full; groups that did not fit are re-pushed ---
            if (S.qcount >= kQueueFlush || S.qover)
                drain_queue(S, a, T, tid, warp, lane, pend, pend_b, false);
            // Row terms of batch b + 2 (read by the generator after the next barrier).
            {
                const int bb = (b + 2) % 3;
                for (int i = tid; i < 4 * (nb + 1); i += kTpb) {
                    const int q = i / (nb + 1), e = i % (nb + 1);
                    const int vi = T.v0 + 4 * (b + 2) + q;
                    S.rows[bb][q][e == 0 ? kMaxBands : e - 1] =
                        vi < a.vrows ? a.rt[(int64_t)vi * a.rstride + (e == 0 ? 0 : a.j0 + e)] : 0u;
                }
                if (tid < 4) {
                    const int vi = T.v0 + 4 * (b + 2) + tid;
                    const int64_t room = a.height_v + 16 - ((int64_t)vi + (int64_t)a.j0 * kPeriod);
                    uint32_t mask = 0;
                    if (vi < a.vrows)
                        for (int m = 0; m < nb; ++m)
                            if (room - (int64_t)m * kPeriod > 0) mask |= 1u << m;
                    S.rvalid[bb][tid] = mask;
                }
            }

            // ---- counter: batch b from ring[buf] ----------------------------------------------
            const int hs = b % 5;
#pragma unroll
            for (int k = 0; k < kSlots; ++k) {
                const int combo = warp + kWarps * k;
                if (combo >= ncombo) break;  // warp-uniform
                const int m = combo >> 1;
                uint32_t n[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const uint32_t* rec = &S.ring[buf][q][lane][0];
                    const uint32_t keep = ((S.rvalid[rb][q] >> m) & 1u) ? cm[k] : 0u;
                    n[q] = nibble_counts(rec[m] & (rec[kSwPlane] ^ fx[k]) & keep);
                }
                const uint32_t n01 = n[0] + n[1], n23 = n[2] + n[3];
                const uint32_t e = (n01 & 0x0F0F0F0Fu) + (n23 & 0x0F0F0F0Fu);
                const uint32_t o = ((n01 >> 4) & 0x0F0F0F0Fu) + ((n23 >> 4) & 0x0F0F0F0Fu);
                uint32_t en = __shfl_down_sync(kFull, e, 1), on = __shfl_down_sync(kFull, o, 1);
                if (lane == kWords - 1) en = on = 0;
                const uint32_t s = e + o, sn = en + on;
                const uint32_t s1 = __funnelshift_r(s, sn, 8);
                const uint32_t ge = s + s1 + __funnelshift_r(e, en, 16);
                const uint32_t go = o + s1 + __funnelshift_r(s, sn, 16);
                guard |= (ge + 0x4C4C4C4Cu) | (go + 0x4C4C4C4Cu);
                re[k] += ge - S.hist_e[hs][combo][lane];
                ro[k] += go - S.hist_o[hs][combo][lane];
                S.hist_e[hs][combo][lane] = ge;
                S.hist_o[hs][combo][lane] = go;
                // hist_n[hs] held batch b-5; batch b-4 is in slot (b+1)%5.
                const uint32_t top01 = S.hist_n[(b + 1) % 5][combo][lane];
                S.hist_n[hs][combo][lane] = n01;
                uint32_t flag = 0;
                if (b >= 4) {
                    const uint32_t te = bytes_at_least(re[k], thr4), to = bytes_at_least(ro[k], thr4);
                    flag = te | (to >> 1);  // even groups at bits 8k+7, odd at 8k+6
                    if (lane == kWords - 1) flag &= 0x0000C0C0u;  // groups 4..7: centres >= 1,008
                }
                // Second test of flagged groups: drop the 8 outer cells of rows 0, 1 (batch b-4)
                // and rows 18, 19 (batch b), which no window of the group reaches.
                const uint32_t top01n = __shfl_down_sync(kFull, top01, 1);
                const uint32_t n23n = __shfl_down_sync(kFull, n23, 1);
                if (flag) {
                    const uint64_t t01 = ((uint64_t)(lane == kWords - 1 ? 0u : top01n) << 32) | top01;
                    const uint64_t b23 = ((uint64_t)(lane == kWords - 1 ? 0u : n23n) << 32) | n23;
                    uint32_t gm = 0;
#pragma unroll
                    for (int g = 0; g < 8; ++g) {
                        const int bit = (g & 1) ? 8 * (g >> 1) + 6 : 8 * (g >> 1) + 7;
                        if (!((flag >> bit) & 1u)) continue;
                        const uint32_t box = (((g & 1) ? ro[k] : re[k]) >> (8 * (g >> 1))) & 0xFFu;
                        const uint32_t outer = (uint32_t)((t01 >> (4 * g)) & 0xF) + (uint32_t)((t01 >> (4 * g + 16)) & 0xF) +
                                               (uint32_t)((b23 >> (4 * g)) & 0xF) + (uint32_t)((b23 >> (4 * g + 16)) & 0xF);
                        // A box byte of 128+ is a conservative report: keep the group.
                        if (box >= 128u || box - outer >= (uint32_t)a.min_size) gm |= 1u << g;
                    }
                    pend[k] = push_groups(S, combo, lane, gm, b);
                    pend_b[k] = b;
                }
            }
        }
        __syncthreads();
        drain_queue(S, a, T, tid, warp, lane, pend, pend_b, true);
    }
    // A 4-row strip with 52+ hits among its 80 cells could carry a box past a byte lane.
    if (guard & 0x80808080u) atomicOr(a.overflow, 1u);
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
    cudaError_t e = cudaFuncSetAttribute(band_scan_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(BandSmem));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(band_scan_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(BandSmem));
}

cudaError_t launch_band_scan(const BandArgs& a, int grid, cudaStream_t s) {
    if (a.mad_add)
        band_scan_kernel<true><<<grid, kTpb, sizeof(BandSmem), s>>>(a);
    else
        band_scan_kernel<false><<<grid, kTpb, sizeof(BandSmem), s>>>(a);
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
