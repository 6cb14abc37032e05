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
//  * Rows advance in batches of 8 (two 4-row strips). Ballots of batch b go to ring slot b % 4,
//    so one barrier per batch separates the generator (batch b+1) from the counter (batch b),
//    which reads batches b-2..b. Row terms arrive by TMA bulk copies two batches ahead.
//  * Counting is SWAR in byte lanes on 4x4 centre groups. A warp owns a combo (phase, band) row
//    with one lane per 32-column word: nibble popcounts of the 4 rows give 4x4 block counts,
//    the neighbour word comes by shuffle, three funnel shifts and two adds give the 20-column
//    strip sums of the word's 8 groups, and a rolling sum over 5 strips gives the 20x20 box of
//    each group, which bounds its 16 windows. A flagged group is re-tested in byte lanes with
//    the 32 cells of rows 0, 1, 18 and 19 that lie outside every window removed (368 cells).
//  * The warp then counts the 16 windows of each surviving group exactly from the ring (the
//    group's 20 rows are still there) and appends the centres in range to the hit list.
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
// Band modes. Shared LCG: two X phases x up to 32 Z bands 2^17 apart, all sharing the low 17 bits
// of the row term. Independent bands: one X phase x up to 32 bands at any row spacing. Grouped
// bands: two X phases x up to 16 bands, in G groups at their own base rows, each group holding P
// copies 2^17 apart that share its low bits (band m = copy * G + group); the swap ballot of group
// g is plane kGrpSw + g.
constexpr int kModeShared = 0, kModeIndep = 1, kModeGrouped = 2;
constexpr int kGrpBands = 16;
constexpr int kGrpSw = kGrpBands;
constexpr int kPlanes = kMaxBands + 1;      // band planes and the swap plane
constexpr int kMaxCombos = 2 * kMaxBands;
constexpr int kSlots = kMaxCombos / kWarps; // combo rows counted per warp
constexpr unsigned kFull = 0xFFFFFFFFu;

// Row-term record of one base row for one group of up to 32 bands (matches the global table
// written by row_terms_kernel, so a batch of 8 rows is one contiguous 1,152-byte bulk copy).
constexpr int kRowWords = 36;
constexpr int kRowLo = 32;      // low 17 bits of the row term (shared by all bands)
constexpr int kRowValid = 33;   // bands of the group that hold this row (prefix count)

// Independent-band record (general mode: bands at any row spacing, no shared low bits):
// [m] high part and [32 + m] low 17 bits of the row term in band m, [64] bands holding the row.
constexpr int kRowWordsI = 72;
constexpr int kRowLoI = 32;
constexpr int kRowValidI = 64;
template <int kMode>
constexpr int row_words() { return kMode == kModeShared ? kRowWords : kRowWordsI; }

constexpr int kBatchRows = 8;               // rows per barrier: two 4-row strips
// Generator layout: each lane evaluates bit `lane` of kGenW consecutive words (kGenW x 32 columns
// per warp); kGenColWarps warps span the 32 words and each generates kGenRows rows of a batch.
// Eight words per lane measured 4% faster on the full-world scan than four (fewer per-row setup
// instructions per generated word), with identical output.
#ifndef SLIME_GEN_WORDS
#define SLIME_GEN_WORDS 8
#endif
constexpr int kGenW = SLIME_GEN_WORDS;
constexpr int kGenColWarps = 32 / kGenW;
constexpr int kGenRows = kBatchRows / (16 / kGenColWarps);
static_assert(kGenW % 4 == 0 && kGenRows >= 1, "generator layout");
constexpr int kCandCap = 64;                // per warp: groups waiting for their union count
constexpr int kRingSlots = 4;               // batches b-2..b are read while b+1 is generated

struct __align__(16) BandSmem {
    uint32_t ring[kRingSlots][kBatchRows][kPlanes][kWords];  // [batch % 4][row][band planes | swap][word]
    uint32_t hist_e[5][kMaxCombos][kWords];   // strip sums of the last 5 strips (even groups)
    uint32_t hist_o[5][kMaxCombos][kWords];   // (odd groups)
    uint32_t rows[3][kBatchRows * kRowWordsI];  // row terms of 3 batches, filled by bulk copies
    unsigned long long rows_bar[3];           // mbarriers of the three row-term buffers
    uint32_t cand[kWarps][kCandCap];          // per warp: combo << 24 | word << 19 | group << 16 | strip
    BandArgs args;                            // batched kernel: the current tile's search
    long long next_tile;                      // batched kernel: tile taken from the queue
    int search;                               // batched kernel: its search
    int failed;  // a bounded wait gave up: the CTA stops
    // Grouped bands, per band m: first area row (before the base row), swap plane, and all ones
    // when its copy index is odd (the phase choice flips with each copy).
    int32_t goff[kGrpBands];
    int32_t gsw[kGrpBands];
    uint32_t gflip[kGrpBands];
    unsigned int hist[kHistBins];             // counts of this CTA's centres in range (if args.hist)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Bulk copy (TMA engine, no multicast) of `bytes` from global memory into shared memory,
// completing on an mbarrier. Addresses and size are multiples of 16 bytes.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          unsigned long long* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// Waits for the mbarrier phase with the given parity; gives up after `polls` polls and returns
// false (the caller flags an error instead of hanging the GPU).
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, uint32_t parity, uint32_t polls) {
    for (uint32_t i = 0; i < polls; ++i) {
        uint32_t done;
        asm volatile("{ .reg .pred p;\n"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     "selp.u32 %0, 1, 0, p; }"
                     : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Per nibble: the number of set bits (0..4); shifts as multiply-highs.
__device__ __forceinline__ uint32_t nibble_counts(uint32_t r) {
    const uint32_t a = r - (__umulhi(r, 1u << 31) & 0x55555555u);
    return (a & 0x33333333u) + (__umulhi(a, 1u << 30) & 0x33333333u);
}

// Per byte: high bit set where v >= t (v, t < 256; borrow-free because v | 0x80 >= 128 >= t').
// Bytes >= 128 always report (a superset is safe: flagged groups are re-tested).
__device__ __forceinline__ uint32_t bytes_at_least(uint32_t v, uint32_t t4) {
    return (((v | 0x80808080u) - t4) | v) & 0x80808080u;
}

struct Tile {
    int u0, v0, i0, out_h;
};

// The kGenW words of one plane at dst (16-byte aligned), as uint4 stores.
__device__ __forceinline__ void store_plane(uint4* dst, const uint32_t (&w)[kGenW]) {
#pragma unroll
    for (int i = 0; i < kGenW / 4; ++i) dst[i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
}
__device__ __forceinline__ void clear_plane(uint4* dst) {
#pragma unroll
    for (int i = 0; i < kGenW / 4; ++i) dst[i] = make_uint4(0u, 0u, 0u, 0u);
}

// Columns of word `word` that exist for phase `ph` of the tile (all ones inside the area).
__device__ __forceinline__ uint32_t column_mask(const BandArgs& a, const Tile& T, int word, int ph) {
    const int64_t first = (int64_t)T.u0 + word * 32 + (int64_t)(T.i0 + ph) * kPeriod;
    const int64_t nvalid = a.ncols - first;
    return nvalid >= 32 ? ~0u : nvalid <= 0 ? 0u : (1u << nvalid) - 1u;
}

// A combo is one (X phase, band) pair: combo = 2 m + phase with the shared LCG, combo = m for
// independent bands (one phase).
template <int kMode>
__device__ __forceinline__ int combo_band(int combo) { return kMode == kModeIndep ? combo : combo >> 1; }
template <int kMode>
__device__ __forceinline__ int combo_phase(int combo) { return kMode == kModeIndep ? 0 : combo & 1; }

// Bits of a combo in ring row `r` (tile-relative input row), word `word`.
template <int kMode>
__device__ __forceinline__ uint32_t combo_word(const BandSmem& S, int r, int combo, uint32_t fx, int word) {
    const int slot = (r >> 3) & (kRingSlots - 1), q = r & 7;
    if (kMode == kModeIndep) return S.ring[slot][q][combo][word];
    const int m = combo >> 1;
    if (kMode == kModeGrouped) return S.ring[slot][q][m][word] & (S.ring[slot][q][S.gsw[m]][word] ^ fx ^ S.gflip[m]);
    return S.ring[slot][q][m][word] & (S.ring[slot][q][kSwPlane][word] ^ fx);
}

// First area row (band axis) of band m, before the tile's base row is added.
template <int kMode>
__device__ __forceinline__ int64_t band_row0(const BandSmem& S, const BandArgs& a, int m) {
    return kMode == kModeGrouped ? (int64_t)S.goff[m] : (int64_t)(a.j0 + m) * a.row_stride;
}

// Row `r` (0..19) of the union of the 16 windows of a 4x4 centre group, as a 20-bit column mask:
// columns 8 - h .. 11 + h with h the widest window row that reaches box row r.
__host__ __device__ constexpr uint32_t group_union_mask(int r) {
    int h = 0;
    for (int dz = 0; dz < 4; ++dz)
        if (r - dz >= 0 && r - dz <= 16 && window_half_width(r - dz) > h) h = window_half_width(r - dz);
    return ((1u << (2 * h + 4)) - 1u) << (8 - h);
}

// Row `r` (0..19) of the union of the 4 windows of the 2x2 sub-group (sx, sy) of a 4x4 group
// (centres dx = 2sx, 2sx+1 and dz = 2sy, 2sy+1), as a 20-bit column mask; 0 outside its rows.
__host__ __device__ constexpr uint32_t subgroup_union_mask(int r, int sx, int sy) {
    int h = -1;
    for (int dz = 2 * sy; dz < 2 * sy + 2; ++dz)
        if (r - dz >= 0 && r - dz <= 16 && window_half_width(r - dz) > h) h = window_half_width(r - dz);
    return h < 0 ? 0u : ((1u << (2 * h + 2)) - 1u) << (2 * sx + 8 - h);
}
constexpr int kSubgroupThreshold = 52;  // at or below: also test the four 2x2 sub-group unions

// Exact window counts of the 16 centres of group g of word `word` for one combo, from the 20
// ring rows of strips st-4..st. Lanes 0..19 fetch one 20-column row slice each. First the whole
// union of the 16 windows (332 cells; `umask` = this lane's row of it) is counted with one
// reduction: below the threshold no window can reach it. Otherwise each lane counts half a window
// of one centre over shuffled slices. Centres in range are appended to the hit list.
// Warp-uniform arguments; called by the whole warp.
template <bool kMasked, int kMode>
__device__ __forceinline__ void exact_group(BandSmem& S, const BandArgs& a, const Tile& T, int combo,
                                         uint32_t fx, int word, int g, int st, int lane, uint32_t umask) {
    const int ph = combo_phase<kMode>(combo), m = combo_band<kMode>(combo);
    const int c0 = word * 32 + 4 * g;       // first window column (tile-relative input col)
    const int r0 = 4 * (st - 4);            // first window row (tile-relative input row)
    uint32_t slice = 0;
    if (lane < 20) {
        uint32_t lo = combo_word<kMode>(S, r0 + lane, combo, fx, word);
        uint32_t hi = word + 1 < kWords ? combo_word<kMode>(S, r0 + lane, combo, fx, word + 1) : 0u;
        if (kMasked) {
            lo &= column_mask(a, T, word, ph);
            hi &= word + 1 < kWords ? column_mask(a, T, word + 1, ph) : 0u;
        }
        slice = __funnelshift_r(lo, hi, 4 * g) & 0xFFFFFu;
    }
    if ((int)__reduce_add_sync(kFull, (unsigned)__popc(slice & umask)) < a.min_size) return;
    // Lane l counts window rows 0..8 (l < 16) or 9..16 (l >= 16) of centre l % 16; the halves
    // are then added across the two half-warps.
    const int dx = lane & 3, dz = (lane >> 2) & 3, half = lane >> 4;
    int count = 0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const uint32_t row = __shfl_sync(kFull, slice, dz + 9 * half + k);
        const uint32_t mask = half ? (k < 8 ? window_row_mask(9 + k) : 0u) : window_row_mask(k);
        count += __popc((row >> dx) & mask);
    }
    count += __shfl_xor_sync(kFull, count, 16);
    bool keep = false;
    int cx = 0, cz = 0;
    if (lane < 16) {
        const int c = c0 + dx, rr = r0 + dz;
        const int64_t u = (int64_t)T.u0 + c, v = (int64_t)T.v0 + rr;
        const int64_t cu = u + (int64_t)(T.i0 + ph) * kPeriod;
        const int64_t cv = v + band_row0<kMode>(S, a, m);
        keep = count >= a.min_size && count <= a.max_size && c < kOutW && u < a.ubase &&
               rr < T.out_h && cu < a.width_u && cv < a.height_v;
        if (keep) {
            cx = (int32_t)(a.transposed ? a.area_x0 + cv : a.area_x0 + cu);
            cz = (int32_t)(a.transposed ? a.area_z0 + cu : a.area_z0 + cv);
            if (a.rd_min_sq) {
                const int64_t ddx = (int64_t)cx - a.center_x, ddz = (int64_t)cz - a.center_z;
                keep = ddx * ddx + ddz * ddz >= a.rd_min_sq;
            }
        }
        // Every centre in range is counted; only those at or above the emission gate are sent.
        if (keep && a.hist) atomicAdd(&S.hist[count], 1u);
        keep = keep && count >= a.emit_min;
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
}

// Per-thread counter state: one entry per combo slot of the warp (lane = word). The combo of
// slot k is warp + 16 k, so all four slots of a warp share one phase and one swap sense.
struct Counter {
    uint32_t cm[kSlots];              // columns of the word that exist for the slot's phase
    uint32_t re[kSlots], ro[kSlots];  // rolling 20x20 boxes (even / odd groups, byte lanes)
};

// Second test of the flagged groups of one combo, all 8 groups at once in byte lanes: the 8
// outer cells of rows 0, 1 (strip st - 4) and of rows 18, 19 (strip st), which no window of the
// group reaches, are removed from the box (368 cells remain; the box bytes are exact, so no byte
// borrows). Survivors are counted exactly. Called by the whole warp.
// The union counts of the warp's candidate groups, 32 at a time (lane = group), then the exact
// counts of those that reach the threshold. Called by the whole warp; the caller empties the list.
template <bool kMasked, int kMode>
__device__ __forceinline__ void flush_cands(BandSmem& S, const BandArgs& a, const Tile& T, uint32_t fx, int warp,
                                         int lane, uint32_t umask, int ncand) {
    __syncwarp();
    for (int base = 0; base < ncand; base += 32) {
        const int j = base + lane;
        uint32_t e = 0;
        bool pass = false;
        if (j < ncand) {
            e = S.cand[warp][j];
            const int combo = (int)(e >> 24), word = (int)((e >> 19) & 31), g = (int)((e >> 16) & 7);
            const int r0 = 4 * ((int)(e & 0xFFFF) - 4);
            uint32_t cml = ~0u, cmh = word + 1 < kWords ? ~0u : 0u;
            if (kMasked) {
                cml = column_mask(a, T, word, combo_phase<kMode>(combo));
                cmh &= word + 1 < kWords ? column_mask(a, T, word + 1, combo_phase<kMode>(combo)) : 0u;
            }
            const int wh = min(word + 1, kWords - 1);
            if (a.min_size > kSubgroupThreshold) {
                int sum = 0;
#pragma unroll
                for (int r = 0; r < 20; ++r) {
                    const uint32_t lo = combo_word<kMode>(S, r0 + r, combo, fx, word) & cml;
                    const uint32_t hi = combo_word<kMode>(S, r0 + r, combo, fx, wh) & cmh;
                    sum += __popc(__funnelshift_r(lo, hi, 4 * g) & group_union_mask(r));
                }
                pass = sum >= a.min_size;
            } else {
                int sum = 0, s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
                for (int r = 0; r < 20; ++r) {
                    const uint32_t lo = combo_word<kMode>(S, r0 + r, combo, fx, word) & cml;
                    const uint32_t hi = combo_word<kMode>(S, r0 + r, combo, fx, wh) & cmh;
                    const uint32_t x = __funnelshift_r(lo, hi, 4 * g);
                    sum += __popc(x & group_union_mask(r));
                    s0 += __popc(x & subgroup_union_mask(r, 0, 0));
                    s1 += __popc(x & subgroup_union_mask(r, 1, 0));
                    s2 += __popc(x & subgroup_union_mask(r, 0, 1));
                    s3 += __popc(x & subgroup_union_mask(r, 1, 1));
                }
                pass = sum >= a.min_size && max(max(s0, s1), max(s2, s3)) >= a.min_size;
            }
        }
        for (unsigned pm = __ballot_sync(kFull, pass); pm; pm &= pm - 1) {
            const uint32_t ee = __shfl_sync(kFull, e, __ffs(pm) - 1);
            exact_group<kMasked, kMode>(S, a, T, (int)(ee >> 24), fx, (int)((ee >> 19) & 31), (int)((ee >> 16) & 7),
                                         (int)(ee & 0xFFFF), lane, umask);
        }
    }
    __syncwarp();
}

template <bool kMasked, int kMode, bool kCands>
__device__ __forceinline__ void second_test(BandSmem& S, const BandArgs& a, const Tile& T, uint32_t flag,
                                            uint32_t re, uint32_t ro, uint32_t n23, uint32_t cm, uint32_t fx,
                                            uint32_t thr4, int combo, int lane, int st, uint32_t umask, int warp,
                                            int& ncand) {
    const int r0 = 4 * (st - 4);  // rows 0 and 1 of strip st - 4
    uint32_t w0 = combo_word<kMode>(S, r0, combo, fx, lane), w1 = combo_word<kMode>(S, r0 + 1, combo, fx, lane);
    if (kMasked) { w0 &= cm; w1 &= cm; }
    const uint32_t top01 = nibble_counts(w0) + nibble_counts(w1);
    // Outer cells of group g: 4-column blocks g and g + 4 of those four rows (byte lanes as in
    // the boxes: even groups from even blocks, odd groups from odd blocks).
    const uint32_t E = (top01 & 0x0F0F0F0Fu) + (n23 & 0x0F0F0F0Fu);
    const uint32_t O = ((top01 >> 4) & 0x0F0F0F0Fu) + ((n23 >> 4) & 0x0F0F0F0Fu);
    // Lane 31 reads its own words here; only its groups 0..3 (which use no neighbour) can flag.
    const uint32_t En = __shfl_down_sync(kFull, E, 1), On = __shfl_down_sync(kFull, O, 1);
    const uint32_t oe = E + __funnelshift_r(E, En, 16), oo = O + __funnelshift_r(O, On, 16);
    const uint32_t f2 = (bytes_at_least(re - oe, thr4) | (bytes_at_least(ro - oo, thr4) >> 1)) & flag;
    uint32_t gm = 0;  // bit 8j+7 -> group 2j, bit 8j+6 -> group 2j+1
    for (uint32_t f = f2; f; f &= f - 1) {
        const int bit = __ffs(f) - 1;
        gm |= 1u << (2 * (bit >> 3) + 7 - (bit & 7));
    }
    if (!kCands) {  // few survivors (high thresholds): count each group at once
        for (unsigned todo = __ballot_sync(kFull, gm != 0); todo; todo &= todo - 1) {
            const int word = __ffs(todo) - 1;
            for (uint32_t gw = __shfl_sync(kFull, gm, word); gw; gw &= gw - 1)
                exact_group<kMasked, kMode>(S, a, T, combo, fx, word, __ffs(gw) - 1, st, lane, umask);
        }
        return;
    }
    // Survivors join the warp's candidate list (lane order, groups ascending); the list is
    // counted at the end of the batch, or now when it would overflow.
    const int n = __popc(gm);
    int pos = n;  // inclusive prefix sum over lanes
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int v = __shfl_up_sync(kFull, pos, d);
        if (lane >= d) pos += v;
    }
    const int total = __shfl_sync(kFull, pos, 31);
    if (total == 0) return;
    // Survivor i of this combo (lane order) goes to list slot ncand + i - placed; a full list is
    // counted (one call site) and refilled until every survivor is placed.
    for (int placed = 0;;) {
        const int room = kCandCap - ncand;
        int idx = pos - n;
        for (uint32_t gw = gm; gw; gw &= gw - 1, ++idx)
            if (idx >= placed && idx < placed + room)
                S.cand[warp][ncand + idx - placed] = ((uint32_t)combo << 24) | ((uint32_t)lane << 19) |
                                                     ((uint32_t)(__ffs(gw) - 1) << 16) | (uint32_t)st;
        const int took = min(room, total - placed);
        ncand += took;
        placed += took;
        if (placed == total) break;
        flush_cands<kMasked, kMode>(S, a, T, fx, warp, lane, umask, ncand);
        ncand = 0;
    }
    __syncwarp();
}

// Counts one 4-row strip (rows 4t..4t+3 of ring slot `slot`) for the warp's four combo slots as
// one straight-line block: 4x4 block counts, 20-column strip sums, rolling 20x20 boxes and the
// threshold test. Only when a lane flags a group does the warp take the second test. With the
// shared LCG, slots of combos beyond the launch's band count read zero planes and never flag;
// independent bands use two slots per warp (32 combos) and skip combos beyond the band count.
template <bool kMasked, int kMode, bool kCands>
__device__ __forceinline__ void count_strip(BandSmem& S, const BandArgs& a, const Tile& T, Counter& C,
                                            int slot, int t, int st, int warp, int lane, uint32_t fx,
                                            uint32_t lastmask, uint32_t thr4, uint32_t umask, uint32_t& guard,
                                            int& ncand) {
    const int r0 = 4 * t;  // t is a compile-time constant after unrolling
    const int hs = st % 5;
    const uint32_t live = st >= 4 ? lastmask : 0u;  // boxes are complete from the fifth strip on
    constexpr int kUsed = kMode == kModeShared ? kSlots : kMaxBands / kWarps;
    uint32_t sel[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) sel[q] = kMode == kModeShared ? S.ring[slot][r0 + q][kSwPlane][lane] ^ fx : ~0u;
    uint32_t fl[kSlots] = {}, n23s[kSlots] = {};
    uint32_t any = 0;
#pragma unroll
    for (int k = 0; k < kUsed; ++k) {
        const int combo = warp + kWarps * k;
        const int m = combo_band<kMode>(combo);
        if (kMode != kModeShared && m >= a.nb) continue;  // warp-uniform
        uint32_t n[4];
        // Grouped bands: the slot's own swap plane and phase sense.
        const int gs = kMode == kModeGrouped ? S.gsw[m] : 0;
        const uint32_t gfx = kMode == kModeGrouped ? fx ^ S.gflip[m] : 0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t w = S.ring[slot][r0 + q][m][lane] &
                         (kMode == kModeGrouped ? S.ring[slot][r0 + q][gs][lane] ^ gfx : sel[q]);
            if (kMasked) w &= C.cm[k];
            n[q] = nibble_counts(w);
        }
        const uint32_t n01 = n[0] + n[1], n23 = n[2] + n[3];
        const uint32_t e = (n01 & 0x0F0F0F0Fu) + (n23 & 0x0F0F0F0Fu);
        const uint32_t o = ((n01 >> 4) & 0x0F0F0F0Fu) + ((n23 >> 4) & 0x0F0F0F0Fu);
        // Lane 31 gets its own words back: they feed only groups 4..7, which it never flags.
        const uint32_t en = __shfl_down_sync(kFull, e, 1), on = __shfl_down_sync(kFull, o, 1);
        const uint32_t s = e + o, sn = en + on;
        const uint32_t s1 = __funnelshift_r(s, sn, 8);
        const uint32_t ge = s + s1 + __funnelshift_r(e, en, 16);
        const uint32_t go = o + s1 + __funnelshift_r(s, sn, 16);
        guard |= (ge + 0x4C4C4C4Cu) | (go + 0x4C4C4C4Cu);
        uint32_t* he = &S.hist_e[hs][combo][lane];
        uint32_t* ho = &S.hist_o[hs][combo][lane];
        C.re[k] += ge - *he;
        C.ro[k] += go - *ho;
        *he = ge;
        *ho = go;
        const uint32_t te = bytes_at_least(C.re[k], thr4), to = bytes_at_least(C.ro[k], thr4);
        fl[k] = (te | (to >> 1)) & live;  // even groups at bits 8j+7, odd groups at 8j+6
        n23s[k] = n23;
        any |= fl[k];
    }
    if (__any_sync(kFull, any != 0)) {
#pragma unroll
        for (int k = 0; k < kUsed; ++k)
            if (__any_sync(kFull, fl[k] != 0))
                second_test<kMasked, kMode, kCands>(S, a, T, fl[k], C.re[k], C.ro[k], n23s[k], kMasked ? C.cm[k] : ~0u,
                                             fx, thr4, warp + kWarps * k, lane, st, umask, warp, ncand);
    }
}

// ---- exact counts of every centre, bit-sliced (low thresholds) ------------------------------
//
// Below a few units above the mean window count (22.1) most 4x4 groups pass every bound, and
// counting each survivor with popcounts costs more than counting every centre exactly. This mode
// does the latter with bit-sliced adders: a 32-bit word holds one bit of the counts of 32
// consecutive centres (bit j = centre j of the lane's word), so a full adder over three words
// (two LOP3) adds 32 centres' bits at once.
//
// For window rows i = 0..16 with half-widths h_i = 2,4,5,6,7,7,8,8,8,8,8,7,7,6,5,4,2, the cells at
// horizontal offset k = |dx| from the centre column lie in the rows with h_i >= k, a contiguous
// run of 17 (k <= 2), 15 (k = 3, 4), 13 (5), 11 (6), 9 (7) or 5 (8) rows. So the window count is
//     sum over dx = -8..8 of V_{L(|dx|)}(column x + dx),
// with V_L the vertical sum of the run of L rows, per column. The six V_L of a word's 32 columns are
// built nested (V5 -> V9 -> ... -> V17, 43 LOP3), the next word's come by shuffle, and 17
// funnel-shifted copies are added in a tree of ripple adders into 8 planes.

__device__ __forceinline__ void bs_fa(uint32_t a, uint32_t b, uint32_t c, uint32_t& s, uint32_t& cy) {
    s = a ^ b ^ c;
    cy = (a & b) | (c & (a | b));
}

// out = a + b over NO planes (a: NA planes, b: NB <= NA planes; the caller knows the sum fits).
template <int NA, int NB, int NO>
__device__ __forceinline__ void bs_add(const uint32_t (&a)[NA], const uint32_t (&b)[NB], uint32_t (&out)[NO]) {
    static_assert(NB <= NA && NO >= NA && NO <= NA + 1, "plane counts");
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < NA; ++i) {
        if (i == 0) {
            out[0] = a[0] ^ b[0];
            c = a[0] & b[0];
        } else if (i < NB) {
            bs_fa(a[i], b[i], c, out[i], c);
        } else {
            out[i] = a[i] ^ c;
            c = a[i] & c;
        }
    }
    if constexpr (NO > NA) out[NA] = c;
}

// Copy of the N planes of v shifted right by dx within the 64-bit pair (own word, next word).
template <int N>
__device__ __forceinline__ void bs_shift(const uint32_t (&v)[N], const uint32_t (&vn)[N], int dx, uint32_t (&out)[N]) {
#pragma unroll
    for (int i = 0; i < N; ++i) out[i] = __funnelshift_r(v[i], vn[i], dx);
}

// Sum of the shifted copies at dx and 16 - dx of one vertical level.
template <int N>
__device__ __forceinline__ void bs_pair(const uint32_t (&v)[N], const uint32_t (&vn)[N], int dx, uint32_t (&out)[N + 1]) {
    uint32_t a[N], b[N];
    bs_shift<N>(v, vn, dx, a);
    bs_shift<N>(v, vn, 16 - dx, b);
    bs_add<N, N, N + 1>(a, b, out);
}

template <int N>
__device__ __forceinline__ void bs_next(const uint32_t (&v)[N], uint32_t (&vn)[N]) {
#pragma unroll
    for (int i = 0; i < N; ++i) vn[i] = __shfl_down_sync(kFull, v[i], 1);
}

// Exact window counts (8 planes) of the 32 centres of the lane's word whose windows start at
// row DZ of the 20 rows in R (window rows R[DZ] .. R[DZ + 16]).
template <int DZ>
__device__ __forceinline__ void bs_window_counts(const uint32_t (&Rr)[20], uint32_t (&cnt)[8]) {
    const uint32_t* R = Rr + DZ;
    // Vertical runs, nested: V5 = rows 6..10, V9 = 4..12, V11 = 3..13, V13 = 2..14, V15 = 1..15,
    // V17 = 0..16.
    uint32_t v5[3], v9[4], v11[4], v13[4], v15[4], v17[5];
    {
        uint32_t s1, c1, c2;
        bs_fa(R[6], R[7], R[8], s1, c1);
        bs_fa(R[9], R[10], s1, v5[0], c2);
        v5[1] = c1 ^ c2;
        v5[2] = c1 & c2;
    }
    {
        uint32_t s, c, cc, c4;
        bs_fa(R[4], R[5], R[11], s, c);
        bs_fa(R[12], s, v5[0], v9[0], cc);
        bs_fa(c, cc, v5[1], v9[1], c4);
        v9[2] = c4 ^ v5[2];
        v9[3] = c4 & v5[2];
    }
    auto add2 = [](const uint32_t (&v)[4], uint32_t x, uint32_t y, uint32_t (&o)[4]) {
        uint32_t c;
        bs_fa(x, y, v[0], o[0], c);
        o[1] = v[1] ^ c; c &= v[1];
        o[2] = v[2] ^ c; c &= v[2];
        o[3] = v[3] ^ c;  // the sum stays below 16
    };
    add2(v9, R[3], R[13], v11);
    add2(v11, R[2], R[14], v13);
    add2(v13, R[1], R[15], v15);
    {
        uint32_t c;
        bs_fa(R[0], R[16], v15[0], v17[0], c);
        v17[1] = v15[1] ^ c; c &= v15[1];
        v17[2] = v15[2] ^ c; c &= v15[2];
        v17[3] = v15[3] ^ c; c &= v15[3];
        v17[4] = c;
    }
    // The next word's levels (lane 31 gets its own back: only its centres 16+ would use them,
    // and those lie beyond the tile's output columns).
    uint32_t n5[3], n9[4], n11[4], n13[4], n15[4], n17[5];
    bs_next<3>(v5, n5);
    bs_next<4>(v9, n9);
    bs_next<4>(v11, n11);
    bs_next<4>(v13, n13);
    bs_next<4>(v15, n15);
    bs_next<5>(v17, n17);
    // Horizontal: offsets dx = 0..16 from the window's first column; level by |dx - 8|.
    uint32_t a1[4], a2[5], a3[5], a4[5], a5[5], a6[5], a7[6], a8[6], a9[5];
    bs_pair<3>(v5, n5, 0, a1);      // dx 0, 16: max 10
    bs_pair<4>(v9, n9, 1, a2);      // dx 1, 15: 18
    bs_pair<4>(v11, n11, 2, a3);    // dx 2, 14: 22
    bs_pair<4>(v13, n13, 3, a4);    // dx 3, 13: 26
    bs_pair<4>(v15, n15, 4, a5);    // dx 4, 12: 30
    bs_pair<4>(v15, n15, 5, a6);    // dx 5, 11: 30
    bs_pair<5>(v17, n17, 6, a7);    // dx 6, 10: 34
    bs_pair<5>(v17, n17, 7, a8);    // dx 7, 9: 34
    bs_shift<5>(v17, n17, 8, a9);   // dx 8: 17
    uint32_t b1[5], b2[6], b3[6], b4[7], c1[7], c2[8], d[8];
    bs_add<5, 4, 5>(a2, a1, b1);    // 28
    bs_add<5, 5, 6>(a3, a4, b2);    // 48
    bs_add<5, 5, 6>(a5, a6, b3);    // 60
    bs_add<6, 6, 7>(a7, a8, b4);    // 68
    bs_add<6, 5, 7>(b2, b1, c1);    // 76
    bs_add<7, 6, 8>(b4, b3, c2);    // 128
    bs_add<8, 7, 8>(c2, c1, d);     // 204
    bs_add<8, 5, 8>(d, a9, cnt);    // 221
}

// Number of set bits among 17 single-bit vectors (per bit position), as 5 planes: a carry-save
// tree of 12 full adders and 3 half adders.
__device__ __forceinline__ void bs_popcount17(const uint32_t (&b)[17], uint32_t (&o)[5]) {
    uint32_t s1[5], c2[8];
#pragma unroll
    for (int i = 0; i < 5; ++i) bs_fa(b[3 * i], b[3 * i + 1], b[3 * i + 2], s1[i], c2[i]);
    // weight 1: s1[0..4], b[15], b[16]
    uint32_t t0, t1, u0;
    bs_fa(s1[0], s1[1], s1[2], t0, c2[5]);
    bs_fa(s1[3], s1[4], b[15], t1, c2[6]);
    bs_fa(t0, t1, b[16], o[0], c2[7]);
    // weight 2: c2[0..7]
    uint32_t w2a, w2b, w4[4];
    bs_fa(c2[0], c2[1], c2[2], w2a, w4[0]);
    bs_fa(c2[3], c2[4], c2[5], w2b, w4[1]);
    bs_fa(c2[6], c2[7], w2a, u0, w4[2]);
    o[1] = u0 ^ w2b;
    w4[3] = u0 & w2b;
    // weight 4: w4[0..3]
    uint32_t w4a, w8[2];
    bs_fa(w4[0], w4[1], w4[2], w4a, w8[0]);
    o[2] = w4a ^ w4[3];
    w8[1] = w4a & w4[3];
    o[3] = w8[0] ^ w8[1];
    o[4] = w8[0] & w8[1];
}

// Window-relative vertical half-extent of column offset dx (0..16 from the window's first column):
// the column holds window rows 8 - H .. 8 + H.
__host__ __device__ constexpr int column_half_height(int dx) {
    return dx == 0 || dx == 16 ? 2 : dx == 1 || dx == 15 ? 4 : dx == 2 || dx == 14 ? 5
         : dx == 3 || dx == 13 ? 6 : dx <= 5 || dx >= 11 ? 7 : 8;
}

// Counts of the windows starting one row lower than `cnt` (window start DZ - 1 -> DZ among the
// rows R / next-word rows Rn): per column one cell enters (row DZ + 8 + H) and one leaves (row
// DZ + 7 - H), so count' = count + entering - leaving (mod 256, exact since counts are 0..221).
// DZ = 0 reads row -1 (R[-1], Rn[-1] must exist).
template <int DZ>
__device__ __forceinline__ void bs_slide(const uint32_t* R, const uint32_t* Rn, uint32_t (&cnt)[8]) {
    uint32_t in[17], out[17];
#pragma unroll
    for (int dx = 0; dx < 17; ++dx) {
        const int h = column_half_height(dx);
        in[dx] = __funnelshift_r(R[DZ + 8 + h], Rn[DZ + 8 + h], dx);
        out[dx] = __funnelshift_r(R[DZ + 7 - h], Rn[DZ + 7 - h], dx);
    }
    uint32_t a[5], b[5];
    bs_popcount17(in, a);
    bs_popcount17(out, b);
    // count + a + ~b + 1 over 8 planes: carry-save, then a ripple add with carry-in 1.
    uint32_t sv[8], cv[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t y = i < 5 ? a[i] : 0u, z = i < 5 ? ~b[i] : ~0u;
        bs_fa(cnt[i], y, z, sv[i], cv[i]);
    }
    uint32_t c = ~0u;  // the +1 of the two's complement
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t y = i == 0 ? 0u : cv[i - 1];
        uint32_t o;
        bs_fa(sv[i], y, c, o, c);
        cnt[i] = o;
    }
}

// Centres whose count is at least t (t in 0..256): the carry out of count + (256 - t), with
// the constant's bits known (one LOP3 per plane).
__device__ __forceinline__ uint32_t bs_at_least(const uint32_t (&cnt)[8], int t) {
    const uint32_t k = 256u - (uint32_t)t;
    uint32_t c = 0;
#pragma unroll
    for (int b = 0; b < 8; ++b) c = ((k >> b) & 1u) ? (cnt[b] | c) : (cnt[b] & c);
    return (k & 256u) ? ~0u : c;
}

__device__ __forceinline__ int bs_value(const uint32_t (&cnt)[8], int j) {
    int v = 0;
#pragma unroll
    for (int b = 0; b < 8; ++b) v |= (int)((cnt[b] >> j) & 1u) << b;
    return v;
}

// Exact counts of strip st (window rows 4(st-4) .. 4st+3, centres of 4 rows) for the warp's
// combos; centres in [min_size, max_size] (and outside the rd_min disc) are appended to the hit
// list. Called by the whole warp; lane = word.
template <bool kMasked, int kMode>
__device__ __forceinline__ void exact_strip(BandSmem& S, const BandArgs& a, const Tile& T, const Counter& C,
                                            int st, int warp, int lane, uint32_t fx) {
    constexpr int kUsed = kMode == kModeShared ? kSlots : kMaxBands / kWarps;
    const int r0 = 4 * (st - 4);
    // Output columns of this word: centre index c = 32 lane + j < kOutW and inside the area.
    const int64_t u_first = (int64_t)T.u0 + 32 * lane;
#pragma unroll 1
    for (int k = 0; k < kUsed; ++k) {
        const int combo = warp + kWarps * k;
        const int m = combo_band<kMode>(combo), ph = combo_phase<kMode>(combo);
        if (m >= a.nb) continue;  // warp-uniform: planes of bands beyond the count are empty
        // Rows r0 - 1 .. r0 + 19 of the combo (row r0 - 1 only when the strip slides on from the
        // previous one; its batch may already be overwritten in the ring, so it comes from what the
        // previous strip saved).
        uint32_t Rx[21], Rnx[21];
        uint32_t* const R = Rx + 1;
        uint32_t* const Rn = Rnx + 1;
#pragma unroll
        for (int i = 0; i < 20; ++i) {
            uint32_t w = combo_word<kMode>(S, r0 + i, combo, fx, lane);
            if (kMasked) w &= C.cm[k];
            R[i] = w;
        }
        // Columns of the word that are output centres of this combo.
        uint32_t colok;
        {
            const int64_t ulim = min((int64_t)a.ubase, a.width_u - (int64_t)(T.i0 + ph) * kPeriod);
            const int64_t nv = min(ulim - u_first, (int64_t)kOutW - 32 * lane);
            colok = nv >= 32 ? ~0u : nv <= 0 ? 0u : (1u << nv) - 1u;
        }
        const int64_t band_v = band_row0<kMode>(S, a, m);
        // The next word's rows (lane 31 gets its own back: only its centres 16+, which lie beyond
        // the tile's output columns, would read them).
#pragma unroll
        for (int i = 0; i < 20; ++i) Rn[i] = __shfl_down_sync(kFull, R[i], 1);
        uint32_t cnt[8];
        // Strips after a tile's first continue from the previous strip's last window row: its 8
        // count planes and its row 3 (this strip's row -1) wait in the box-sum history, which the
        // exact modes do not use (9 words per combo and lane).
        uint32_t* const saved = &S.hist_e[0][0][0] + (size_t)combo * 9 * kWords + lane;
        const bool slide_in = st > 4 && a.rd_min_sq == 0;
        if (slide_in) {
#pragma unroll
            for (int i = 0; i < 8; ++i) cnt[i] = saved[i * kWords];
            Rx[0] = saved[8 * kWords];
        } else {
            Rx[0] = 0u;
        }
        Rnx[0] = __shfl_down_sync(kFull, Rx[0], 1);
        // Annulus searches: skip the strip when all of its centres lie inside the rd_min disc
        // (warp-uniform: the strip's 4 rows across the tile's output columns).
        if (a.rd_min_sq) {
            const int64_t u0 = (int64_t)T.u0 + (int64_t)(T.i0 + ph) * kPeriod, u1 = u0 + kOutW - 1;
            const int64_t v0 = (int64_t)T.v0 + r0 + band_v, v1 = v0 + 3;
            const int64_t x0 = a.transposed ? v0 : u0, x1 = a.transposed ? v1 : u1;
            const int64_t z0 = a.transposed ? u0 : v0, z1 = a.transposed ? u1 : v1;
            if (rect_inside_disc(a.area_x0 + x0, a.area_x0 + x1, a.area_z0 + z0, a.area_z0 + z1, a.center_x,
                                 a.center_z, a.rd_min_sq))
                continue;
        }
#pragma unroll
        for (int dz = 0; dz < 4; ++dz) {
            const int rr = r0 + dz;  // window start row = centre row index in the tile
            const int64_t v = (int64_t)T.v0 + rr;
            const bool rowok = rr < T.out_h && v + band_v < a.height_v;
            // A tile's first window row is counted in full; every later one slides down a row.
            if (dz == 0) {
                if (slide_in) bs_slide<0>(R, Rn, cnt);
                else bs_window_counts<0>(*reinterpret_cast<const uint32_t(*)[20]>(R), cnt);
            } else if (dz == 1) bs_slide<1>(R, Rn, cnt);
            else if (dz == 2) bs_slide<2>(R, Rn, cnt);
            else bs_slide<3>(R, Rn, cnt);
            uint32_t pass = rowok ? colok & bs_at_least(cnt, a.min_size) : 0u;
            if (a.max_size < 221) pass &= ~bs_at_least(cnt, a.max_size + 1);
            if (!__any_sync(kFull, pass != 0)) continue;
            // This lane's centres in range outside the rd_min disc: all counted, those at or above
            // the emission gate appended.
            const int64_t cv = v + band_v;
            const uint32_t gate = a.emit_min > a.min_size ? bs_at_least(cnt, a.emit_min) : ~0u;
            uint32_t keep = 0;
            for (uint32_t p = pass; p; p &= p - 1) {
                const int j = __ffs(p) - 1;
                if (a.rd_min_sq) {
                    const int64_t cu = u_first + j + (int64_t)(T.i0 + ph) * kPeriod;
                    const int32_t cx = (int32_t)(a.transposed ? a.area_x0 + cv : a.area_x0 + cu);
                    const int32_t cz = (int32_t)(a.transposed ? a.area_z0 + cu : a.area_z0 + cv);
                    const int64_t ddx = (int64_t)cx - a.center_x, ddz = (int64_t)cz - a.center_z;
                    if (ddx * ddx + ddz * ddz < a.rd_min_sq) continue;
                }
                if (a.hist) atomicAdd(&S.hist[bs_value(cnt, j)], 1u);
                keep |= (gate >> j & 1u) << j;
            }
            const int n = __popc(keep);
            int pos = n;
#pragma unroll
            for (int d2 = 1; d2 < 32; d2 <<= 1) {
                const int t = __shfl_up_sync(kFull, pos, d2);
                if (lane >= d2) pos += t;
            }
            const int total = __shfl_sync(kFull, pos, 31);
            if (total == 0) continue;
            unsigned long long base = 0;
            if (lane == 31) base = atomicAdd(a.emitted, (unsigned long long)total);
            base = __shfl_sync(kFull, base, 31) + (unsigned long long)(pos - n);
            for (uint32_t p = keep; p; p &= p - 1, ++base) {
                const int j = __ffs(p) - 1;
                const int64_t cu = u_first + j + (int64_t)(T.i0 + ph) * kPeriod;
                const int32_t cx = (int32_t)(a.transposed ? a.area_x0 + cv : a.area_x0 + cu);
                const int32_t cz = (int32_t)(a.transposed ? a.area_z0 + cu : a.area_z0 + cv);
                if (base < a.cap) a.out[base] = Hit{bs_value(cnt, j), cx, cz};
            }
        }
        if (a.rd_min_sq == 0) {  // for the next strip of the tile
#pragma unroll
            for (int i = 0; i < 8; ++i) saved[i * kWords] = cnt[i];
            saved[8 * kWords] = R[3];
        }
    }
}

// First-draw test of one chunk from split terms (independent bands: nothing is shared).
template <bool kMadAdd>
__device__ __forceinline__ bool indep_hit(uint32_t xl, uint32_t xh, uint32_t zl, uint32_t zh, uint32_t one) {
    const uint32_t s = kMadAdd ? xl * one + zl : xl + zl;
    const uint32_t l = (s & 0x1FFFFu) ^ kXorLo;
    const uint64_t prod = (uint64_t)l * kA32 + 11u;
    const uint32_t q = (uint32_t)(prod >> kPeriodBits) + l * kQLimbMul;
    const uint32_t h = (xh + zh + (s >> kPeriodBits)) ^ kXorHi;
    const uint32_t t = h * kA32 + q;  // bits (mod 2^32): even and t * 2/5 small <=> slime
    return !(t & 1u) && t * kTwoInv5 < kHitBelow;
}

// CTA set-up shared by the kernels: mbarriers and a zeroed ring (with the shared LCG, planes of
// bands beyond nb are never generated: they stay zero and count nothing).
__device__ __forceinline__ void band_cta_init(BandSmem& S, int tid) {
    if (tid == 0) {
        S.failed = 0;
        for (int r = 0; r < 3; ++r)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&S.rows_bar[r])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < kRingSlots * kBatchRows * kPlanes * kWords; i += kTpb) (&S.ring[0][0][0][0])[i] = 0;
    for (int i = tid; i < kHistBins; i += kTpb) S.hist[i] = 0;
    __syncthreads();
}

// One tile of one search (block-uniform arguments; all threads). Returns false when a bounded
// wait gave up (the search's overflow word gets bit 4 and the CTA must stop).
template <bool kMadAdd, int kMode, bool kCands, bool kExact = false>
__device__ __forceinline__ bool band_tile(BandSmem& S, const BandArgs& a, int64_t tile, int tid, int lane,
                                          int warp, uint32_t& bar_phase) {
    const int nb = a.nb;
    const uint32_t thr4 = (uint32_t)min(a.min_size, 128) * 0x01010101u;
    const uint32_t one = a.one;  // 1 at run time: keeps the band add on the multiply pipe
    // Counter constants: the swap sense of the warp's phase and the groups lane 31 may flag
    // (groups 4..7 of word 31 hold centres 1,008+ of the tile, which belong to the next tile).
    // (Grouped bands: the phase alone; each band's copy parity is applied per combo.)
    const uint32_t fx = kMode == kModeGrouped ? ((warp & 1) ? 0u : ~0u) : (((warp ^ (warp >> 1)) & 1) ? 0u : ~0u);
    const uint32_t lastmask = lane == kWords - 1 ? 0x0000C0C0u : ~0u;
    const uint32_t umask = lane < 20 ? group_union_mask(lane) : 0u;
    uint32_t guard = 0;
    int ncand = 0;  // warp-uniform length of this warp's candidate list
    {
        Tile T;
        const int ut = (int)(tile % a.u_tiles);
        const int64_t rest = tile / a.u_tiles;
        const int vt = (int)(rest % a.v_tiles);
        T.i0 = kMode == kModeIndep ? 0 : 2 * (int)(rest / a.v_tiles);
        T.u0 = ut * kOutW;
        T.v0 = vt * a.band_h;
        // Tiles with no centre of the area in any of their combos are skipped (block-uniform).
        if ((int64_t)T.u0 + (int64_t)T.i0 * kPeriod >= a.width_u ||
            (int64_t)T.v0 + (int64_t)a.j0 * a.row_stride >= a.height_v)
            return true;
        T.out_h = min(a.band_h, a.vbase - T.v0);
        const int strips = (T.out_h + 16 + 3) / 4;
        const int batches = (strips + 1) / 2;
        constexpr int kRW = row_words<kMode>();
        constexpr uint32_t kBatchBytes = kBatchRows * kRW * 4;

        // Generator columns of this thread: words kGenW*(warp % kGenColWarps) .. + kGenW - 1, lane =
        // bit; the warp generates rows kGenRows*(warp / kGenColWarps) .. of every 8-row batch.
        const int gw = (warp % kGenColWarps) * kGenW, gq = (warp / kGenColWarps) * kGenRows;
        uint32_t lox[kGenW], xh0[kGenW], xh1[kGenW];
#pragma unroll
        for (int k = 0; k < kGenW; ++k) {
            const int64_t idx0 = (int64_t)T.u0 + (gw + k) * 32 + lane + (int64_t)T.i0 * kPeriod;
            const uint64_t x0 = idx0 < a.ncols ? a.ct[idx0] : 0;
            const uint64_t x1 = idx0 + kPeriod < a.ncols ? a.ct[idx0 + kPeriod] : 0;
            lox[k] = (uint32_t)x0 & 0x1FFFFu;
            xh0[k] = (uint32_t)(x0 >> kPeriodBits);
            xh1[k] = (uint32_t)(x1 >> kPeriodBits);
        }
        // Counter slots of this warp: combo rows warp + 16*k; lane = word.
        Counter C;
#pragma unroll
        for (int k = 0; k < kSlots; ++k) {
            C.cm[k] = column_mask(a, T, lane, combo_phase<kMode>(warp + kWarps * k));
            C.re[k] = C.ro[k] = 0;
        }
        // Tiles whose columns all exist in both phases skip the column masks (block-uniform).
        // Rows need no mask: the generator writes zero words for bands that do not hold a row.
        const bool interior = (int64_t)T.u0 + kWords * 32 + (int64_t)(T.i0 + (kMode == kModeIndep ? 0 : 1)) * kPeriod <= a.ncols;
        for (int i = tid; i < 5 * kMaxCombos * kWords; i += kTpb) {
            (&S.hist_e[0][0][0])[i] = 0;
            (&S.hist_o[0][0][0])[i] = 0;
        }
        // Grouped bands: per band its first area row, swap plane and copy parity.
        if (kMode == kModeGrouped && tid < kGrpBands) {
            const int G = a.groups;
            S.goff[tid] = (tid / G) * (int32_t)kPeriod + (tid % G) * (int32_t)a.row_stride;
            S.gsw[tid] = kGrpSw + tid % G;
            S.gflip[tid] = ((tid / G) & 1) ? ~0u : 0u;
        }
        // Row terms of batches 0 and 1 (batch b lives in rows[b % 3]).
        if (tid == 0) {
            bulk_load(&S.rows[0][0], a.rt + (int64_t)T.v0 * kRW, kBatchBytes, &S.rows_bar[0]);
            if (batches > 1)
                bulk_load(&S.rows[1][0], a.rt + (int64_t)(T.v0 + kBatchRows) * kRW, kBatchBytes, &S.rows_bar[1]);
        }
        __syncthreads();

        for (int b = 0; b < batches; ++b) {
            const int rb = b % 3, slot = b & (kRingSlots - 1);
            // ---- generator: batch b into ring slot b % 4 ------------------------------------
            if (!bar_wait(&S.rows_bar[rb], (bar_phase >> rb) & 1u, a.poll_limit)) {
                S.failed = 1;
                if (lane == 0) atomicOr(a.overflow, 4u);
            }
            bar_phase ^= 1u << rb;
            if constexpr (kMode == kModeIndep) {
#pragma unroll 1
            for (int qq = 0; qq < kGenRows; ++qq) {
                const int q = gq + qq;
                const uint32_t* zr = &S.rows[rb][q * kRowWordsI];
                const int nv = __shfl_sync(kFull, min((int)zr[kRowValidI], nb), 0);  // warp-uniform
                uint4* dst = reinterpret_cast<uint4*>(&S.ring[slot][q][0][gw]);
                constexpr int kPlaneStep = kWords / 4;
                int m = 0;
                for (; m + 1 < nv; m += 2) {
                    const uint2 zh = *reinterpret_cast<const uint2*>(zr + m);
                    const uint2 zl = *reinterpret_cast<const uint2*>(zr + kRowLoI + m);
                    uint32_t wa[kGenW], wb[kGenW];
#pragma unroll
                    for (int k = 0; k < kGenW; ++k) {
                        wa[k] = __ballot_sync(kFull, indep_hit<kMadAdd>(lox[k], xh0[k], zl.x, zh.x, one));
                        wb[k] = __ballot_sync(kFull, indep_hit<kMadAdd>(lox[k], xh0[k], zl.y, zh.y, one));
                    }
                    store_plane(dst + m * kPlaneStep, wa);
                    store_plane(dst + (m + 1) * kPlaneStep, wb);
                }
                if (m < nv) {
                    uint32_t wa[kGenW];
#pragma unroll
                    for (int k = 0; k < kGenW; ++k)
                        wa[k] = __ballot_sync(kFull, indep_hit<kMadAdd>(lox[k], xh0[k], zr[kRowLoI + m], zr[m], one));
                    store_plane(dst + m * kPlaneStep, wa);
                    ++m;
                }
                for (; m < nb; ++m) clear_plane(dst + m * kPlaneStep);  // rows outside band m
            }
            } else if constexpr (kMode == kModeGrouped) {
#pragma unroll 1
            for (int qq = 0; qq < kGenRows; ++qq) {
                const int q = gq + qq;
                const uint32_t* zr = &S.rows[rb][q * kRowWordsI];
                const int nv = __shfl_sync(kFull, min((int)zr[kRowValidI], nb), 0);  // warp-uniform
                uint4* dst = reinterpret_cast<uint4*>(&S.ring[slot][q][0][gw]);
                constexpr int kPlaneStep = kWords / 4;
                const int G = a.groups;
                auto hit = [&](uint32_t x, uint32_t z, uint32_t d) {
                    const uint32_t t = kMadAdd ? z * one + x : z + x;
                    return ((t ^ kXorHi) * kMulH + d) < kHitBelow;
                };
#pragma unroll 1
                for (int g = 0; g < G; ++g) {
                    // Group g: the shared part from the low bits of its row (the same in every copy)
                    // and, from copy 0's high part, which phase of the pair each copy tests.
                    const uint32_t zlo = zr[kRowLoI + g];
                    const uint32_t zpar = (zr[g] ^ kXorHi) & 1u;
                    uint32_t xa[kGenW], xb[kGenW], dd[kGenW], sw[kGenW];
#pragma unroll
                    for (int k = 0; k < kGenW; ++k) {
                        const Shared sh = shared_part(lox[k], zlo);
                        const uint32_t pi = (sh.q0 ^ xh0[k] ^ sh.carry ^ zpar) & 1u;
                        xa[k] = (pi ? xh1[k] : xh0[k]) + sh.carry;
                        xb[k] = (pi ? xh0[k] : xh1[k]) + sh.carry;
                        dd[k] = sh.d;
                        sw[k] = __ballot_sync(kFull, pi != 0);
                    }
                    store_plane(dst + (kGrpSw + g) * kPlaneStep, sw);
                    // Copies c and c + 1: bands m = c G + g and m + G (even copies test the phase
                    // of xa, odd copies that of xb). Bands from nv on do not hold this row.
#pragma unroll 1
                    for (int m = g; m < nb; m += 2 * G) {
                        const int m1 = m + G;
                        uint32_t wa[kGenW], wb[kGenW];
                        if (m1 < nv) {
                            const uint32_t z0 = zr[m], z1 = zr[m1];
#pragma unroll
                            for (int k = 0; k < kGenW; ++k) {
                                wa[k] = __ballot_sync(kFull, hit(xa[k], z0, dd[k]));
                                wb[k] = __ballot_sync(kFull, hit(xb[k], z1, dd[k]));
                            }
                            store_plane(dst + m * kPlaneStep, wa);
                            store_plane(dst + m1 * kPlaneStep, wb);
                        } else {
                            if (m < nv) {
                                const uint32_t z0 = zr[m];
#pragma unroll
                                for (int k = 0; k < kGenW; ++k) wa[k] = __ballot_sync(kFull, hit(xa[k], z0, dd[k]));
                                store_plane(dst + m * kPlaneStep, wa);
                            } else {
                                clear_plane(dst + m * kPlaneStep);
                            }
                            if (m1 < nb) clear_plane(dst + m1 * kPlaneStep);
                        }
                    }
                }
            }
            } else {
#pragma unroll 1
            for (int qq = 0; qq < kGenRows; ++qq) {
                const int q = gq + qq;
                const uint32_t* zr = &S.rows[rb][q * kRowWords];
                const uint32_t zlo = zr[kRowLo];
                // Bands 0..nv-1 hold this row. The broadcast tells the compiler that the value
                // (and the loops it bounds) is warp-uniform.
                const int nv = __shfl_sync(kFull, min((int)zr[kRowValid], nb), 0);
                const uint32_t zpar = (zr[0] ^ kXorHi) & 1u;
                uint32_t xa[kGenW], xb[kGenW], dd[kGenW], sw[kGenW];
#pragma unroll
                for (int k = 0; k < kGenW; ++k) {
                    const Shared sh = shared_part(lox[k], zlo);
                    const uint32_t pi = (sh.q0 ^ xh0[k] ^ sh.carry ^ zpar) & 1u;
                    xa[k] = (pi ? xh1[k] : xh0[k]) + sh.carry;
                    xb[k] = (pi ? xh0[k] : xh1[k]) + sh.carry;
                    dd[k] = sh.d;
                    sw[k] = __ballot_sync(kFull, pi != 0);
                }
                // Plane m of the warp's 4 words at dst + m * kWords (16-byte aligned). Every lane
                // stores the same ballot words to the same address: no predicate, no branch.
                uint4* dst = reinterpret_cast<uint4*>(&S.ring[slot][q][0][gw]);
                constexpr int kPlaneStep = kWords / 4;  // uint4 per plane
                store_plane(dst + kSwPlane * kPlaneStep, sw);
                auto hit = [&](uint32_t x, uint32_t z, uint32_t d) {
                    const uint32_t t = kMadAdd ? z * one + x : z + x;
                    return ((t ^ kXorHi) * kMulH + d) < kHitBelow;
                };
                // Bands 0..count-1 of the row; returns count.
                auto bands = [&](const int count) {
                    int m = 0;
                    // Two band pairs per iteration (measured 2 % faster on the full-world scan).
#pragma unroll 2
                    for (; m + 1 < count; m += 2) {
                        const uint2 z2 = *reinterpret_cast<const uint2*>(zr + m);  // m even: aligned
                        uint32_t wa[kGenW], wb[kGenW];
#pragma unroll
                        for (int k = 0; k < kGenW; ++k) {
                            wa[k] = __ballot_sync(kFull, hit(xa[k], z2.x, dd[k]));
                            wb[k] = __ballot_sync(kFull, hit(xb[k], z2.y, dd[k]));
                        }
                        store_plane(dst + m * kPlaneStep, wa);
                        store_plane(dst + (m + 1) * kPlaneStep, wb);
                    }
                    if (m < count) {  // odd count: the last band (m even) uses the even-band phase choice
                        const uint32_t z0 = zr[m];
                        uint32_t wa[kGenW];
#pragma unroll
                        for (int k = 0; k < kGenW; ++k) wa[k] = __ballot_sync(kFull, hit(xa[k], z0, dd[k]));
                        store_plane(dst + m * kPlaneStep, wa);
                    }
                };
                if (nv == nb) {
                    bands(nb);  // the common case: the kernel-uniform band count bounds the loop
                } else {
                    bands(nv);
                    for (int m = nv; m < nb; ++m) clear_plane(dst + m * kPlaneStep);  // rows outside band m
                }
            }
            }
            __syncthreads();
            if (S.failed) {  // block-uniform after the barrier
                // Before the CTA leaves, wait (bounded) for its row-term copies still in flight:
                // batch b's (the wait that gave up) and batch b + 1's.
                if (tid == 0) {
                    constexpr uint32_t kDrainPolls = 1u << 22;
                    bar_wait(&S.rows_bar[rb], ((bar_phase >> rb) & 1u) ^ 1u, kDrainPolls);
                    if (b + 1 < batches) {
                        const int rn = (b + 1) % 3;
                        bar_wait(&S.rows_bar[rn], (bar_phase >> rn) & 1u, kDrainPolls);
                    }
                }
                __syncthreads();
                return false;
            }

            // Row terms of batch b + 2 (its buffer was last read before this batch's barrier).
            if (tid == kTpb - 32 && b + 2 < batches)
                bulk_load(&S.rows[(b + 2) % 3][0], a.rt + (int64_t)(T.v0 + kBatchRows * (b + 2)) * kRW,
                          kBatchBytes, &S.rows_bar[(b + 2) % 3]);

            // ---- counter: the two strips of batch b ------------------------------------------
            if constexpr (kExact) {
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    if (2 * b + t < 4) continue;  // windows complete from the fifth strip on
                    if (interior) exact_strip<false, kMode>(S, a, T, C, 2 * b + t, warp, lane, fx);
                    else exact_strip<true, kMode>(S, a, T, C, 2 * b + t, warp, lane, fx);
                }
                continue;
            } else {
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    if (interior)
                        count_strip<false, kMode, kCands>(S, a, T, C, slot, t, 2 * b + t, warp, lane, fx, lastmask, thr4,
                                                           umask, guard, ncand);
                    else
                        count_strip<true, kMode, kCands>(S, a, T, C, slot, t, 2 * b + t, warp, lane, fx, lastmask, thr4,
                                                          umask, guard, ncand);
                }
            }
            // Candidates of this batch need rows of batches b-2..b, which stay in the ring until
            // batch b+2 is generated (after the next barrier).
            if (kCands && ncand) {
                if (interior) flush_cands<false, kMode>(S, a, T, fx, warp, lane, umask, ncand);
                else flush_cands<true, kMode>(S, a, T, fx, warp, lane, umask, ncand);
                ncand = 0;
            }
        }
        __syncthreads();  // the next tile reuses ring slots and histories still read above
    }
    // A 4-row strip with 52+ hits among its 80 cells could carry a box past a byte lane.
    if (guard & 0x80808080u) atomicOr(a.overflow, 1u);
    return true;
}

// Survivor handling: below this threshold the 368-cell survivors are many, and batching their
// union counts per warp (kCands) pays; above it they are rare and are counted at once.
constexpr int kCandThreshold = 56;

template <bool kMadAdd, int kMode, bool kCands, bool kExact = false>
__global__ void __launch_bounds__(kTpb, 1) band_scan_kernel(const BandArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BandSmem& S = *reinterpret_cast<BandSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31;
    const int warp = __shfl_sync(kFull, tid >> 5, 0);  // warp-uniform for the compiler
    uint32_t bar_phase = 0;  // bit r: parity of the next completion of rows_bar[r]
    band_cta_init(S, tid);
    for (int64_t tile = a.tile_begin + blockIdx.x; tile < a.tile_end; tile += gridDim.x)
        if (!band_tile<kMadAdd, kMode, kCands, kExact>(S, a, tile, tid, lane, warp, bar_phase)) return;
    if (a.hist) {
        __syncthreads();
        for (int i = tid; i < kHistBins; i += kTpb)
            if (S.hist[i]) atomicAdd(&a.hist[i], S.hist[i]);
    }
}

// Many searches of one launch class (band mode, survivor lists, exact counts) in one persistent
// launch: each CTA takes the next tile of the launch from a device counter, finds its search in
// the tile prefix sums and copies that search's arguments into shared memory. Work item i covers
// tiles args[i].tile_begin .. + (prefix[i+1] - prefix[i]) of its search; prefix[0] need not be 0.
// One class per launch keeps the kernel as lean as the single-search one (no spills). Stale
// planes of a previous search with more bands are never read by the independent- and grouped-
// band counters or the exact counts (they skip bands beyond the band count) and are cleared
// before a shared-LCG tile.
template <int kMode, bool kCands, bool kExact>
__global__ void __launch_bounds__(kTpb, 1) band_batch_kernel(const BandArgs* args, const int64_t* prefix,
                                                             int32_t nsearch, unsigned long long* head) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BandSmem& S = *reinterpret_cast<BandSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31;
    const int warp = __shfl_sync(kFull, tid >> 5, 0);
    uint32_t bar_phase = 0;
    band_cta_init(S, tid);
    const int64_t first = prefix[0], total = prefix[nsearch];
    for (;;) {
        if (tid == 0) {
            const long long t = first + (long long)atomicAdd(head, 1ull);
            int lo = 0, hi = nsearch - 1;  // last search whose first tile is <= t
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (prefix[mid] <= t) lo = mid; else hi = mid - 1;
            }
            S.next_tile = t;
            S.search = lo;
        }
        __syncthreads();
        const int64_t t = S.next_tile;
        if (t >= total) return;  // block-uniform
        const int s = S.search;
        constexpr int kArgWords = (int)(sizeof(BandArgs) / 4);
        for (int i = tid; i < kArgWords; i += kTpb)
            reinterpret_cast<uint32_t*>(&S.args)[i] = reinterpret_cast<const uint32_t*>(&args[s])[i];
        __syncthreads();
        if (kMode == kModeShared && !kExact) {
            // The shared-LCG counter reads every plane: clear planes of bands this search does
            // not generate (a previous search may have left bits there).
            for (int i = tid; i < kRingSlots * kBatchRows * kMaxBands * kWords; i += kTpb) {
                const int m = (i / kWords) % kMaxBands;
                if (m >= S.args.nb) {
                    const int w = i % kWords, r = i / (kWords * kMaxBands);
                    S.ring[r / kBatchRows][r % kBatchRows][m][w] = 0;
                }
            }
            __syncthreads();
        }
        if (!band_tile<true, kMode, kCands, kExact>(S, S.args, S.args.tile_begin + t - prefix[s], tid, lane, warp,
                                                     bar_phase)) {
            if (tid == 0) atomicOr(S.args.overflow, 4u);
            return;
        }
        // The tile's search keeps a count histogram: add this tile's counts to it (band_tile ended
        // with a barrier) and clear them before the next tile, which may be another search's.
        if (S.args.hist) {
            for (int i = tid; i < kHistBins; i += kTpb)
                if (S.hist[i]) {
                    atomicAdd(&S.args.hist[i], S.hist[i]);
                    S.hist[i] = 0;
                }
        }
    }
}

// Row-term table, one record per (band group g, base row v), records of a group contiguous.
// Band j = 32 g + m holds base row v at input row v + j * stride (stride 2^17 with the shared
// LCG). Shared-LCG records (kRowWords): [m] = high part (>> 17) of the row term in band m (0 where
// the row lies outside the area plus halo), [kRowLo] = its low 17 bits (the same in every band),
// [kRowValid] = number of bands of the group that hold the row. Independent records
// (kRowWordsI): [m] high part, [kRowLoI + m] low 17 bits, [kRowValidI] bands holding the row.
// Grouped bands use the independent layout with band j = c * G + g at input row
// v + c * 2^17 + g * stride (G * stride = 2^17 when there are several copies, so the bands' rows
// increase with j and the bands holding a row are a prefix). Rows v >= vrows (padding) are zero.
template <int kMode>
__global__ void row_terms_kernel(uint32_t* rt, int32_t vrows_alloc, int32_t vrows, int32_t nj,
                                 int32_t first, int64_t limit, int64_t stride, int64_t seed,
                                 int32_t use_x_term, int32_t G) {
    constexpr bool kSplit = kMode != kModeShared;  // low bits per band
    constexpr int kRW = row_words<kMode>();
    constexpr int kLo = kSplit ? kRowLoI : kRowLo;
    constexpr int kValid = kSplit ? kRowValidI : kRowValid;
    const int32_t groups = (nj + kMaxBands - 1) / kMaxBands;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)groups * vrows_alloc * kRW) return;
    const int32_t w = (int32_t)(e % kRW);
    const int64_t rec = e / kRW;
    const int32_t v = (int32_t)(rec % vrows_alloc), g = (int32_t)(rec / vrows_alloc);
    auto band_off = [&](int32_t j) -> int64_t {
        return kMode == kModeGrouped ? (int64_t)(j / G) * kPeriod + (int64_t)(j % G) * stride : (int64_t)j * stride;
    };
    uint32_t out = 0;
    if (v < vrows) {
        const bool hi = w < kMaxBands;
        const bool lo = kSplit ? (w >= kLo && w < kLo + kMaxBands) : w == kLo;
        if (hi || lo) {
            const int32_t m = hi ? w : kSplit ? w - kLo : 0;
            const int32_t j = (!kSplit && lo) ? 0 : g * kMaxBands + m;
            const int64_t off = (int64_t)v + band_off(j);
            if (j < nj && off < limit) {
                const int32_t c = (int32_t)((int64_t)first + off);
                const uint64_t t = (use_x_term ? x_term(c) : z_term(c)) + (uint64_t)seed;
                out = lo ? (uint32_t)t & 0x1FFFFu : (uint32_t)(t >> kPeriodBits);
            }
        } else if (w == kValid) {
            if (kMode == kModeGrouped) {  // one group of at most 16 bands, rows increasing with j
                int32_t n = 0;
                while (n < nj && (int64_t)v + band_off(n) < limit) ++n;
                out = (uint32_t)n;
            } else {
                // bands j = 32g + m with v + j * stride < limit, capped at the group's size
                const int64_t jmax = (limit - 1 - v) / stride;  // last band holding the row
                const int64_t n = min((int64_t)nj, jmax + 1) - (int64_t)g * kMaxBands;
                out = (uint32_t)max((int64_t)0, min((int64_t)kMaxBands, n));
            }
        }
    }
    rt[e] = out;
}

__global__ void col_terms_kernel(uint64_t* ct, int32_t first, int32_t n, int32_t use_x_term) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t c = (int32_t)((int64_t)first + i);
    ct[i] = use_x_term ? x_term(c) : z_term(c);
}

}  // namespace

size_t band_smem_bytes() { return sizeof(BandSmem); }

namespace {
// The batch kernel of launch class `cls` (band_class): launched over `grid` CTAs, or, with
// grid == 0, given its dynamic shared-memory size (`prepare_bytes`).
template <int kMode, bool kCands, bool kExact>
cudaError_t batch_one(const BandArgs* args, const int64_t* prefix, int32_t n, unsigned long long* head, int grid,
                      cudaStream_t s, int prepare_bytes) {
    if (grid == 0)
        return cudaFuncSetAttribute(band_batch_kernel<kMode, kCands, kExact>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    prepare_bytes);
    band_batch_kernel<kMode, kCands, kExact><<<grid, kTpb, sizeof(BandSmem), s>>>(args, prefix, n, head);
    return cudaGetLastError();
}
cudaError_t band_batch_launch(int cls, const BandArgs* args, const int64_t* prefix, int32_t n, unsigned long long* head,
                              int grid, cudaStream_t s, int prepare_bytes) {
    switch (cls) {
        case 0: return batch_one<kModeShared, true, false>(args, prefix, n, head, grid, s, prepare_bytes);
        case 1: return batch_one<kModeShared, false, false>(args, prefix, n, head, grid, s, prepare_bytes);
        case 2: return batch_one<kModeIndep, true, false>(args, prefix, n, head, grid, s, prepare_bytes);
        case 3: return batch_one<kModeIndep, false, false>(args, prefix, n, head, grid, s, prepare_bytes);
        case 4: return batch_one<kModeGrouped, true, false>(args, prefix, n, head, grid, s, prepare_bytes);
        case 5: return batch_one<kModeGrouped, false, false>(args, prefix, n, head, grid, s, prepare_bytes);
        case 6: return batch_one<kModeShared, false, true>(args, prefix, n, head, grid, s, prepare_bytes);
        case 7: return batch_one<kModeIndep, false, true>(args, prefix, n, head, grid, s, prepare_bytes);
        case 8: return batch_one<kModeGrouped, false, true>(args, prefix, n, head, grid, s, prepare_bytes);
        default: return cudaErrorInvalidValue;
    }
}
}  // namespace
int band_tile_out_w() { return kOutW; }
int band_max_bands() { return kMaxBands; }

template <bool kMadAdd, int kMode, bool kCands, bool kExact = false>
cudaError_t prepare_one(int bytes) {
    return cudaFuncSetAttribute(band_scan_kernel<kMadAdd, kMode, kCands, kExact>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t band_prepare() {
    const int bytes = (int)sizeof(BandSmem);
    cudaError_t e;
    if ((e = prepare_one<false, kModeShared, false>(bytes)) != cudaSuccess || (e = prepare_one<true, kModeShared, false>(bytes)) != cudaSuccess ||
        (e = prepare_one<false, kModeIndep, false>(bytes)) != cudaSuccess || (e = prepare_one<true, kModeIndep, false>(bytes)) != cudaSuccess ||
        (e = prepare_one<false, kModeShared, true>(bytes)) != cudaSuccess || (e = prepare_one<true, kModeShared, true>(bytes)) != cudaSuccess ||
        (e = prepare_one<false, kModeIndep, true>(bytes)) != cudaSuccess || (e = prepare_one<true, kModeIndep, true>(bytes)) != cudaSuccess ||
        (e = prepare_one<true, kModeGrouped, false>(bytes)) != cudaSuccess || (e = prepare_one<true, kModeGrouped, true>(bytes)) != cudaSuccess ||
        (e = prepare_one<true, kModeShared, false, true>(bytes)) != cudaSuccess ||
        (e = prepare_one<true, kModeIndep, false, true>(bytes)) != cudaSuccess ||
        (e = prepare_one<true, kModeGrouped, false, true>(bytes)) != cudaSuccess)
        return e;
    for (int cls = 0; cls < kBandClasses; ++cls)
        if ((e = band_batch_launch(cls, nullptr, nullptr, 0, nullptr, 0, nullptr, bytes)) != cudaSuccess) return e;
    return cudaSuccess;
}

int band_class(const BandArgs& a) {
    if (a.exact) return a.indep ? 7 : a.groups ? 8 : 6;
    const int nc = a.min_size < kCandThreshold ? 0 : 1;
    return (a.indep ? 2 : a.groups ? 4 : 0) + nc;
}

cudaError_t launch_band_batch(const BandArgs* args, const int64_t* prefix, int32_t nsearch,
                              unsigned long long* head, int cls, int grid, cudaStream_t s) {
    return band_batch_launch(cls, args, prefix, nsearch, head, grid, s, 0);
}

cudaError_t launch_band_scan(const BandArgs& a, int grid, cudaStream_t s) {
    const size_t bytes = sizeof(BandSmem);
    if (a.exact) {  // bit-sliced exact counts of every centre (multiply-add band adds)
        if (a.indep) band_scan_kernel<true, kModeIndep, false, true><<<grid, kTpb, bytes, s>>>(a);
        else if (a.groups) band_scan_kernel<true, kModeGrouped, false, true><<<grid, kTpb, bytes, s>>>(a);
        else band_scan_kernel<true, kModeShared, false, true><<<grid, kTpb, bytes, s>>>(a);
        return cudaGetLastError();
    }
    const bool cands = a.min_size < kCandThreshold;
    if (a.groups) {  // grouped bands (multiply-add band adds)
        if (cands) band_scan_kernel<true, kModeGrouped, true><<<grid, kTpb, bytes, s>>>(a);
        else band_scan_kernel<true, kModeGrouped, false><<<grid, kTpb, bytes, s>>>(a);
        return cudaGetLastError();
    }
    const int v = (a.mad_add ? 1 : 0) | (a.indep ? 2 : 0) | (cands ? 4 : 0);
    switch (v) {
        case 0: band_scan_kernel<false, kModeShared, false><<<grid, kTpb, bytes, s>>>(a); break;
        case 1: band_scan_kernel<true, kModeShared, false><<<grid, kTpb, bytes, s>>>(a); break;
        case 2: band_scan_kernel<false, kModeIndep, false><<<grid, kTpb, bytes, s>>>(a); break;
        case 3: band_scan_kernel<true, kModeIndep, false><<<grid, kTpb, bytes, s>>>(a); break;
        case 4: band_scan_kernel<false, kModeShared, true><<<grid, kTpb, bytes, s>>>(a); break;
        case 5: band_scan_kernel<true, kModeShared, true><<<grid, kTpb, bytes, s>>>(a); break;
        case 6: band_scan_kernel<false, kModeIndep, true><<<grid, kTpb, bytes, s>>>(a); break;
        default: band_scan_kernel<true, kModeIndep, true><<<grid, kTpb, bytes, s>>>(a); break;
    }
    return cudaGetLastError();
}

int band_row_words(bool split) { return split ? kRowWordsI : kRowWords; }

cudaError_t launch_band_terms(uint64_t* ct, int32_t col_first, int32_t ncols, uint32_t* rt,
                              int32_t vrows_alloc, int32_t vrows, int32_t nj, int32_t row_first,
                              int64_t row_limit, int64_t row_stride, int64_t seed, bool transposed,
                              bool indep, int32_t groups, cudaStream_t s) {
    // Columns carry no seed; rows carry it. Transposed searches swap which axis is x.
    col_terms_kernel<<<(ncols + 255) / 256, 256, 0, s>>>(ct, col_first, ncols, transposed ? 0 : 1);
    const int64_t ngroups = (nj + kMaxBands - 1) / kMaxBands;
    const int64_t n = ngroups * vrows_alloc * band_row_words(indep || groups > 0);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (groups > 0)
        row_terms_kernel<kModeGrouped><<<blocks, 256, 0, s>>>(rt, vrows_alloc, vrows, nj, row_first, row_limit,
                                                              row_stride, seed, transposed ? 1 : 0, groups);
    else if (indep)
        row_terms_kernel<kModeIndep><<<blocks, 256, 0, s>>>(rt, vrows_alloc, vrows, nj, row_first, row_limit,
                                                            row_stride, seed, transposed ? 1 : 0, 1);
    else
        row_terms_kernel<kModeShared><<<blocks, 256, 0, s>>>(rt, vrows_alloc, vrows, nj, row_first, row_limit,
                                                             row_stride, seed, transposed ? 1 : 0, 1);
    return cudaGetLastError();
}

}  // namespace slime
