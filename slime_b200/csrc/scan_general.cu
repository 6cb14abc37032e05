// scan_general.cu -- the general-purpose scan: any area, any threshold, exact predicate.
//
// Behaviour follows the reference GPU search (SlimeCoreGPU.cu:501-610, 3164-3851): every centre
// of the area whose exact 221-cell count lies in [min_size, max_size] (outside the rd_min disc)
// is kept. Design on B200: a persistent grid walks (x tile, z band) tiles; each warp evaluates
// 32 x-adjacent chunks per ballot and publishes the words of a row into a 32-row shared ring;
// each thread keeps rolling 17x17 square counts for its centre columns (square >= circle and
// square - 68 <= circle), and only square survivors get the exact circle count. Survivors are
// queued per warp and counted lane-parallel (one centre per lane) while their 17 rows are still in
// the ring, so a warp never runs the 17-row count with most lanes idle. Kept centres are
// histogrammed by count and those at or above `emit_min` are appended with one atomic per warp.
#include "engine.h"

namespace slime {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

template <int TPB, int CPT>
struct GeneralTile {
    static constexpr int kWarps = TPB / 32;
    static constexpr int kWords = kWarps * CPT;   // 32-bit words per ring row
    static constexpr int kStride = kWords + 4;    // + zero padding word(s), 16-byte rows
    static constexpr int kInW = kWords * 32;
    static constexpr int kOutW = kInW - 16;
};

__device__ __forceinline__ uint32_t slice17(const uint32_t* row, int word, int lane) {
    return __funnelshift_r(row[word], row[word + 1], lane) & 0x1FFFFu;
}

constexpr int kCandCap = 64;   // per warp: square survivors waiting for their exact count
constexpr int kCandAge = 14;   // rows a survivor may wait: its rows stay in the 32-row ring

// Exact counts of the warp's queued centres (entry = column << 16 | centre row in the tile), one
// per lane, 32 at a time; counts in range are histogrammed, those >= emit_min emitted. The rows
// read are at most kCandAge + 16 behind the newest, so the next row written never overwrites them.
template <int TPB, int CPT>
__device__ __forceinline__ void general_flush(const ScanArgs& a, const uint32_t* ring, unsigned int* hist_s,
                                              const uint32_t* cand, int ncand, int x_base, int z_base, int lane) {
    using T = GeneralTile<TPB, CPT>;
    __syncwarp();
    for (int base = 0; base < ncand; base += 32) {
        bool want = false;
        int exact = 0, col = 0, j = 0;
        if (base + lane < ncand) {
            const uint32_t e = cand[base + lane];
            col = (int)(e >> 16);
            j = (int)(e & 0xFFFFu);
            const int word = col >> 5, bit = col & 31;
#pragma unroll
            for (int i = 0; i < 17; ++i)
                exact += __popc(slice17(ring + ((j + i) & 31) * T::kStride, word, bit) & window_row_mask(i));
            if (exact >= a.min_size && exact <= a.max_size) {
                atomicAdd(&hist_s[exact], 1u);
                want = exact >= a.emit_min;
            }
        }
        const unsigned m = __ballot_sync(kFull, want);
        if (m) {
            const int leader = __ffs(m) - 1;
            unsigned long long pos = 0;
            if (lane == leader) pos = atomicAdd(a.emitted, (unsigned long long)__popc(m));
            pos = __shfl_sync(kFull, pos, leader);
            if (want) {
                const unsigned long long idx = pos + __popc(m & ((1u << lane) - 1u));
                if (idx < a.cap) a.out[idx] = Hit{exact, a.area_x0 + x_base + col, a.area_z0 + z_base + j};
            }
        }
    }
    __syncwarp();
}

template <int TPB, int CPT>
__global__ void __launch_bounds__(TPB) general_scan_kernel(const ScanArgs a) {
    using T = GeneralTile<TPB, CPT>;
    __shared__ __align__(16) uint32_t ring[32 * T::kStride];
    __shared__ unsigned int hist_s[kHistBins];
    __shared__ uint32_t cand_s[T::kWarps][kCandCap];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < kHistBins; i += TPB) hist_s[i] = 0;
    for (int i = tid; i < 32 * (T::kStride - T::kWords); i += TPB)
        ring[(i / (T::kStride - T::kWords)) * T::kStride + T::kWords +
             i % (T::kStride - T::kWords)] = 0;
    __syncthreads();

    const int64_t tiles = (int64_t)a.tiles_x * a.tiles_z;
    const bool no_upper = a.max_size >= 221;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int x_base = (int)(t % a.tiles_x) * T::kOutW;
        const int z_base = a.slab_z0 + (int)(t / a.tiles_x) * a.band_h;
        const int out_w = min(T::kOutW, a.width - x_base);
        const int out_h = min(a.band_h, a.slab_z0 + a.slab_h - z_base);
        const int in_w = out_w + 16, in_h = out_h + 16;
        // Annulus searches: a tile whose centres all lie inside the rd_min disc keeps nothing
        // (block-uniform; the farthest corner decides).
        if (a.rd_min_sq && rect_inside_disc(a.area_x0 + (int64_t)x_base, a.area_x0 + (int64_t)x_base + out_w - 1,
                                            a.area_z0 + (int64_t)z_base, a.area_z0 + (int64_t)z_base + out_h - 1,
                                            a.center_x, a.center_z, a.rd_min_sq))
            continue;

        uint64_t xt[CPT];
        int sq[CPT];
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int col = (warp * CPT + k) * 32 + lane;
            xt[k] = col < in_w ? a.xt[x_base + col] : 0;
            sq[k] = 0;
        }

        uint32_t* cand = cand_s[warp];
        int ncand = 0, first_r = 0;  // warp-uniform: queued survivors, row of the oldest
        for (int r = 0; r < in_h; ++r) {
            const uint64_t zt = a.zt[z_base + r];
            uint32_t words[CPT];
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int col = (warp * CPT + k) * 32 + lane;
                words[k] = __ballot_sync(kFull, col < in_w && slime_from_terms(xt[k], zt));
            }
            uint32_t* row = ring + (r & 31) * T::kStride;
            if (lane == 0) {
#pragma unroll
                for (int k = 0; k < CPT; k += (CPT >= 4 ? 4 : 1)) {
                    if constexpr (CPT >= 4)
                        *reinterpret_cast<uint4*>(row + warp * CPT + k) =
                            make_uint4(words[k], words[k + 1], words[k + 2], words[k + 3]);
                    else
                        row[warp * CPT + k] = words[k];
                }
            }
            __syncthreads();

            if (ncand && r - first_r >= kCandAge) {
                general_flush<TPB, CPT>(a, ring, hist_s, cand, ncand, x_base, z_base, lane);
                ncand = 0;
            }
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int word = warp * CPT + k;
                const int col = word * 32 + lane;
                const bool active = col < out_w;
                if (active) {
                    sq[k] += __popc(slice17(row, word, lane));
                    if (r >= 17) sq[k] -= __popc(slice17(ring + ((r - 17) & 31) * T::kStride, word, lane));
                }
                bool flag = active && r >= 16 && sq[k] >= a.min_size && (no_upper || sq[k] <= a.max_size + 68);
                if (flag && a.rd_min_sq != 0) {
                    const int64_t dx = (int64_t)(a.area_x0 + x_base + col) - a.center_x;
                    const int64_t dz = (int64_t)(a.area_z0 + z_base + r - 16) - a.center_z;
                    flag = dx * dx + dz * dz >= a.rd_min_sq;
                }
                const unsigned m = __ballot_sync(kFull, flag);
                if (m) {
                    if (ncand + __popc(m) > kCandCap) {
                        general_flush<TPB, CPT>(a, ring, hist_s, cand, ncand, x_base, z_base, lane);
                        ncand = 0;
                    }
                    if (ncand == 0) first_r = r;
                    if (flag) cand[ncand + __popc(m & ((1u << lane) - 1u))] = ((uint32_t)col << 16) | (uint32_t)(r - 16);
                    ncand += __popc(m);
                }
            }
        }
        if (ncand) general_flush<TPB, CPT>(a, ring, hist_s, cand, ncand, x_base, z_base, lane);
        __syncthreads();  // the next tile reuses ring slots still read above
    }
    for (int i = tid; i < kHistBins; i += TPB)
        if (hist_s[i]) atomicAdd(&a.hist[i], hist_s[i]);
}

__global__ void terms_kernel(uint64_t* xt, int32_t x0, int32_t nx, uint64_t* zt, int32_t z0,
                             int32_t nz, int64_t seed) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nx) xt[i] = x_term((int32_t)((int64_t)x0 + i));
    if (i < nz) zt[i] = z_term((int32_t)((int64_t)z0 + i)) + (uint64_t)seed;
}

__global__ void predicate_kernel(int64_t seed, const int64_t* x, const int64_t* z, uint8_t* out,
                                 int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = is_slime(seed, x[i], z[i]) ? 1 : 0;
}

constexpr int kWideTpb = 256, kWideCpt = 4;
constexpr int kNarrowTpb = 256, kNarrowCpt = 1;

}  // namespace

int general_out_width(bool narrow) {
    return narrow ? GeneralTile<kNarrowTpb, kNarrowCpt>::kOutW : GeneralTile<kWideTpb, kWideCpt>::kOutW;
}

int general_max_grid(bool narrow) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (narrow)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, general_scan_kernel<kNarrowTpb, kNarrowCpt>, kNarrowTpb, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, general_scan_kernel<kWideTpb, kWideCpt>, kWideTpb, 0);
    return (sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : 1);
}

cudaError_t launch_general_scan(const ScanArgs& a, bool narrow, int grid, cudaStream_t s) {
    if (narrow)
        general_scan_kernel<kNarrowTpb, kNarrowCpt><<<grid, kNarrowTpb, 0, s>>>(a);
    else
        general_scan_kernel<kWideTpb, kWideCpt><<<grid, kWideTpb, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_terms(uint64_t* xt, int32_t x0, int32_t nx, uint64_t* zt, int32_t z0,
                         int32_t nz, int64_t seed, cudaStream_t s) {
    const int32_t n = nx > nz ? nx : nz;
    terms_kernel<<<(n + 255) / 256, 256, 0, s>>>(xt, x0, nx, zt, z0, nz, seed);
    return cudaGetLastError();
}

cudaError_t launch_predicate(int64_t seed, const int64_t* x, const int64_t* z, uint8_t* out,
                             int64_t n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    predicate_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(seed, x, z, out, n);
    return cudaGetLastError();
}

}  // namespace slime
