// noalloc.cu -- a search entry point that allocates nothing.
//
// Some callers cannot allocate device memory while they run a search: an application that hands
// all GPU memory to its own pool or caching allocator up front (so a driver allocation could
// fail or fragment that pool), a long-running service that must not pay cudaMalloc's implicit
// device synchronisation on its request path, or a program with a fixed memory budget checked at
// start-up. For them, slime_b200_search_noalloc() runs the general scan out of one fixed scratch
// array that is part of the loaded library (every GPU that loads the library holds it until the
// process exits), and it calls no cudaMalloc, cudaFree, cudaMallocHost or host heap allocation.
//
// Limits: search radius <= kMaxRadius chunks, max_results <= kMaxResults. Larger requests are
// rejected with -1 and an error text (slime_b200_last_error). No precise AFK scoring. A call also
// fails with -1 in the unlikely case that a single 64-row band emits more than kHitCap centres at
// or above its gate (the gate is the exact count the histogram pass chose for max_results).
//
// Calls hold the library lock for their whole duration, like every other entry point, so error
// texts (a fixed buffer of the library) are written without racing another thread's search.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/slimecore_b200.h"
#include "driver.h"
#include "engine.h"

namespace slime {
namespace {

constexpr int64_t kMaxRadius = 8191;                         // width <= 16,383 centres
constexpr int32_t kMaxResults = 65536;
constexpr size_t kTermBytes = (2 * kMaxRadius + 1 + 16) * sizeof(uint64_t);
constexpr size_t kScratchBytes = 4u << 20;                   // 4 MiB per device
constexpr size_t kHitsOffset = 2 * kTermBytes + 1024;        // after xt, zt, counters, histogram
constexpr uint64_t kHitCap = (kScratchBytes - kHitsOffset) / sizeof(Hit);
constexpr int kMaxDevices = 64;
constexpr int kCopyChunk = 2048;                             // hits copied back per memcpy

// The scratch array. In host code this name is only a host-side stand-in for the device
// symbol, never a device address: the kernels get the address from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Device address of g_scratch per device ordinal, looked up once (under the library lock).
// cleanup_gpu_resources() forgets them; a device reset by the caller unloads the module, so a
// caller that resets a device must call cleanup_gpu_resources() before the next search here.
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Set-up, once per device, with that device current: the device address of g_scratch.
bool scratch_for_current_device(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        ctx().set_error("no-alloc search: device", e == cudaSuccess ? cudaErrorInvalidDevice : e);
        return false;
    }
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            ctx().set_error("no-alloc search: cudaGetSymbolAddress", e == cudaSuccess ? cudaErrorUnknown : e);
            return false;
        }
        g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[dev];
    return true;
}

// Ranking order of the reference (size desc, block x asc, block z asc). As a heap comparator it
// keeps the worst kept result on top.
bool ranks_before(const ExtChunkResult& a, const ExtChunkResult& b) {
    if (a.size != b.size) return a.size > b.size;
    if (a.center_x != b.center_x) return a.center_x < b.center_x;
    return a.center_z < b.center_z;
}

}  // namespace

void forget_noalloc_scratch() {
    for (auto& p : g_scratch_ptr) p = nullptr;
}

int64_t search_noalloc(int64_t seed, int64_t rd_max, int32_t min_size, int32_t max_size,
                       int64_t rd_min, int32_t cx, int32_t cz, ExtChunkResult* results,
                       int32_t max_results) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    if (!validate_search(rd_max, min_size, max_size, rd_min, cx, cz, results, max_results)) return -1;
    if (rd_max > kMaxRadius || max_results > kMaxResults) {
        ctx().set_error_text("no-alloc search: radius above 8191 chunks or max_results above 65536 "
                             "(the fixed 4 MiB scratch array does not hold larger searches)");
        return -1;
    }
    unsigned char* base = nullptr;
    if (!scratch_for_current_device(&base)) return -1;
    const int64_t width = 2 * rd_max + 1, height = width;
    uint64_t* xt = reinterpret_cast<uint64_t*>(base);
    uint64_t* zt = reinterpret_cast<uint64_t*>(base + kTermBytes);
    unsigned long long* emitted = reinterpret_cast<unsigned long long*>(base + 2 * kTermBytes);
    unsigned int* hist = reinterpret_cast<unsigned int*>(base + 2 * kTermBytes + 64);
    Hit* hits = reinterpret_cast<Hit*>(base + kHitsOffset);
    const int32_t x0 = (int32_t)((int64_t)cx - rd_max), z0 = (int32_t)((int64_t)cz - rd_max);
    cudaStream_t s = 0;  // the legacy default stream: creating a stream is avoided too
    cudaError_t e = launch_terms(xt, x0 - 8, (int32_t)(width + 16), zt, z0 - 8, (int32_t)(width + 16), seed, s);
    if (e != cudaSuccess) { ctx().set_error("no-alloc search: terms", e); return -1; }

    const bool narrow = width < 8192;
    const int out_w = general_out_width(narrow);
    const int tiles_x = (int)((width + out_w - 1) / out_w);
    const int max_grid = general_max_grid(narrow);
    const int band_h = 64;
    const int32_t tiles_z_all = (int32_t)((height + band_h - 1) / band_h);

    auto run = [&](int32_t emit_min, int32_t slab_z0, int32_t slab_h, uint64_t* n_emitted,
                   uint32_t* hist_out) -> bool {
        ScanArgs a{};
        a.xt = xt;
        a.zt = zt;
        a.area_x0 = x0;
        a.area_z0 = z0;
        a.width = (int32_t)width;
        a.height = (int32_t)height;
        a.slab_z0 = slab_z0;
        a.slab_h = slab_h;
        a.band_h = band_h;
        a.tiles_x = tiles_x;
        a.tiles_z = (slab_h + band_h - 1) / band_h;
        a.min_size = min_size;
        a.max_size = max_size;
        a.emit_min = emit_min;
        a.rd_min_sq = rd_min * rd_min;
        a.center_x = cx;
        a.center_z = cz;
        a.out = hits;
        a.cap = kHitCap;
        a.emitted = emitted;
        a.hist = hist;
        const int64_t tiles = (int64_t)a.tiles_x * a.tiles_z;
        unsigned long long n = 0;
        // Counter and histogram keep the previous call's contents: clear them first.
        if ((e = cudaMemsetAsync(emitted, 0, 8, s)) != cudaSuccess ||
            (e = cudaMemsetAsync(hist, 0, kHistBins * 4, s)) != cudaSuccess ||
            (e = launch_general_scan(a, narrow, (int)std::min<int64_t>(tiles, max_grid), s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(&n, emitted, 8, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
            (hist_out && (e = cudaMemcpyAsync(hist_out, hist, kHistBins * 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess) ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess) {
            ctx().set_error("no-alloc search: scan", e);
            return false;
        }
        *n_emitted = n;
        return true;
    };

    // Pass 1: the exact count histogram of the whole area (nothing emitted).
    uint32_t h[kHistBins];
    uint64_t none = 0;
    if (!run(222, 0, (int32_t)height, &none, h)) return -1;
    uint64_t total = 0;
    for (int i = min_size; i <= max_size; ++i) total += h[i];
    const uint64_t need = std::min<uint64_t>(total, (uint64_t)max_results);
    if (need == 0) return (int64_t)total;
    // Gate: the highest count whose cumulative number of centres covers `need`.
    int32_t gate = max_size;
    for (uint64_t acc = 0; gate >= min_size; --gate) {
        acc += h[gate];
        if (acc >= need) break;
    }

    // Pass 2: emit centres with count >= gate slab by slab (a slab that overflows the scratch
    // hit list is split), keeping the best `need` in a heap inside the caller's buffer.
    int32_t kept = 0;
    for (int32_t tz = 0; tz < tiles_z_all;) {
        int32_t bands = tiles_z_all - tz;
        uint64_t n = 0;
        for (;;) {
            const int32_t rows = (int32_t)std::min<int64_t>((int64_t)bands * band_h, height - (int64_t)tz * band_h);
            if (!run(gate, tz * band_h, rows, &n, nullptr)) return -1;
            if (n <= kHitCap) break;
            if (bands == 1) {
                ctx().set_error_text("no-alloc search: one 64-row band overflows the scratch hit list");
                return -1;
            }
            bands = (bands + 1) / 2;
        }
        Hit chunk[kCopyChunk];
        for (uint64_t off = 0; off < n; off += kCopyChunk) {
            const uint64_t m = std::min<uint64_t>(kCopyChunk, n - off);
            if ((e = cudaMemcpy(chunk, hits + off, m * sizeof(Hit), cudaMemcpyDeviceToHost)) != cudaSuccess) {
                ctx().set_error("no-alloc search: copy", e);
                return -1;
            }
            for (uint64_t i = 0; i < m; ++i) {
                ExtChunkResult r{chunk[i].count, block_of(chunk[i].cx), block_of(chunk[i].cz), 0, 0, 0};
                r.afk_x = r.center_x;
                r.afk_z = r.center_z;
                if (kept < (int32_t)need) {
                    results[kept++] = r;
                    std::push_heap(results, results + kept, ranks_before);
                } else if (ranks_before(r, results[0])) {
                    std::pop_heap(results, results + kept, ranks_before);
                    results[kept - 1] = r;
                    std::push_heap(results, results + kept, ranks_before);
                }
            }
        }
        tz += bands;
    }
    std::sort_heap(results, results + kept, ranks_before);
    return (int64_t)total;
}

}  // namespace slime

extern "C" int64_t slime_b200_search_noalloc(int64_t seed, int64_t rd_max, int32_t min_size,
                                             int32_t max_size, int64_t rd_min,
                                             int32_t search_center_x, int32_t search_center_z,
                                             ExtChunkResult* results_buffer, int32_t max_results) {
    return slime::search_noalloc(seed, rd_max, min_size, max_size, rd_min, search_center_x,
                                 search_center_z, reinterpret_cast<slime::ExtChunkResult*>(results_buffer),
                                 max_results);
}
