// driver.h -- process-wide state of the C-ABI library (one device, one stream, cached buffers).
#pragma once

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "engine.h"
#include "slime_core.cuh"

namespace slime {

// Device buffer that only grows; freed by cleanup_gpu_resources().
template <typename T>
struct DeviceBuffer {
    T* ptr = nullptr;
    size_t count = 0;
    cudaError_t reserve(size_t n) {
        if (n <= count) return cudaSuccess;
        free();
        const cudaError_t e = cudaMalloc(&ptr, n * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            return e;
        }
        count = n;
        return cudaSuccess;
    }
    void free() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
};

struct SearchSpec {
    int64_t seed;
    int64_t rd_max;
    int32_t min_size;
    int32_t max_size;
    int64_t rd_min;
    int32_t center_x;
    int32_t center_z;
    int32_t max_results;
    int32_t precise_afk;
    // Biome exclusion: bit 0 Deep Dark, bit 1 Mushroom Fields, bit 2 large biomes; 0 = none.
    int32_t biome_flags = 0;
    int32_t biome_version = 0;  // Minecraft version code of the biome tree (e.g. 2602)
};

constexpr int64_t kNeedMoreSites = -3;  // finish(): the biome exclusion needs more ranked sites

// Values reported by get_gpu_v1_algorithm().
constexpr int32_t kAlgoGeneral = 100;
constexpr int32_t kAlgoBand = 200;
constexpr int32_t kAlgoIndep = 300;
// The band engines with bit-sliced exact counts of every centre (low thresholds).
constexpr int32_t kAlgoBandExact = 210;
constexpr int32_t kAlgoIndepExact = 310;
// Grouped bands: X phase pairs and groups of Z period copies (areas one to a few periods wide).
constexpr int32_t kAlgoGrouped = 220;
constexpr int32_t kAlgoGroupedExact = 230;  // grouped bands with bit-sliced exact counts
// Grouped bands hold at most this many bands; the rule uses them up to this width in periods.
constexpr int64_t kGroupedMaxBands = 16;
constexpr int64_t kGroupedMaxPeriods = 16;
constexpr int64_t kGroupedExactMinPeriods = 4;  // exact counts: grouped bands from this width

// Band mode (band_geometry) of a band algorithm.
inline int band_mode_of(int32_t algo) {
    return algo == kAlgoIndep || algo == kAlgoIndepExact                 ? kBandIndep
           : algo == kAlgoGrouped || algo == kAlgoGroupedExact ? kBandGrouped
                                                                : kBandShared;
}
// Band algorithms that count every centre exactly (bit-sliced).
inline bool algo_exact(int32_t algo) {
    return algo == kAlgoBandExact || algo == kAlgoIndepExact || algo == kAlgoGroupedExact;
}

constexpr size_t kPinnedBytes = 1 << 20;

// Result entries the scan may materialise per launch: at least 4M, and 4x the requested top-K.
inline size_t hit_capacity(int32_t max_results) {
    const size_t k = (size_t)(max_results > 0 ? max_results : 1) * 4;
    return k > (4u << 20) ? k : (4u << 20);
}

// Chunk coordinates to the reference's 32-bit block coordinate (wraps like the reference).
inline int32_t block_of(int32_t c) { return (int32_t)((uint32_t)c * 16u + 8u); }

// Ranking order of the reference: size desc, block x asc, block z asc (SlimeCoreGPU.cu:213-220).
inline bool hit_order(const Hit& a, const Hit& b) {
    if (a.count != b.count) return a.count > b.count;
    const int32_t ax = block_of(a.cx), bx = block_of(b.cx);
    if (ax != bx) return ax < bx;
    return block_of(a.cz) < block_of(b.cz);
}

bool validate_search(int64_t rd_max, int32_t min_size, int32_t max_size, int64_t rd_min,
                     int32_t cx, int32_t cz, const void* results, int32_t max_results);

struct Context {
    std::mutex mu;
    int device = -1;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    void* pinned = nullptr;
    // Last error text: a fixed buffer, so that recording an error never allocates.
    char last_error[256] = {};

    DeviceBuffer<uint64_t> xt, zt;
    DeviceBuffer<Hit> hits;
    DeviceBuffer<unsigned long long> counters;
    DeviceBuffer<unsigned int> hist;
    DeviceBuffer<ExtChunkResult> sites;

    // Band engine: packed row terms, the rare redraw table and the correction buffers.
    DeviceBuffer<uint32_t> rt;
    DeviceBuffer<uint64_t> rare_targets;
    DeviceBuffer<uint32_t> rare_offsets;
    DeviceBuffer<int2> rare;
    DeviceBuffer<Hit> fixed;
    DeviceBuffer<unsigned int> flags;  // [0] overflow, [1] fix-up error, [2] rare count

    // Batched searches (batch.cu): pools of all searches of a batch, sliced per search.
    DeviceBuffer<uint64_t> bt_ct;
    DeviceBuffer<uint32_t> bt_rt;
    DeviceBuffer<Hit> bt_hits;
    DeviceBuffer<int2> bt_rare;
    DeviceBuffer<unsigned int> bt_flags;          // per search: overflow, fix-up error, rare count, spare
    DeviceBuffer<unsigned long long> bt_counts;   // per search: emitted, fixed; then the tile queue
    DeviceBuffer<BandArgs> bt_args;
    DeviceBuffer<int64_t> bt_prefix;
    bool band_ready = false;
    // 0 auto, 1 general scan, 2 band engine, 3 independent bands, 4 / 5 the band / independent-band
    // engine with bit-sliced exact counts, 6 / 7 grouped bands (bounded / exact counts).
    int32_t engine_override = 0;
    // Engine rule (engine_for; slime_b200_set_engine_rule): the shared-LCG band engine for areas
    // at least band_min_periods periods wide from band_min_threshold, or band_fast_periods wide
    // from band_fast_threshold; independent bands for areas of indep_min_centres centres or more
    // from indep_min_threshold; the general scan otherwise. Defaults: the rule slime_b200/
    // autotune.py derived on B200 (slime_b200/tuning_b200.json).
    int32_t band_min_threshold = 44;
    int32_t band_min_periods = 15;
    int32_t band_fast_threshold = 44;
    int32_t band_fast_periods = 15;
    int32_t indep_min_threshold = 42;
    int64_t indep_min_centres = 400040001;
    // Below exact_below_threshold, areas of exact_min_centres centres or more use the band engines
    // with bit-sliced exact counts (shared LCG on areas band_fast_periods periods wide, else
    // independent bands), as long as the expected number of sites stays below kExactMaxSites.
    int32_t exact_below_threshold = 45;
    int64_t exact_min_centres = 400040001;
    // Grouped bands for areas grouped_min_width .. grouped_max_width chunks wide (at most
    // kGroupedMaxPeriods periods) from grouped_min_threshold, before the shared-LCG rule.
    int32_t grouped_min_threshold = 46;
    // Areas kGroupedExactMinPeriods periods wide or more use exact counts below this threshold
    // instead (their exact modes share more of the generator's work).
    int32_t exact_wide_below_threshold = 45;
    int64_t grouped_min_width = 200001;
    int64_t grouped_max_width = 2000001;
    int64_t last_rare = 0;             // rare redraw chunks found by the last band search
    int64_t band_fallbacks = 0;        // band searches redone by the general scan
    int32_t band_mad_add = 1;          // generator variant: band adds on the multiply pipe
    uint32_t wait_polls = 1u << 22;    // bounded mbarrier waits of the band kernels

    // Y-scan configuration (set_y_scan_config) and the tables built from it.
    int32_t y_enabled = 0, platform_y = -64, y_min = -64, y_max = 64, y_step = 4;
    bool y_ready = false;
    int32_t y_count = 1;
    DeviceBuffer<int32_t> y_values;
    DeviceBuffer<int16_t> outer, inner;
    DeviceBuffer<uint16_t> weights;

    // Control plane (polled between slabs).
    std::atomic<int> cancel{0}, paused{0}, progress{0};
    std::atomic<int64_t> processed{0}, work_ns{0};
    int32_t last_algorithm = -1, last_shape = 0, rng_override = -1;

    // Statistics of the last search: kernel time measured with CUDA events on the library's
    // stream around every scan launch, and the number of kernels this library launched.
    double last_kernel_ms = 0.0;
    int64_t last_launches = 0;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;

    void set_error(const char* where, cudaError_t e);
    void set_error_text(const char* text);
    bool ensure_device();
    bool ensure_y_tables();
    void release();
    void release_extra();

    bool scan_general(const SearchSpec& q, std::vector<Hit>& best, std::vector<uint32_t>& hist_out,
                      bool& cancelled);
    bool ensure_band();
    int32_t engine_for(const SearchSpec& q) const;
    bool scan_band(const SearchSpec& q, std::vector<Hit>& best, std::vector<uint32_t>& hist_out,
                   bool& cancelled, int mode, bool exact = false);
    bool score(int64_t seed, ExtChunkResult* host, int32_t n, int32_t scan_xz, bool pack);
    int64_t search(const SearchSpec& q, ExtChunkResult* results);
    // Total in range, ranked results and precise scores of a finished scan (-1 on failure). With
    // a biome exclusion the results are the best sites whose window passes the filter; when
    // fewer than max_results pass and `best` misses sites of the area, kNeedMoreSites.
    int64_t finish(const SearchSpec& q, std::vector<Hit>& best, const std::vector<uint32_t>& h,
                   ExtChunkResult* results);
    int64_t finish_biome(const SearchSpec& q, std::vector<Hit>& best, int64_t total, ExtChunkResult* results);
    // Sites examined and excluded by the biome filter in the last search.
    int64_t last_biome_examined = 0, last_biome_excluded = 0;
    // Many searches: those the independent-band kernel can take share one persistent launch.
    int32_t search_batch(const SearchSpec* q, int32_t n, ExtChunkResult* results, int64_t* totals);
    // Sites and histogram of a finished band search from its emitted hits (already filtered
    // against its rare chunks on the device) plus the rare-chunk fix-up.
    bool collect_band(const SearchSpec& q, int32_t area_x0, int32_t area_z0, const Hit* hits_host, uint64_t n,
                      const int2* rare_dev, uint32_t nrare, unsigned long long* fixed_count_dev,
                      unsigned int* ferr_dev, std::vector<Hit>& best, std::vector<uint32_t>& h);
};

Context& ctx();

// Forgets the cached device addresses of the no-alloc search's scratch array (noalloc.cu).
void forget_noalloc_scratch();

// Biome verdict masks (bit 0 Deep Dark, bit 1 Mushroom Fields) of n candidate centre chunks in
// host memory, with a biome context of (world seed, version, large biomes) cached across calls
// (biome.cu). Under the library lock. False on a CUDA failure or an unsupported version.
bool biome_masks(int64_t world_seed, int32_t version, int32_t large, int32_t flags, const int32_t* cx,
                 const int32_t* cz, int64_t n, int32_t* mask);
void release_biome();

// Sizing of per-search slices (batch.cu): the share of centres a threshold keeps in a window of
// independent p = 0.1 cells, and the share of chunks that are rare redraw chunks.
double tail_share(int min_size);
double rare_share();

}  // namespace slime
