// api.cu -- the C ABI of libslime_b200.so (declared in include/slimecore_b200.h).
//
// Host driver of the search: argument checks, per-area term tables, engine choice, slab loop
// with cancel/pause/progress, exact count histogram, top-K ranking and precise scoring. The
// observable behaviour follows search_slime_clusters_gpu_v1_impl (SlimeCoreGPU.cu:3164-3915).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/slimecore_b200.h"
#include "driver.h"
#include "engine.h"

namespace slime {

Context& ctx() {
    static Context c;
    return c;
}

void Context::set_error(const char* where, cudaError_t e) {
    std::snprintf(last_error, sizeof(last_error), "%s: %s", where, cudaGetErrorString(e));
    cudaGetLastError();  // clear a sticky launch error so later calls start clean
}

void Context::set_error_text(const char* text) {
    std::snprintf(last_error, sizeof(last_error), "%s", text);
}

bool Context::ensure_device() {
    if (stream) return true;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0) {
        set_error("no CUDA device", e == cudaSuccess ? cudaErrorNoDevice : e);
        return false;
    }
    if ((e = cudaGetDevice(&device)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess) {
        set_error("stream", e);
        stream = nullptr;
        return false;
    }
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
    if (cudaEventCreate(&ev_a) != cudaSuccess || cudaEventCreate(&ev_b) != cudaSuccess) {
        set_error("events", cudaErrorUnknown);
        return false;
    }
    if (cudaMallocHost(&pinned, kPinnedBytes) != cudaSuccess) {
        pinned = nullptr;
        set_error("pinned", cudaErrorMemoryAllocation);
        return false;
    }
    return true;
}

// Buffers of engines other than the general scan (none yet).
void Context::release_extra() {}

void Context::release() {
    release_biome();
    xt.free();
    zt.free();
    hits.free();
    counters.free();
    hist.free();
    sites.free();
    y_values.free();
    weights.free();
    outer.free();
    inner.free();
    y_ready = false;
    bt_ct.free();
    bt_rt.free();
    bt_hits.free();
    bt_rare.free();
    bt_flags.free();
    bt_counts.free();
    bt_args.free();
    bt_prefix.free();
    release_extra();
    if (pinned) cudaFreeHost(pinned);
    pinned = nullptr;
    if (ev_a) cudaEventDestroy(ev_a);
    if (ev_b) cudaEventDestroy(ev_b);
    ev_a = ev_b = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

// rebuild_gpu_y_tables (SlimeCoreGPU.cu:78-184): Y levels, outer/inner radius per |dx| <= 128,
// and the per-(alignment, chunk, Y) block-column weights used by precise scoring.
bool Context::ensure_y_tables() {
    if (y_ready) return true;
    int32_t y0 = y_enabled ? y_min : platform_y;
    int32_t y1 = y_enabled ? y_max : platform_y;
    int32_t step = y_enabled ? y_step : 1;
    if (step <= 0) step = 1;
    if (y1 < y0) std::swap(y0, y1);
    int32_t count = (y1 - y0) / step + 1;
    if (count <= 0) count = 1;
    std::vector<int32_t> ys(count);
    std::vector<int16_t> out((size_t)count * 257, -1), in((size_t)count * 257, -1);
    auto isqrt = [](int32_t v) {
        int32_t r = 0;
        for (int32_t bit = 1 << 15; bit; bit >>= 1)
            if ((int64_t)(r | bit) * (r | bit) <= v) r |= bit;
        return r;
    };
    for (int32_t yi = 0; yi < count; ++yi) {
        const int32_t y = y0 + yi * step, dy = platform_y - y;
        ys[yi] = y;
        for (int32_t dx = -128; dx <= 128; ++dx) {
            const int32_t o = 16384 - dy * dy - dx * dx, n = 576 - dy * dy - dx * dx;
            if (o >= 0) out[(size_t)yi * 257 + dx + 128] = (int16_t)isqrt(o);
            if (n >= 0) in[(size_t)yi * 257 + dx + 128] = (int16_t)isqrt(n);
        }
    }
    cudaError_t e;
    if ((e = y_values.reserve(count)) != cudaSuccess || (e = outer.reserve(out.size())) != cudaSuccess ||
        (e = inner.reserve(in.size())) != cudaSuccess ||
        (e = weights.reserve((size_t)16 * 16 * 441 * count)) != cudaSuccess) {
        set_error("y tables", e);
        return false;
    }
    if ((e = cudaMemcpyAsync(y_values.ptr, ys.data(), ys.size() * 4, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(outer.ptr, out.data(), out.size() * 2, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(inner.ptr, in.data(), in.size() * 2, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = launch_weight_table(weights.ptr, outer.ptr, inner.ptr, count, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
        set_error("y tables", e);
        return false;
    }
    y_count = count;
    y_ready = true;
    return true;
}

// ---------------------------------------------------------------------------------------------

namespace {

// log P(Binomial(221, 0.1) >= s): the expected share of centres whose count reaches s.
double log_tail(int s) {
    if (s <= 0) return 0.0;
    double acc = -INFINITY;
    for (int k = s; k <= 221; ++k) {
        const double lp = std::lgamma(222.0) - std::lgamma(k + 1.0) - std::lgamma(222.0 - k) +
                          k * std::log(0.1) + (221 - k) * std::log(0.9);
        acc = std::max(acc, lp) + std::log1p(std::exp(-std::fabs(acc - lp)));
    }
    return acc;
}

inline bool hit_better(const Hit& a, const Hit& b) { return hit_order(a, b); }

void keep_best(std::vector<Hit>& v, size_t k) {
    if (v.size() > k) {
        std::nth_element(v.begin(), v.begin() + (ptrdiff_t)k, v.end(), hit_better);
        v.resize(k);
    }
}

}  // namespace

bool validate_search(int64_t rd_max, int32_t min_size, int32_t max_size, int64_t rd_min,
                     int32_t cx, int32_t cz, const void* results, int32_t max_results) {
    // SlimeCoreGPU.cu:3169-3175
    if (!results || max_results <= 0 || rd_max < 0 || rd_max > (INT32_MAX - 19LL) / 2LL ||
        rd_min < 0 || rd_min > rd_max || min_size < 0 || min_size > 221 || max_size < min_size)
        return false;
    if ((int64_t)cx - rd_max - 8LL < INT32_MIN || (int64_t)cx + rd_max + 8LL > INT32_MAX ||
        (int64_t)cz - rd_max - 8LL < INT32_MIN || (int64_t)cz + rd_max + 8LL > INT32_MAX)
        return false;
    return true;
}

// Scans one area with the general engine; fills `best` (<= max_results, unsorted) and `hist`.
bool Context::scan_general(const SearchSpec& q, std::vector<Hit>& best, std::vector<uint32_t>& h,
                           bool& cancelled) {
    const int64_t width = 2 * q.rd_max + 1;
    const int32_t area_x0 = (int32_t)((int64_t)q.center_x - q.rd_max);
    const int32_t area_z0 = (int32_t)((int64_t)q.center_z - q.rd_max);
    const size_t nterms = (size_t)width + 16;
    cudaError_t e;
    if ((e = xt.reserve(nterms)) != cudaSuccess || (e = zt.reserve(nterms)) != cudaSuccess ||
        (e = counters.reserve(4)) != cudaSuccess || (e = hist.reserve(kHistBins)) != cudaSuccess ||
        (e = hits.reserve(hit_capacity(q.max_results))) != cudaSuccess) {
        set_error("alloc", e);
        return false;
    }
    if ((e = launch_terms(xt.ptr, area_x0 - 8, (int32_t)nterms, zt.ptr, area_z0 - 8, (int32_t)nterms,
                          q.seed, stream)) != cudaSuccess) {
        set_error("terms", e);
        return false;
    }
    ++last_launches;
    const bool narrow = width < 8192;
    const int out_w = general_out_width(narrow);
    const int tiles_x = (int)((width + out_w - 1) / out_w);
    const int max_grid = general_max_grid(narrow);
    const int64_t height = width;
    // Enough tiles for ~2 waves of the persistent grid, but bands of at least 64 rows.
    int band_h = (int)std::min<int64_t>(2048, std::max<int64_t>(64, (height * tiles_x) / (2LL * max_grid) + 1));
    const uint64_t cap = hits.count;
    const double area = (double)width * (double)height;

    // Materialise only counts that keep the expected emission well inside the buffer; the exact
    // histogram decides afterwards whether a lower gate is needed (second pass).
    int emit_min = q.min_size;
    while (emit_min < q.max_size && area * std::exp(log_tail(emit_min)) > (double)cap / 8.0 &&
           area * std::exp(log_tail(emit_min + 1)) >= 4.0 * q.max_results)
        ++emit_min;

    for (int pass = 0; pass < 3; ++pass) {
        best.clear();
        std::fill(h.begin(), h.end(), 0u);
        // Rows per launch: ~4e10 centres, and an expected emission of at most cap / 4.
        const double per_row = (double)width * std::exp(log_tail(emit_min));
        int64_t slab = std::min<int64_t>(height, std::max<int64_t>(band_h, (int64_t)(4e10 / width)));
        if (per_row > 0) slab = std::min<int64_t>(slab, std::max<int64_t>(band_h, (int64_t)(cap / 4 / per_row)));
        slab = std::max<int64_t>(band_h, (slab / band_h) * band_h);
        for (int64_t z0 = 0; z0 < height;) {
            while (paused.load() && !cancel.load()) std::this_thread::sleep_for(std::chrono::milliseconds(20));
            if (cancel.load()) { cancelled = true; return true; }
            const int32_t rows = (int32_t)std::min<int64_t>(slab, height - z0);
            ScanArgs a{};
            a.xt = xt.ptr;
            a.zt = zt.ptr;
            a.area_x0 = area_x0;
            a.area_z0 = area_z0;
            a.width = (int32_t)width;
            a.height = (int32_t)height;
            a.slab_z0 = (int32_t)z0;
            a.slab_h = rows;
            a.band_h = band_h;
            a.tiles_x = tiles_x;
            a.tiles_z = (rows + band_h - 1) / band_h;
            a.min_size = q.min_size;
            a.max_size = q.max_size;
            a.emit_min = emit_min;
            a.rd_min_sq = q.rd_min * q.rd_min;
            a.center_x = q.center_x;
            a.center_z = q.center_z;
            a.out = hits.ptr;
            a.cap = cap;
            a.emitted = counters.ptr;
            a.hist = hist.ptr;
            const int64_t tiles = (int64_t)a.tiles_x * a.tiles_z;
            const auto t0 = std::chrono::steady_clock::now();
            // Per-slab counter and histogram: a slab that overflows the buffer is redone in halves
            // and its partial counts must not be kept.
            if ((e = cudaMemsetAsync(counters.ptr, 0, 8, stream)) != cudaSuccess ||
                (e = cudaMemsetAsync(hist.ptr, 0, kHistBins * 4, stream)) != cudaSuccess ||
                (e = cudaEventRecord(ev_a, stream)) != cudaSuccess ||
                (e = launch_general_scan(a, narrow, (int)std::min<int64_t>(tiles, max_grid), stream)) != cudaSuccess ||
                (e = cudaEventRecord(ev_b, stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(pinned, counters.ptr, 8, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync((char*)pinned + 64, hist.ptr, kHistBins * 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
                set_error("scan", e);
                return false;
            }
            const auto t1 = std::chrono::steady_clock::now();
            float kms = 0.f;
            cudaEventElapsedTime(&kms, ev_a, ev_b);
            last_kernel_ms += kms;
            ++last_launches;
            const uint64_t emitted = *(unsigned long long*)pinned;
            if (emitted > cap) {
                if (rows <= band_h) { set_error("result buffer overflow", cudaErrorMemoryAllocation); return false; }
                slab = std::max<int64_t>(band_h, ((rows / 2) / band_h) * band_h);
                continue;
            }
            const uint32_t* slab_hist = (const uint32_t*)((const char*)pinned + 64);
            for (int i = 0; i < kHistBins; ++i) h[i] += slab_hist[i];
            processed.fetch_add((int64_t)rows * width);
            work_ns.fetch_add(std::max<int64_t>(1, std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count()));
            if (emitted) {
                const size_t old = best.size();
                best.resize(old + emitted);
                if ((e = cudaMemcpyAsync(best.data() + old, hits.ptr, emitted * sizeof(Hit),
                                         cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                    (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
                    set_error("copy", e);
                    return false;
                }
                if (best.size() > 2 * (size_t)q.max_results + 1000000) keep_best(best, q.max_results);
            }
            z0 += rows;
            progress.store(1 + (int32_t)((z0 * 79) / std::max<int64_t>(1, height)));
        }
        keep_best(best, q.max_results);
        uint64_t total = 0, have = 0;
        for (int s = q.min_size; s <= q.max_size; ++s) {
            total += h[s];
            if (s >= emit_min) have += h[s];
        }
        const uint64_t need = std::min<uint64_t>(total, (uint64_t)q.max_results);
        if (have >= need || emit_min <= q.min_size) return true;
        // Exact gate for the second pass: the highest score whose cumulative count covers `need`.
        uint64_t acc = 0;
        int gate = q.max_size;
        for (int s = q.max_size; s >= q.min_size; --s) {
            acc += h[s];
            gate = s;
            if (acc >= need) break;
        }
        emit_min = gate;
    }
    set_error("gate did not converge", cudaErrorUnknown);
    return false;
}

bool Context::score(int64_t seed, ExtChunkResult* host, int32_t n, int32_t scan_xz, bool pack) {
    if (n <= 0) return true;
    if (!ensure_y_tables()) return false;
    cudaError_t e;
    if ((e = sites.reserve((size_t)n)) != cudaSuccess) { set_error("alloc", e); return false; }
    PreciseArgs p{};
    p.seed = seed;
    p.sites = sites.ptr;
    p.n = n;
    p.scan_xz = scan_xz;
    // Without a Y scan the table holds exactly one level, the platform Y.
    p.y_count = y_count;
    p.y_values = y_values.ptr;
    p.weights = weights.ptr;
    p.platform_y = platform_y;
    p.pack_y = pack ? 1 : 0;
    if ((e = cudaMemcpyAsync(sites.ptr, host, (size_t)n * sizeof(ExtChunkResult), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = launch_precise(p, stream)) != cudaSuccess || (++last_launches, false) ||
        (e = cudaMemcpyAsync(host, sites.ptr, (size_t)n * sizeof(ExtChunkResult), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
        set_error("precise", e);
        return false;
    }
    return true;
}

int64_t Context::search(const SearchSpec& q, ExtChunkResult* results) {
    if (!validate_search(q.rd_max, q.min_size, q.max_size, q.rd_min, q.center_x, q.center_z, results,
                         q.max_results))
        return -1;
    if (!ensure_device()) return -1;
    progress.store(1);
    last_kernel_ms = 0.0;
    last_launches = 0;
    last_biome_examined = last_biome_excluded = 0;
    std::vector<Hit> best;
    std::vector<uint32_t> h(kHistBins, 0u);
    bool cancelled = false;
    last_rare = 0;
    const int32_t algo = engine_for(q);
    last_algorithm = algo;
    last_shape = algo == kAlgoBand || algo == kAlgoBandExact || algo == kAlgoGrouped || algo == kAlgoGroupedExact ? 3
               : algo == kAlgoIndep || algo == kAlgoIndepExact ? 4
               : (2 * q.rd_max + 1) < 8192 ? 1 : 2;
    // With a biome exclusion the scan keeps more ranked sites than max_results (some fail the
    // filter); when they run out before max_results pass, it runs again keeping four times more.
    SearchSpec qs = q;
    if (q.biome_flags & 3)
        qs.max_results = (int32_t)std::min<int64_t>(INT32_MAX / 8, 2LL * q.max_results + 1024);
    for (;;) {
        const bool exact = algo_exact(algo);
        if (!(algo == kAlgoGeneral ? scan_general(qs, best, h, cancelled)
                                   : scan_band(qs, best, h, cancelled, band_mode_of(algo), exact))) {
            progress.store(0);
            return -1;
        }
        const int64_t total = finish(q, best, h, results);
        if (total == kNeedMoreSites && qs.max_results < INT32_MAX / 8) {
            qs.max_results = (int32_t)std::min<int64_t>(INT32_MAX / 8, 4LL * qs.max_results);
            best.clear();
            std::fill(h.begin(), h.end(), 0u);
            continue;
        }
        if (total < 0) progress.store(0);
        else progress.store(90);
        return total == kNeedMoreSites ? -1 : total;
    }
}

// Biome exclusion after a scan: the ranked sites are filtered in rank order, a few thousand at a
// time, until max_results pass (verdict mask & flags == 0) or the sites run out.
int64_t Context::finish_biome(const SearchSpec& q, std::vector<Hit>& best, int64_t total, ExtChunkResult* results) {
    std::sort(best.begin(), best.end(), hit_better);
    const int32_t flags = q.biome_flags & 3, large = (q.biome_flags >> 2) & 1;
    int32_t kept = 0;
    size_t pos = 0;
    std::vector<int32_t> cx, cz, mask;
    while (kept < q.max_results && pos < best.size()) {
        const size_t m = std::min(best.size() - pos, std::max<size_t>(4096, 2 * (size_t)(q.max_results - kept) + 256));
        cx.resize(m);
        cz.resize(m);
        mask.resize(m);
        for (size_t i = 0; i < m; ++i) {
            cx[i] = best[pos + i].cx;
            cz[i] = best[pos + i].cz;
        }
        if (!biome_masks(q.seed, q.biome_version, large, flags, cx.data(), cz.data(), (int64_t)m, mask.data()))
            return -1;
        for (size_t i = 0; i < m && kept < q.max_results; ++i) {
            ++last_biome_examined;
            if (mask[i] & flags) {
                ++last_biome_excluded;
                continue;
            }
            const Hit& b = best[pos + i];
            ExtChunkResult& r = results[kept++];
            r.size = b.count;
            r.center_x = block_of(b.cx);
            r.center_z = block_of(b.cz);
            r.obs_count = 0;
            r.afk_x = r.center_x;
            r.afk_z = r.center_z;
        }
        pos += m;
    }
    if (kept < q.max_results && (int64_t)best.size() < total) return kNeedMoreSites;
    // Records the exclusion left empty (up to the min(total, max_results) a caller expects)
    // carry size -1.
    for (int64_t i = kept; i < std::min<int64_t>(total, q.max_results); ++i)
        results[i] = ExtChunkResult{-1, 0, 0, 0, 0, 0};
    if (q.precise_afk && !cancel.load() && kept > 0) {
        if (!score(q.seed, results, std::min(kept, 100), 1, y_enabled != 0)) return -1;
    }
    return total;
}

int64_t Context::finish(const SearchSpec& q, std::vector<Hit>& best, const std::vector<uint32_t>& h,
                        ExtChunkResult* results) {
    int64_t total = 0;
    for (int s = q.min_size; s <= q.max_size; ++s) total += h[s];
    if (q.biome_flags & 3) return finish_biome(q, best, total, results);
    if (best.size() > (size_t)q.max_results)
        std::nth_element(best.begin(), best.begin() + q.max_results, best.end(), hit_better);
    const int32_t n = (int32_t)std::min<size_t>(best.size(), (size_t)q.max_results);
    std::sort(best.begin(), best.begin() + n, hit_better);
    for (int32_t i = 0; i < n; ++i) {
        ExtChunkResult& r = results[i];
        r.size = best[i].count;
        r.center_x = block_of(best[i].cx);
        r.center_z = block_of(best[i].cz);
        r.obs_count = 0;
        r.afk_x = r.center_x;
        r.afk_z = r.center_z;
    }
    if (q.precise_afk && !cancel.load() && n > 0) {
        // The search-time refinement covers the best 100 (SlimeCoreGPU.cu:3884).
        if (!score(q.seed, results, std::min(n, 100), 1, y_enabled != 0)) return -1;
    }
    return total;
}

}  // namespace slime

using slime::ctx;

namespace {

int64_t search_entry(int64_t seed, int64_t rd_max, int32_t min_size, int32_t max_size, int64_t rd_min,
                     int32_t cx, int32_t cz, ExtChunkResult* results, int32_t max_results,
                     int32_t precise_afk, int32_t biome_flags = 0, int32_t biome_version = 0) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    slime::SearchSpec q{seed, rd_max, min_size, max_size, rd_min, cx, cz, max_results, precise_afk,
                        biome_flags, biome_version};
    return ctx().search(q, reinterpret_cast<slime::ExtChunkResult*>(results));
}

}  // namespace

extern "C" {

int64_t search_slime_clusters_gpu_v1(int64_t seed, int64_t rd_max, int32_t min_size, int32_t max_size,
                                     int64_t rd_min, ExtChunkResult* results_buffer,
                                     int32_t max_results, int32_t precise_afk) {
    return search_entry(seed, rd_max, min_size, max_size, rd_min, 0, 0, results_buffer, max_results,
                        precise_afk);
}

int64_t search_slime_clusters_gpu_v1_centered(int64_t seed, int64_t rd_max, int32_t min_size,
                                              int32_t max_size, int64_t rd_min, int32_t search_center_x,
                                              int32_t search_center_z, ExtChunkResult* results_buffer,
                                              int32_t max_results, int32_t precise_afk) {
    return search_entry(seed, rd_max, min_size, max_size, rd_min, search_center_x, search_center_z,
                        results_buffer, max_results, precise_afk);
}

int64_t search_slime_clusters_gpu_v34(int64_t seed, int64_t rd_max, int32_t min_size, int32_t max_size,
                                      int64_t rd_min, ExtChunkResult* results_buffer,
                                      int32_t max_results, int32_t precise_afk) {
    return search_slime_clusters_gpu_v1(seed, rd_max, min_size, max_size, rd_min, results_buffer,
                                        max_results, precise_afk);
}

int64_t search_slime_clusters_gpu_v34_centered(int64_t seed, int64_t rd_max, int32_t min_size,
                                               int32_t max_size, int64_t rd_min, int32_t search_center_x,
                                               int32_t search_center_z, ExtChunkResult* results_buffer,
                                               int32_t max_results, int32_t precise_afk) {
    return search_slime_clusters_gpu_v1_centered(seed, rd_max, min_size, max_size, rd_min,
                                                 search_center_x, search_center_z, results_buffer,
                                                 max_results, precise_afk);
}

int64_t slime_b200_search_biome(int64_t seed, int64_t rd_max, int32_t min_size, int32_t max_size,
                                int64_t rd_min, int32_t search_center_x, int32_t search_center_z,
                                ExtChunkResult* results_buffer, int32_t max_results, int32_t precise_afk,
                                int32_t biome_flags, int32_t biome_version) {
    if ((biome_flags & ~7) != 0) return -1;
    return search_entry(seed, rd_max, min_size, max_size, rd_min, search_center_x, search_center_z,
                        results_buffer, max_results, precise_afk, biome_flags, biome_version);
}

void slime_b200_last_biome_stats(int64_t* examined, int64_t* excluded) {
    if (examined) *examined = ctx().last_biome_examined;
    if (excluded) *excluded = ctx().last_biome_excluded;
}

void refine_candidates_y(int64_t seed, ExtChunkResult* results_buffer, int32_t count) {
    if (!results_buffer || count <= 0) return;
    std::lock_guard<std::mutex> lock(ctx().mu);
    if (!ctx().ensure_device()) return;
    ctx().progress.store(90);
    ctx().score(seed, reinterpret_cast<slime::ExtChunkResult*>(results_buffer), count, 1, true);
    ctx().progress.store(99);
}

void score_candidates_precise(int64_t seed, ExtChunkResult* results_buffer, int32_t count,
                              int32_t threads, int32_t scan_xz) {
    (void)threads;
    if (!results_buffer || count <= 0) return;
    std::lock_guard<std::mutex> lock(ctx().mu);
    if (!ctx().ensure_device()) return;
    ctx().progress.store(90);
    ctx().score(seed, reinterpret_cast<slime::ExtChunkResult*>(results_buffer), count, scan_xz,
                ctx().y_enabled != 0);
    ctx().progress.store(99);
}

void set_y_scan_config(int32_t enabled, int32_t platform_y, int32_t y_min, int32_t y_max, int32_t y_step) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    auto& c = ctx();
    const int32_t en = enabled ? 1 : 0, step = y_step > 0 ? y_step : 4;
    if (c.y_enabled == en && c.platform_y == platform_y && c.y_min == y_min && c.y_max == y_max &&
        c.y_step == step)
        return;
    c.y_enabled = en;
    c.platform_y = platform_y;
    c.y_min = y_min;
    c.y_max = y_max;
    c.y_step = step;
    c.y_ready = false;
}

void request_cancel(void) {
    ctx().cancel.store(1);
    ctx().paused.store(0);
}
void request_pause(void) { ctx().paused.store(1); }
void resume_search(void) { ctx().paused.store(0); }
void reset_cancel(void) {
    ctx().cancel.store(0);
    ctx().paused.store(0);
    ctx().progress.store(0);
    ctx().processed.store(0);
    ctx().work_ns.store(0);
}
int32_t get_progress(void) { return ctx().progress.load(); }
int64_t get_processed_centers(void) { return ctx().processed.load(); }
int64_t get_gpu_scan_work_ns(void) { return ctx().work_ns.load(); }

int32_t get_cuda_device_count(void) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return count;
}

int32_t get_cuda_device_name(char* buffer, int32_t buffer_size) {
    if (!buffer || buffer_size <= 1) return 0;
    int dev = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        buffer[0] = '\0';
        return 0;
    }
    const size_t n = std::min((size_t)buffer_size - 1, std::strlen(prop.name));
    std::memcpy(buffer, prop.name, n);
    buffer[n] = '\0';
    return (int32_t)n;
}

int32_t get_gpu_v1_shape(void) { return ctx().last_shape; }
int32_t get_gpu_v1_algorithm(void) { return ctx().last_algorithm; }
int32_t get_gpu_v1_rng(void) { return 0; }
void set_gpu_v1_rng_override(int32_t value) { ctx().rng_override = (value >= 0 && value <= 2) ? value : -1; }
int32_t get_gpu_v34_shape(void) { return get_gpu_v1_shape(); }
int32_t get_gpu_v34_rng(void) { return get_gpu_v1_rng(); }
void set_gpu_v34_rng_override(int32_t value) { set_gpu_v1_rng_override(value); }

void cleanup_gpu_resources(void) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    ctx().release();
    slime::forget_noalloc_scratch();
}

bool is_slime_chunk_c(int64_t seed, int64_t cx, int64_t cz) { return slime::is_slime(seed, cx, cz); }

const char* slime_b200_version(void) { return "slime_b200 0.1 (sm_100a)"; }

void slime_b200_last_search_stats(double* kernel_ms, int64_t* launches) {
    if (kernel_ms) *kernel_ms = ctx().last_kernel_ms;
    if (launches) *launches = ctx().last_launches;
}

int64_t slime_b200_last_rare_chunks(void) { return ctx().last_rare; }

void slime_b200_set_tuning(int32_t band_mad_add) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    ctx().band_mad_add = band_mad_add ? 1 : 0;
}

int64_t slime_b200_set_wait_limit(int64_t polls) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    const int64_t before = ctx().wait_polls;
    ctx().wait_polls = polls < 0 ? (1u << 22) : (uint32_t)std::min<int64_t>(polls, UINT32_MAX);
    return before;
}

void slime_b200_set_engine(int32_t mode, int32_t band_min_threshold) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    ctx().engine_override = (mode >= 0 && mode <= 7) ? mode : 0;
    if (band_min_threshold >= 28 && band_min_threshold <= 221) ctx().band_min_threshold = band_min_threshold;
}

const char* slime_b200_last_error(void) { return ctx().last_error; }

int32_t slime_b200_set_engine_rule(const int64_t* rule, int32_t n) {
    if (!rule || (n != 6 && n != 8 && n != 12)) return -1;
    const int64_t bt = rule[0], bp = rule[1], ft = rule[2], fp = rule[3], it = rule[4], ic = rule[5];
    const int64_t et = n >= 8 ? rule[6] : ctx().exact_below_threshold, ec = n >= 8 ? rule[7] : ctx().exact_min_centres;
    const int64_t gt = n == 12 ? rule[8] : ctx().grouped_min_threshold;
    const int64_t gw = n == 12 ? rule[9] : ctx().grouped_min_width, gx = n == 12 ? rule[10] : ctx().grouped_max_width;
    const int64_t ew = n == 12 ? rule[11] : ctx().exact_wide_below_threshold;
    if (bt < 28 || bt > 222 || ft < 28 || ft > 222 || it < 28 || it > 222 || bp < 2 || bp > 64 ||
        fp < 2 || fp > 64 || ic < 0 || et < 0 || et > 222 || ec < 0 || gt < 28 || gt > 222 || gw < 0 || gx < 0 || ew < 0 || ew > 222)
        return -1;
    std::lock_guard<std::mutex> lock(ctx().mu);
    slime::Context& c = ctx();
    c.band_min_threshold = (int32_t)bt;
    c.band_min_periods = (int32_t)bp;
    c.band_fast_threshold = (int32_t)ft;
    c.band_fast_periods = (int32_t)fp;
    c.indep_min_threshold = (int32_t)it;
    c.indep_min_centres = ic;
    c.exact_below_threshold = (int32_t)et;
    c.exact_min_centres = ec;
    c.grouped_min_threshold = (int32_t)gt;
    c.grouped_min_width = gw;
    c.grouped_max_width = gx;
    c.exact_wide_below_threshold = (int32_t)ew;
    return 0;
}

int32_t slime_b200_get_engine_rule(int64_t* rule, int32_t n) {
    if (!rule || (n != 6 && n != 8 && n != 12)) return -1;
    std::lock_guard<std::mutex> lock(ctx().mu);
    const slime::Context& c = ctx();
    rule[0] = c.band_min_threshold;
    rule[1] = c.band_min_periods;
    rule[2] = c.band_fast_threshold;
    rule[3] = c.band_fast_periods;
    rule[4] = c.indep_min_threshold;
    rule[5] = c.indep_min_centres;
    if (n >= 8) {
        rule[6] = c.exact_below_threshold;
        rule[7] = c.exact_min_centres;
    }
    if (n == 12) {
        rule[8] = c.grouped_min_threshold;
        rule[9] = c.grouped_min_width;
        rule[10] = c.grouped_max_width;
        rule[11] = c.exact_wide_below_threshold;
    }
    return 0;
}

int32_t slime_b200_search_batch(const SlimeBatchRequest* requests, int32_t n, ExtChunkResult* results,
                                int64_t* totals) {
    std::lock_guard<std::mutex> lock(ctx().mu);
    if (n < 0 || (n > 0 && (!requests || !results || !totals))) return -1;
    std::vector<slime::SearchSpec> q((size_t)n);
    for (int32_t i = 0; i < n; ++i) {
        const SlimeBatchRequest& r = requests[i];
        q[i] = slime::SearchSpec{r.seed, r.rd_max, r.min_size, r.max_size, r.rd_min, r.center_x, r.center_z,
                                 r.max_results, r.precise_afk, r.biome_flags, r.biome_version};
    }
    return ctx().search_batch(q.data(), n, reinterpret_cast<slime::ExtChunkResult*>(results), totals);
}

int32_t slime_b200_is_slime_batch(int64_t seed, const int64_t* x, const int64_t* z, uint8_t* out, int64_t n) {
    if (n <= 0) return 0;
    if (!x || !z || !out) return -1;
    std::lock_guard<std::mutex> lock(ctx().mu);
    auto& c = ctx();
    if (!c.ensure_device()) return -1;
    int64_t* dx = nullptr;
    int64_t* dz = nullptr;
    uint8_t* dout = nullptr;
    cudaError_t e;
    if ((e = cudaMallocAsync(&dx, n * 8, c.stream)) != cudaSuccess ||
        (e = cudaMallocAsync(&dz, n * 8, c.stream)) != cudaSuccess ||
        (e = cudaMallocAsync(&dout, n, c.stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dx, x, n * 8, cudaMemcpyHostToDevice, c.stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dz, z, n * 8, cudaMemcpyHostToDevice, c.stream)) != cudaSuccess ||
        (e = slime::launch_predicate(seed, dx, dz, dout, n, c.stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(out, dout, n, cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c.stream)) != cudaSuccess) {
        c.set_error("predicate", e);
    }
    if (dx) cudaFreeAsync(dx, c.stream);
    if (dz) cudaFreeAsync(dz, c.stream);
    if (dout) cudaFreeAsync(dout, c.stream);
    cudaStreamSynchronize(c.stream);
    return e == cudaSuccess ? 0 : -1;
}

}  // extern "C"
