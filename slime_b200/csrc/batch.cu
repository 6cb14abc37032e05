// batch.cu -- many searches in one persistent launch of the independent-band kernel.
//
// No reference counterpart: the reference runs one search per call. Searches whose threshold
// the band kernel's byte-lane bound accepts (min_size >= 28) and whose expected site count fits
// the batch's hit pool are tiled together; one launch of band_batch_kernel takes their tiles
// from a device queue, so small and large areas share the GPU with no per-search tail. Term
// tables, rare-chunk scans, filters and fix-ups of all searches are queued on the library stream
// around that launch; ranking and precise scoring then follow per search on the host, exactly as
// for a single search. Every other request runs through the single-search path.
#include <algorithm>
#include <cmath>
#include <vector>

#include "driver.h"
#include "engine.h"

namespace slime {

// P(count >= k) for a 221-cell window of independent p = 0.1 cells: the expected share of
// centres a threshold keeps, used to size a search's hit slice (batches and the server).
double tail_share(int k) {
    static const std::vector<double> tail = [] {  // built once (thread-safe static init)
        std::vector<double> pmf(222, 0.0), t(223, 0.0);
        pmf[0] = std::pow(0.9, 221);
        for (int i = 1; i <= 221; ++i) pmf[i] = pmf[i - 1] * (221 - i + 1) / i * (0.1 / 0.9);
        for (int i = 221; i >= 0; --i) t[i] = t[i + 1] + pmf[i];
        return t;
    }();
    return tail[std::max(0, std::min(222, k))];
}

// Chunks of an area whose first draw is rejected and redrawn into a slime chunk: 104,848 of the
// 2^48 LCG states.
double rare_share() { return 104848.0 / 281474976710656.0; }

namespace {

struct Planned {
    int32_t idx;          // request index
    BandGeom g;
    bool exact;  // bit-sliced exact counts
    int32_t area_x0, area_z0;
    size_t ct_off, rt_off, hit_off, rare_off;
    uint64_t hit_cap;
    uint32_t rare_cap;
};

constexpr uint64_t kHitPoolMax = 48ull << 20;   // Hit records in the batch pool (576 MB)
constexpr uint64_t kHitCapMax = 16ull << 20;    // per search; larger searches run alone

}  // namespace

cudaError_t run_band_items(std::vector<BandArgs>& items, BandArgs* args_dev, int64_t* prefix_dev,
                           unsigned long long* heads_dev, int grid, cudaStream_t s, int64_t* launches) {
    const size_t m = items.size();
    if (m == 0) return cudaSuccess;
    std::stable_sort(items.begin(), items.end(),
                     [](const BandArgs& x, const BandArgs& y) { return band_class(x) < band_class(y); });
    std::vector<int64_t> prefix(m + 1, 0);
    for (size_t i = 0; i < m; ++i) prefix[i + 1] = prefix[i] + (items[i].tile_end - items[i].tile_begin);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(args_dev, items.data(), m * sizeof(BandArgs), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(prefix_dev, prefix.data(), (m + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(heads_dev, 0, kBandClasses * sizeof(unsigned long long), s)) != cudaSuccess)
        return e;
    for (size_t i0 = 0; i0 < m;) {
        const int cls = band_class(items[i0]);
        size_t i1 = i0 + 1;
        while (i1 < m && band_class(items[i1]) == cls) ++i1;
        if ((e = launch_band_batch(args_dev + i0, prefix_dev + i0, (int32_t)(i1 - i0), heads_dev + cls, cls, grid, s)) !=
            cudaSuccess)
            return e;
        if (launches) ++*launches;
        i0 = i1;
    }
    return cudaSuccess;
}

bool Context::collect_band(const SearchSpec& q, int32_t area_x0, int32_t area_z0, const Hit* hits_host,
                           uint64_t n, const int2* rare_dev, uint32_t nrare, unsigned long long* fixed_count_dev,
                           unsigned int* ferr_dev, std::vector<Hit>& best, std::vector<uint32_t>& h) {
    std::fill(h.begin(), h.end(), 0u);
    best.clear();
    best.reserve(n);
    for (uint64_t k = 0; k < n; ++k) {
        const Hit& hit = hits_host[k];
        if (hit.count < 0) continue;  // window holds a rare chunk: fixed below
        ++h[hit.count];
        best.push_back(hit);
    }
    if (!nrare) return true;
    FixArgs f{};
    f.area_x0 = area_x0;
    f.area_z0 = area_z0;
    f.width = 2 * q.rd_max + 1;
    f.height = 2 * q.rd_max + 1;
    f.rd_min_sq = q.rd_min * q.rd_min;
    f.center_x = q.center_x;
    f.center_z = q.center_z;
    f.min_size = q.min_size;
    f.max_size = q.max_size;
    f.fixed = fixed.ptr;
    f.fixed_count = fixed_count_dev;
    f.cap = fixed.count;
    f.error = ferr_dev;
    cudaError_t e;
    uint64_t nf = 0;
    uint32_t ferr = 0;
    if ((e = cudaMemsetAsync(fixed_count_dev, 0, 8, stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(ferr_dev, 0, 4, stream)) != cudaSuccess ||
        (e = launch_fixup(rare_dev, (int32_t)nrare, q.seed, f, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&nf, fixed_count_dev, 8, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&ferr, ferr_dev, 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
        set_error("fixup", e);
        return false;
    }
    ++last_launches;
    if (nf > fixed.count || ferr) { set_error("fixup overflow", cudaErrorUnknown); return false; }
    if (nf) {
        const size_t old = best.size();
        best.resize(old + nf);
        if ((e = cudaMemcpyAsync(best.data() + old, fixed.ptr, nf * sizeof(Hit), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
            set_error("copy", e);
            return false;
        }
        for (size_t k = old; k < best.size(); ++k) ++h[best[k].count];
    }
    return true;
}

int32_t Context::search_batch(const SearchSpec* reqs, int32_t n, ExtChunkResult* results, int64_t* totals) {
    if (n < 0 || (n > 0 && (!reqs || !results || !totals))) {
        set_error_text("batch: invalid arguments");
        return -1;
    }
    if (!ensure_device() || !ensure_band()) return -1;
    last_kernel_ms = 0.0;
    last_launches = 0;
    progress.store(1);
    std::vector<int64_t> res_off((size_t)n + 1, 0);
    for (int32_t i = 0; i < n; ++i) res_off[i + 1] = res_off[i] + std::max<int32_t>(0, reqs[i].max_results);

    // ---- plan ------------------------------------------------------------------------------
    std::vector<Planned> plan;
    std::vector<int32_t> alone;
    size_t ct_total = 0, rt_total = 0, rare_total = 0;
    uint64_t hit_total = 0;
    for (int32_t i = 0; i < n; ++i) {
        const SearchSpec& q = reqs[i];
        totals[i] = -1;
        if (!validate_search(q.rd_max, q.min_size, q.max_size, q.rd_min, q.center_x, q.center_z,
                             results + res_off[i], q.max_results) || (q.biome_flags & ~7) != 0)
            continue;
        // The batch takes what the single search would run on a band engine (whatever the
        // area's size: small areas fill the GPU together); the general scan's searches run alone.
        const int32_t algo = engine_for(q);
        const bool exact = algo_exact(algo);
        const bool band_ok = (q.min_size >= 28 || exact) && engine_override != 1 &&
                             (algo != kAlgoGeneral || q.min_size >= indep_min_threshold);
        if (!band_ok) {
            alone.push_back(i);
            continue;
        }
        Planned p{};
        p.idx = i;
        p.exact = exact;
        const int64_t W = 2 * q.rd_max + 1;
        p.g = band_geometry(W, W, algo == kAlgoGeneral ? kBandIndep : band_mode_of(algo), sm_count);
        p.area_x0 = (int32_t)((int64_t)q.center_x - q.rd_max);
        p.area_z0 = (int32_t)((int64_t)q.center_z - q.rd_max);
        const double centres = (double)W * (double)W;
        const double expect = centres * tail_share(q.min_size);
        p.hit_cap = (uint64_t)std::min<double>((double)kHitCapMax, 2.0 * expect + 65536.0);
        if (expect * 1.5 > (double)kHitCapMax || hit_total + p.hit_cap > kHitPoolMax) {
            alone.push_back(i);
            continue;
        }
        const double halo = (double)(W + 16) * (double)(W + 16);
        p.rare_cap = (uint32_t)std::min<double>(1 << 20, 3.0 * halo * rare_share() + 1024.0);
        p.ct_off = ct_total;
        p.rt_off = rt_total;
        p.hit_off = hit_total;
        p.rare_off = rare_total;
        ct_total += (size_t)p.g.width_u + 16;
        rt_total += (size_t)p.g.ngroups * p.g.vrows_alloc * band_row_words(p.g.indep || p.g.groups > 0);
        hit_total += p.hit_cap;
        rare_total += p.rare_cap;
        plan.push_back(p);
    }
    const int32_t m = (int32_t)plan.size();

    // ---- device work of the batched searches ------------------------------------------------
    std::vector<uint64_t> emitted(m, 0), counts_h((size_t)m * 2, 0);
    std::vector<uint32_t> flags_h((size_t)m * 4, 0);
    std::vector<Hit> hits_h;
    std::vector<uint64_t> hoff((size_t)m + 1, 0);  // first host record of each search's sites
    if (m > 0) {
        cudaError_t e;
        // Per search: [0] overflow, [1] fix-up error, [2] rare count, [3] spare; then emitted
        // and fixed counters (u64).
        if ((e = bt_ct.reserve(ct_total)) != cudaSuccess || (e = bt_rt.reserve(rt_total)) != cudaSuccess ||
            (e = bt_hits.reserve(hit_total)) != cudaSuccess || (e = bt_rare.reserve(rare_total)) != cudaSuccess ||
            (e = bt_flags.reserve((size_t)m * 4)) != cudaSuccess || (e = bt_counts.reserve((size_t)m * 2 + kBandClasses)) != cudaSuccess ||
            (e = bt_args.reserve((size_t)m)) != cudaSuccess || (e = bt_prefix.reserve((size_t)m + 1)) != cudaSuccess ||
            (e = fixed.reserve(1u << 20)) != cudaSuccess) {
            set_error("batch alloc", e);
            return -1;
        }
        std::vector<BandArgs> args(m);
        for (int32_t s = 0; s < m; ++s) {
            const Planned& p = plan[s];
            const SearchSpec& q = reqs[p.idx];
            const BandGeom& g = p.g;
            BandArgs& a = args[s];
            a.ct = bt_ct.ptr + p.ct_off;
            a.ncols = g.width_u + 16;
            a.rt = bt_rt.ptr + p.rt_off;
            a.vrows = g.vrows;
            a.vbase = g.vbase;
            a.ubase = g.ubase;
            a.width_u = g.width_u;
            a.height_v = g.height_v;
            a.j0 = 0;
            a.nb = (int32_t)g.nJ;
            a.u_tiles = (int32_t)g.u_tiles;
            a.v_tiles = (int32_t)g.v_tiles;
            a.band_h = g.band_h;
            a.tile_begin = 0;
            a.tile_end = g.tiles;
            a.min_size = q.min_size;
            a.max_size = q.max_size;
            a.rd_min_sq = q.rd_min * q.rd_min;
            a.area_x0 = p.area_x0;
            a.area_z0 = p.area_z0;
            a.center_x = q.center_x;
            a.center_z = q.center_z;
            a.transposed = g.transposed ? 1 : 0;
            a.out = bt_hits.ptr + p.hit_off;
            a.cap = p.hit_cap;
            a.emitted = bt_counts.ptr + 2 * s;
            a.overflow = bt_flags.ptr + 4 * s;
            a.one = 1u;
            a.mad_add = band_mad_add;
            a.exact = p.exact ? 1 : 0;
            a.poll_limit = wait_polls;
            a.indep = g.indep ? 1 : 0;
            a.groups = g.groups;
            a.row_stride = g.stride;
        }
        if ((e = cudaMemsetAsync(bt_flags.ptr, 0, (size_t)m * 4 * sizeof(unsigned int), stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(bt_counts.ptr, 0, (size_t)m * 2 * sizeof(unsigned long long), stream)) != cudaSuccess) {
            set_error("batch setup", e);
            return -1;
        }
        for (int32_t s = 0; s < m; ++s) {
            const Planned& p = plan[s];
            const SearchSpec& q = reqs[p.idx];
            const BandGeom& g = p.g;
            const int64_t W = 2 * q.rd_max + 1;
            const int32_t col_first = (g.transposed ? p.area_z0 : p.area_x0) - 8;
            const int32_t row_first = (g.transposed ? p.area_x0 : p.area_z0) - 8;
            if ((e = launch_band_terms(bt_ct.ptr + p.ct_off, col_first, (int32_t)(g.width_u + 16), bt_rt.ptr + p.rt_off,
                                       g.vrows_alloc, g.vrows, (int32_t)g.nJ, row_first, g.height_v + 16,
                                       g.stride, q.seed, g.transposed, g.indep, g.groups, stream)) != cudaSuccess ||
                (e = launch_rare_scan(rare_targets.ptr, rare_offsets.ptr, q.seed, p.area_z0 - 8, (int32_t)(W + 16),
                                      p.area_x0 - 8, (int32_t)(W + 16), bt_rare.ptr + p.rare_off, p.rare_cap,
                                      bt_flags.ptr + 4 * s + 2, stream)) != cudaSuccess) {
                set_error("batch terms", e);
                return -1;
            }
            last_launches += 3;
        }
        if (cancel.load()) { progress.store(0); return -1; }
        if ((e = cudaEventRecord(ev_a, stream)) != cudaSuccess ||
            (e = run_band_items(args, bt_args.ptr, bt_prefix.ptr, bt_counts.ptr + 2 * m, sm_count, stream,
                                &last_launches)) != cudaSuccess ||
            (e = cudaEventRecord(ev_b, stream)) != cudaSuccess) {
            set_error("batch scan", e);
            return -1;
        }
        // Rare-chunk counts, then the filter of each search's sites against its rare chunks.
        if ((e = cudaMemcpyAsync(flags_h.data(), bt_flags.ptr, (size_t)m * 4 * sizeof(unsigned int), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(counts_h.data(), bt_counts.ptr, (size_t)m * 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
            set_error("batch scan", e);
            return -1;
        }
        float kms = 0.f;
        cudaEventElapsedTime(&kms, ev_a, ev_b);
        last_kernel_ms += kms;
        for (int32_t s = 0; s < m; ++s) emitted[s] = counts_h[2 * s];  // pairs (emitted, fixed)
        for (int32_t s = 0; s < m; ++s) {
            const uint32_t nrare = flags_h[4 * s + 2];
            if (nrare > plan[s].rare_cap) { set_error("batch: too many rare chunks", cudaErrorMemoryAllocation); return -1; }
            if (flags_h[4 * s] & 4u) { set_error("band engine: row-term copy timed out", cudaErrorLaunchTimeout); return -1; }
            if (emitted[s] && nrare && emitted[s] <= plan[s].hit_cap) {
                if ((e = launch_filter_hits(bt_hits.ptr + plan[s].hit_off, (int64_t)emitted[s], bt_rare.ptr + plan[s].rare_off,
                                            (int32_t)nrare, false, stream)) != cudaSuccess) {
                    set_error("batch filter", e);
                    return -1;
                }
                ++last_launches;
            }
        }
        // Each search's emitted sites, packed on the host (searches whose slice overflowed run alone).
        for (int32_t s = 0; s < m; ++s)
            hoff[s + 1] = hoff[s] + (emitted[s] <= plan[s].hit_cap ? emitted[s] : 0);
        hits_h.resize(hoff[m]);
        for (int32_t s = 0; s < m; ++s)
            if (hoff[s + 1] > hoff[s] &&
                (e = cudaMemcpyAsync(hits_h.data() + hoff[s], bt_hits.ptr + plan[s].hit_off,
                                     (hoff[s + 1] - hoff[s]) * sizeof(Hit), cudaMemcpyDeviceToHost, stream)) != cudaSuccess) {
                set_error("batch copy", e);
                return -1;
            }
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) {
            set_error("batch copy", e);
            return -1;
        }
    }

    // ---- per search: fix-up, histogram, ranking, precise scores ------------------------------
    std::vector<uint32_t> h(kHistBins, 0u);
    for (int32_t s = 0; s < m; ++s) {
        const Planned& p = plan[s];
        const SearchSpec& q = reqs[p.idx];
        if ((flags_h[4 * s] & 1u) || emitted[s] > p.hit_cap) {  // dense strip or full slice: alone
            alone.push_back(p.idx);
            continue;
        }
        std::vector<Hit> best;
        if (!collect_band(q, p.area_x0, p.area_z0, hits_h.data() + hoff[s], emitted[s], bt_rare.ptr + p.rare_off,
                          flags_h[4 * s + 2], bt_counts.ptr + 2 * s + 1, bt_flags.ptr + 4 * s + 1, best, h))
            return -1;
        const int64_t total = finish(q, best, h, results + res_off[p.idx]);
        if (total == kNeedMoreSites) {  // biome exclusion beyond the kept sites: run it alone
            alone.push_back(p.idx);
            continue;
        }
        if (total < 0) return -1;
        totals[p.idx] = total;
        progress.store(1 + (int32_t)(80.0 * (s + 1) / std::max(1, m)));
    }

    // ---- the rest, one by one ----------------------------------------------------------------
    std::sort(alone.begin(), alone.end());
    for (int32_t i : alone) {
        if (cancel.load()) break;
        const double kms = last_kernel_ms;
        const int64_t launches = last_launches;
        const int64_t t = search(reqs[i], results + res_off[i]);
        last_kernel_ms += kms;
        last_launches += launches;
        if (t < 0) return -1;
        totals[i] = t;
    }
    last_algorithm = kAlgoIndep;
    progress.store(90);
    return 0;
}

}  // namespace slime
