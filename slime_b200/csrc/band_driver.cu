// band_driver.cu -- host side of the band engine (scan_band.cu) and its redraw correction.
#include <algorithm>
#include <chrono>
#include <thread>
#include <vector>

#include "band_math.cuh"
#include "driver.h"
#include "engine.h"

namespace slime {

namespace {
constexpr int64_t kP = band::kPeriod;
constexpr uint32_t kRareCap = 1u << 20;
}  // namespace

bool Context::ensure_band() {
    if (band_ready) return true;
    cudaError_t e = band_prepare();
    if (e != cudaSuccess) { set_error("band smem", e); return false; }
    std::vector<uint64_t> t;
    std::vector<uint32_t> o;
    rare_target_table(t, o);
    if ((e = rare_targets.reserve(t.size())) != cudaSuccess || (e = rare_offsets.reserve(o.size())) != cudaSuccess ||
        (e = flags.reserve(4)) != cudaSuccess || (e = rare.reserve(kRareCap)) != cudaSuccess ||
        (e = cudaMemcpyAsync(rare_targets.ptr, t.data(), t.size() * 8, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(rare_offsets.ptr, o.data(), o.size() * 4, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
        set_error("rare table", e);
        return false;
    }
    band_ready = true;
    return true;
}

// Engine choice. The band engines need a threshold >= 28 (their byte-lane bound test). The
// shared-LCG band engine wants an area spanning two periods on one axis; the independent-band
// engine wants enough centres to fill the GPU. Below their thresholds the exact counts of the
// many surviving 4x4 groups dominate and the general scan is faster.
int32_t Context::engine_for(const SearchSpec& q) const {
    if (engine_override == 4) return kAlgoBandExact;
    if (engine_override == 5) return kAlgoIndepExact;
    if (engine_override == 7) return kAlgoGroupedExact;
    if (engine_override == 1 || q.min_size < 28) return kAlgoGeneral;
    if (engine_override == 2) return kAlgoBand;
    if (engine_override == 3) return kAlgoIndep;
    if (engine_override == 6) return kAlgoGrouped;
    // The rule's numbers are measured crossovers (slime_b200/autotune.py writes them; the
    // defaults are the B200 values). The shared LCG pays off with many periods (its work is
    // shared by every band and phase pair) and a high threshold.
    const int64_t w = 2 * q.rd_max + 1;
    // Low thresholds: exact counts of every centre, while the sites stay few enough to collect
    // (the band engines emit every site in range; the general scan gates by count on the device).
    constexpr double kExactMaxSites = 1e9;
    const int32_t exact_below =
        w >= kGroupedExactMinPeriods * kP ? std::max(exact_below_threshold, exact_wide_below_threshold) : exact_below_threshold;
    if (q.min_size < exact_below && w * w >= exact_min_centres &&
        (double)w * (double)w * tail_share(q.min_size) <= kExactMaxSites)
        // Exact counts cost the same per centre in every mode; the generator's sharing decides:
        // independent bands on narrow areas, grouped bands from 4 periods (measured on B200:
        // 1.1-1.3 against 1.0 T/s at 4.6-9 periods, 0.9 against 1.0 at 3 periods), the shared
        // LCG on the widest.
        return w >= (int64_t)band_fast_periods * kP ? kAlgoBandExact
               : w >= kGroupedExactMinPeriods * kP && w <= grouped_max_width && w <= kGroupedMaxPeriods * kP
                   ? kAlgoGroupedExact
                   : kAlgoIndepExact;
    // Areas one to several periods wide: X phase pairs with groups of Z period copies.
    if (q.min_size >= grouped_min_threshold && w >= grouped_min_width && w <= grouped_max_width &&
        w <= kGroupedMaxPeriods * kP)
        return kAlgoGrouped;
    if ((q.min_size >= band_min_threshold && w >= (int64_t)band_min_periods * kP) ||
        (q.min_size >= band_fast_threshold && w >= (int64_t)band_fast_periods * kP))
        return kAlgoBand;
    if (w * w >= indep_min_centres && q.min_size >= indep_min_threshold) return kAlgoIndep;
    return kAlgoGeneral;
}

BandGeom band_geometry(int64_t W, int64_t H, int mode, int sm_count) {
    BandGeom g{};
    const bool indep = mode == kBandIndep, grouped = mode == kBandGrouped;
    g.indep = indep;
    g.transposed = mode == kBandShared && W < 2 * kP && H >= 2 * kP;
    g.width_u = g.transposed ? H : W;
    g.height_v = g.transposed ? W : H;
    const int out_w = band_tile_out_w();
    const int nb_max = band_max_bands();
    // Shared LCG: X phases and Z bands 2^17 apart. Independent bands: one phase, nJ bands of
    // `stride` rows each (at least 256 rows a band, at most 32 bands). Grouped bands: X phase
    // pairs and G groups of `copies` bands 2^17 apart (G a power of two, G * copies <= 16), group
    // g starting at row g * stride with G * stride = 2^17 (or the whole height in one copy).
    g.nI = indep ? 1 : (g.width_u + kP - 1) / kP;
    if (grouped) {
        const int64_t copies = std::max<int64_t>(1, (g.height_v + kP - 1) / kP);
        int64_t G = kGroupedMaxBands;
        while (G > 1 && G * copies > kGroupedMaxBands) G >>= 1;
        g.groups = (int32_t)G;
        g.nJ = G * copies;
        g.stride = copies > 1 ? kP / G : (g.height_v + G - 1) / G;
    } else {
        g.nJ = indep ? std::max<int64_t>(1, std::min<int64_t>(nb_max, g.height_v / 256)) : (g.height_v + kP - 1) / kP;
        g.stride = indep ? (g.height_v + g.nJ - 1) / g.nJ : kP;
    }
    g.ubase = (int32_t)(indep ? g.width_u : std::min(kP, g.width_u));
    g.vbase = (int32_t)std::min(g.stride, g.height_v);
    g.vrows = g.vbase + 16;
    g.vrows_alloc = g.vbase + 32;  // zero rows: 8-row bulk copies never run past the end
    g.ngroups = (g.nJ + nb_max - 1) / nb_max;
    g.u_tiles = (g.ubase + out_w - 1) / out_w;
    g.band_h = (int32_t)std::min<int64_t>(2048, std::max<int64_t>(256, g.vbase));
    if (indep) {
        // Enough tiles for two waves of CTAs where the area allows it, tiles of 64+ rows.
        const int64_t want = (2 * (int64_t)sm_count + g.u_tiles - 1) / g.u_tiles;
        const int64_t vt = std::max<int64_t>((g.vbase + 2047) / 2048, std::min<int64_t>((g.vbase + 63) / 64, want));
        g.band_h = (int32_t)((g.vbase + vt - 1) / vt);
    }
    g.v_tiles = (g.vbase + g.band_h - 1) / g.band_h;
    g.pairs = (g.nI + 1) / 2;
    g.tiles = g.u_tiles * g.v_tiles * g.pairs;
    return g;
}

bool Context::scan_band(const SearchSpec& q, std::vector<Hit>& best, std::vector<uint32_t>& h,
                        bool& cancelled, int mode, bool exact) {
    if (!ensure_band()) return false;
    const int64_t W = 2 * q.rd_max + 1, H = W;
    const int32_t area_x0 = (int32_t)((int64_t)q.center_x - q.rd_max);
    const int32_t area_z0 = (int32_t)((int64_t)q.center_z - q.rd_max);
    const BandGeom G = band_geometry(W, H, mode, sm_count);
    const bool indep = G.indep, split = G.indep || G.groups > 0;
    const bool transposed = G.transposed;
    const int64_t width_u = G.width_u, height_v = G.height_v;
    const int nb_max = band_max_bands();
    const int64_t nJ = G.nJ, stride = G.stride;
    const int32_t ubase = G.ubase, vbase = G.vbase, vrows = G.vrows, vrows_alloc = G.vrows_alloc;
    const int64_t ngroups = G.ngroups;
    cudaError_t e;
    if ((e = xt.reserve((size_t)width_u + 16)) != cudaSuccess ||
        (e = rt.reserve((size_t)ngroups * vrows_alloc * band_row_words(split))) != cudaSuccess ||
        (e = counters.reserve(4)) != cudaSuccess ||
        (e = hits.reserve(hit_capacity(q.max_results))) != cudaSuccess ||
        (e = fixed.reserve(1u << 20)) != cudaSuccess) {
        set_error("alloc", e);
        return false;
    }
    const int32_t col_first = (transposed ? area_z0 : area_x0) - 8;
    const int32_t row_first = (transposed ? area_x0 : area_z0) - 8;
    if ((e = launch_band_terms(xt.ptr, col_first, (int32_t)(width_u + 16), rt.ptr, vrows_alloc, vrows,
                               (int32_t)nJ, row_first, height_v + 16, stride, q.seed, transposed, indep, G.groups,
                               stream)) != cudaSuccess) {
        set_error("band terms", e);
        return false;
    }
    last_launches += 2;

    // Rare redraw chunks of the area and its 8-chunk halo, found before the scan so that the
    // scan's hits can be filtered on the device.
    if ((e = cudaMemsetAsync(flags.ptr, 0, 16, stream)) != cudaSuccess ||
        (e = launch_rare_scan(rare_targets.ptr, rare_offsets.ptr, q.seed, area_z0 - 8, (int32_t)(H + 16),
                              area_x0 - 8, (int32_t)(W + 16), rare.ptr, kRareCap, flags.ptr + 2, stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(pinned, flags.ptr + 2, 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
        set_error("rare scan", e);
        return false;
    }
    ++last_launches;
    const uint32_t nrare = *(uint32_t*)pinned;
    if (nrare > kRareCap) { set_error("too many rare chunks", cudaErrorMemoryAllocation); return false; }
    last_rare = nrare;
    // The rare list sorted by x: the hit filter then binary-searches it.
    if (nrare > 1) {
        std::vector<int2> rl(nrare);
        if ((e = cudaMemcpyAsync(rl.data(), rare.ptr, (size_t)nrare * sizeof(int2), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
            set_error("rare list", e);
            return false;
        }
        std::sort(rl.begin(), rl.end(), [](const int2& a, const int2& b) { return a.x != b.x ? a.x < b.x : a.y < b.y; });
        if ((e = cudaMemcpyAsync(rare.ptr, rl.data(), (size_t)nrare * sizeof(int2), cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
            set_error("rare list", e);
            return false;
        }
    }

    const int64_t u_tiles = G.u_tiles, v_tiles = G.v_tiles;
    const int32_t band_h = G.band_h;
    const int grid = sm_count;
    const uint64_t cap = hits.count;
    // Count histogram on the device (first-draw counts of every centre in range, corrected for
    // rare chunks by the fix-up) and an emission gate: only centres whose count reaches emit_min
    // are sent to the host, chosen so that the expected emission stays well inside the buffer but
    // covers max_results several times; if it falls short, the scan runs again with the exact
    // gate the histogram gives.
    if ((e = hist.reserve(2 * kHistBins)) != cudaSuccess) { set_error("alloc", e); return false; }
    unsigned int* dhist = hist.ptr;
    int* ddelta = reinterpret_cast<int*>(hist.ptr + kHistBins);
    const double area = (double)W * (double)H;
    int32_t emit_min = q.min_size;
    while (emit_min < q.max_size && area * tail_share(emit_min) > (double)cap / 8.0 &&
           area * tail_share(emit_min + 1) >= 4.0 * q.max_results)
        ++emit_min;

    for (int pass = 0; pass < 3; ++pass) {
        best.clear();
        std::fill(h.begin(), h.end(), 0u);
        if ((e = cudaMemsetAsync(dhist, 0, 2 * kHistBins * sizeof(unsigned int), stream)) != cudaSuccess) {
            set_error("band histogram", e);
            return false;
        }
        for (int64_t g = 0; g < ngroups; ++g) {
            const int32_t j0 = (int32_t)(g * nb_max);
            const int32_t nb = (int32_t)std::min<int64_t>(nb_max, nJ - j0);
            if (nb <= 0) break;
            const int64_t tiles = G.tiles;
            int64_t chunk = std::max<int64_t>(grid, std::min<int64_t>(tiles, (int64_t)grid * 24));
            for (int64_t t0 = 0; t0 < tiles;) {
                while (paused.load() && !cancel.load()) std::this_thread::sleep_for(std::chrono::milliseconds(20));
                if (cancel.load()) { cancelled = true; return true; }
                const int64_t t1 = std::min(tiles, t0 + chunk);
                BandArgs a{};
                a.ct = xt.ptr;
                a.ncols = width_u + 16;
                a.rt = rt.ptr + (size_t)g * vrows_alloc * band_row_words(split);
                a.vrows = vrows;
                a.vbase = vbase;
                a.ubase = ubase;
                a.width_u = width_u;
                a.height_v = height_v;
                a.j0 = j0;
                a.nb = nb;
                a.u_tiles = (int32_t)u_tiles;
                a.v_tiles = (int32_t)v_tiles;
                a.band_h = band_h;
                a.tile_begin = t0;
                a.tile_end = t1;
                a.min_size = q.min_size;
                a.max_size = q.max_size;
                a.rd_min_sq = q.rd_min * q.rd_min;
                a.area_x0 = area_x0;
                a.area_z0 = area_z0;
                a.center_x = q.center_x;
                a.center_z = q.center_z;
                a.transposed = transposed ? 1 : 0;
                a.out = hits.ptr;
                a.cap = cap;
                a.emitted = counters.ptr;
                a.overflow = flags.ptr;
                a.one = 1u;
                a.mad_add = band_mad_add;
                a.indep = indep ? 1 : 0;
                a.groups = G.groups;
                a.exact = exact ? 1 : 0;
                a.poll_limit = wait_polls;
                a.hist = dhist;
                a.emit_min = emit_min;
                a.row_stride = stride;
                const auto c0 = std::chrono::steady_clock::now();
                // A launch whose hits overflow the buffer is redone in halves: its histogram
                // counts are taken back first (snapshot before, restore after).
                if ((e = cudaMemcpyAsync(ddelta, dhist, kHistBins * sizeof(unsigned int), cudaMemcpyDeviceToDevice,
                                         stream)) != cudaSuccess ||
                    (e = cudaMemsetAsync(counters.ptr, 0, 8, stream)) != cudaSuccess ||
                    (e = cudaEventRecord(ev_a, stream)) != cudaSuccess ||
                    (e = launch_band_scan(a, (int)std::min<int64_t>(grid, t1 - t0), stream)) != cudaSuccess ||
                    (e = cudaEventRecord(ev_b, stream)) != cudaSuccess ||
                    (e = cudaMemcpyAsync(pinned, counters.ptr, 8, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                    (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
                    set_error("band scan", e);
                    return false;
                }
                const auto c1 = std::chrono::steady_clock::now();
                float kms = 0.f;
                cudaEventElapsedTime(&kms, ev_a, ev_b);
                last_kernel_ms += kms;
                ++last_launches;
                const uint64_t emitted = *(unsigned long long*)pinned;
                if (emitted > cap) {
                    if (t1 - t0 <= 1) { set_error("band hit buffer overflow", cudaErrorMemoryAllocation); return false; }
                    if ((e = cudaMemcpyAsync(dhist, ddelta, kHistBins * sizeof(unsigned int), cudaMemcpyDeviceToDevice,
                                             stream)) != cudaSuccess) {
                        set_error("band histogram", e);
                        return false;
                    }
                    chunk = std::max<int64_t>(1, (t1 - t0) / 2);
                    continue;
                }
                work_ns.fetch_add(std::max<int64_t>(1, std::chrono::duration_cast<std::chrono::nanoseconds>(c1 - c0).count()));
                if (emitted) {
                    if ((e = launch_filter_hits(hits.ptr, (int64_t)emitted, rare.ptr, (int32_t)nrare, true, stream)) != cudaSuccess) {
                        set_error("filter", e);
                        return false;
                    }
                    if (nrare) ++last_launches;
                    const size_t old = best.size();
                    best.resize(old + emitted);
                    if ((e = cudaMemcpyAsync(best.data() + old, hits.ptr, emitted * sizeof(Hit), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                        (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
                        set_error("copy", e);
                        return false;
                    }
                    size_t w = old;
                    for (size_t i = old; i < best.size(); ++i)
                        if (best[i].count >= 0) best[w++] = best[i];  // window holds a rare chunk: fixed below
                    best.resize(w);
                    if (best.size() > 2 * (size_t)q.max_results + 1000000) {
                        std::nth_element(best.begin(), best.begin() + q.max_results, best.end(),
                                         [](const Hit& x, const Hit& y) { return hit_order(x, y); });
                        best.resize(q.max_results);
                    }
                }
                const double done = ((double)g * tiles + (double)t1) / ((double)ngroups * tiles);
                processed.store((int64_t)(done * (double)W * (double)H));
                progress.store(1 + (int32_t)(done * 78));
                t0 = t1;
            }
        }

        // Exact counts of every centre whose window holds a rare redraw chunk, and the matching
        // correction of the histogram (first-draw count out, exact count in).
        if ((e = cudaMemsetAsync(ddelta, 0, kHistBins * sizeof(int), stream)) != cudaSuccess) {
            set_error("band histogram", e);
            return false;
        }
        if (nrare) {
            FixArgs f{};
            f.area_x0 = area_x0;
            f.area_z0 = area_z0;
            f.width = W;
            f.height = H;
            f.rd_min_sq = q.rd_min * q.rd_min;
            f.center_x = q.center_x;
            f.center_z = q.center_z;
            f.min_size = q.min_size;
            f.max_size = q.max_size;
            f.fixed = fixed.ptr;
            f.fixed_count = counters.ptr + 1;
            f.cap = fixed.count;
            f.error = flags.ptr + 1;
            f.hist_delta = ddelta;
            if ((e = cudaMemsetAsync(counters.ptr + 1, 0, 8, stream)) != cudaSuccess ||
                (e = launch_fixup(rare.ptr, (int32_t)nrare, q.seed, f, stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(pinned, counters.ptr + 1, 8, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync((char*)pinned + 8, flags.ptr, 8, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
                set_error("fixup", e);
                return false;
            }
            ++last_launches;
            const uint64_t nf = *(unsigned long long*)pinned;
            const uint32_t* fl = (const uint32_t*)((char*)pinned + 8);
            if (nf > fixed.count || fl[1]) { set_error("fixup overflow", cudaErrorUnknown); return false; }
            if (nf) {
                const size_t old = best.size();
                best.resize(old + nf);
                if ((e = cudaMemcpyAsync(best.data() + old, fixed.ptr, nf * sizeof(Hit), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                    (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
                    set_error("copy", e);
                    return false;
                }
            }
        }
        if ((e = cudaMemcpyAsync(pinned, flags.ptr, 4, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync((char*)pinned + 64, dhist, 2 * kHistBins * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                 stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess) {
            set_error("flags", e);
            return false;
        }
        if (*(uint32_t*)pinned & 4u) { set_error("band engine: row-term copy timed out", cudaErrorLaunchTimeout); return false; }
        if ((*(uint32_t*)pinned & 1u) && !exact) {
            // A 4-row strip too dense for the byte-lane box: redo the search with the general scan.
            band_fallbacks++;
            std::fill(h.begin(), h.end(), 0u);
            best.clear();
            return scan_general(q, best, h, cancelled);
        }
        const uint32_t* hs = (const uint32_t*)((const char*)pinned + 64);
        const int32_t* hd = (const int32_t*)(hs + kHistBins);
        for (int i = 0; i < kHistBins; ++i) h[i] = (uint32_t)((int64_t)hs[i] + hd[i]);
        uint64_t total = 0, have = 0;
        for (int c = q.min_size; c <= q.max_size; ++c) {
            total += h[c];
            if (c >= emit_min) have += h[c];
        }
        const uint64_t need = std::min<uint64_t>(total, (uint64_t)q.max_results);
        if (have >= need || emit_min <= q.min_size) return true;
        // Too few sites sent: the exact gate (highest count whose cumulative number covers need).
        uint64_t acc = 0;
        int32_t gate = q.max_size;
        for (int c = q.max_size; c >= q.min_size; --c) {
            acc += h[c];
            gate = c;
            if (acc >= need) break;
        }
        emit_min = gate;
    }
    set_error("band gate did not converge", cudaErrorUnknown);
    return false;
}

}  // namespace slime
