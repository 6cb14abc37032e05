// server.cu -- a search server over the batched band kernel: continuous batching with
// memory-gated admission. No reference counterpart (the reference serves one blocking call at a
// time).
//
// Clients submit requests (the arguments of one search) and get a ticket; a worker thread runs
// steps. Each step admits queued requests in arrival order while their device memory fits the
// budget, starts the admitted ones (term tables, rare-chunk scan), then launches the persistent
// batch kernel over a quantum of tiles of every admitted band search. A search whose last tile
// ran is finished (filter, fix-up, ranking, precise scores) and released, so small requests
// complete while large ones are still in flight, and new arrivals join the next step. Requests
// the single search would send to the general scan (thresholds below the band engines' range)
// run whole inside a step. Results are exactly those of the single search.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <vector>

#include "../../include/slimecore_b200.h"
#include "driver.h"
#include "engine.h"

namespace slime {
namespace {

using Clock = std::chrono::steady_clock;

enum : int32_t { kQueued = 0, kRunning = 1, kDone = 2, kFailed = -1, kUnknown = -2 };

struct Job {
    int64_t ticket = 0;
    SearchSpec q{};
    int32_t state = kQueued;
    bool band = false;        // runs in the batch kernel (else: the single search, whole)
    bool exact = false;       // band work with bit-sliced exact counts
    bool started = false;
    Clock::time_point t_submit, t_done;
    int64_t total = -1;
    std::vector<ExtChunkResult> results;
    // Band work: geometry, capacities and one device block holding all of the job's buffers.
    BandGeom g{};
    int32_t area_x0 = 0, area_z0 = 0;
    uint64_t hit_cap = 0;
    uint32_t rare_cap = 0;
    size_t bytes = 0;
    int64_t next_tile = 0;
    void* mem = nullptr;
    uint64_t* ct = nullptr;
    uint32_t* rt = nullptr;
    Hit* hits = nullptr;
    int2* rare = nullptr;
    unsigned int* flags = nullptr;            // overflow, fix-up error, rare count, spare
    unsigned long long* counts = nullptr;     // emitted, fixed
    // Count histogram of every centre in range and its rare-chunk correction (2 x kHistBins), and
    // the emission gate: only centres from emit_min on are written to the hit slice.
    unsigned int* hist = nullptr;
    int32_t emit_min = 0;
};

constexpr uint64_t kServerHitCap = 16u << 20;  // hit records of one job's slice at most

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace

struct Server {
    int64_t budget = 0;       // device bytes for admitted jobs
    int32_t tiles_per_step = 0;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    std::deque<Job*> queued;
    std::vector<Job*> active;
    std::map<int64_t, std::unique_ptr<Job>> jobs;
    int64_t next_ticket = 0;
    int64_t used = 0;
    bool stop = false;
    std::thread worker;
    DeviceBuffer<BandArgs> args;
    DeviceBuffer<int64_t> prefix;
    DeviceBuffer<unsigned long long> head;

    void run();
    bool step(std::vector<Job*>& live);
    void complete(Job* j, int64_t total, bool ok);
    bool start(Job* j);
    // 1 finished, 0 failed, 2 to be rescanned with a lower emission gate.
    int finish_band(Job* j);
};

namespace {

// Device bytes a request holds while admitted.
void plan_job(Job& j, const Context& c) {
    const SearchSpec& q = j.q;
    const int64_t W = 2 * q.rd_max + 1;
    const int32_t algo = c.engine_for(q);
    const double centres = (double)W * (double)W;
    // Emission gate, as the single search chooses it: the smallest count whose expected number of
    // centres fits an eighth of the largest slice while still covering the ranked results
    // (biome requests keep more, as the single search does) four times over.
    const int64_t want = (q.biome_flags & 3) ? 2LL * q.max_results + 1024 : (int64_t)q.max_results;
    int32_t emit = q.min_size;
    while (emit < q.max_size && centres * tail_share(emit) > (double)kServerHitCap / 8.0 &&
           centres * tail_share(emit + 1) >= 4.0 * (double)want)
        ++emit;
    j.emit_min = emit;
    const double expect = centres * tail_share(emit);
    j.exact = algo_exact(algo);
    j.band = (q.min_size >= 28 || j.exact) && algo != kAlgoGeneral && expect * 1.5 < (double)kServerHitCap;
    if (!j.band) {
        // The single search's term tables and hit buffer (library buffers, counted for gating).
        j.bytes = (size_t)(W + 16) * 16 + hit_capacity(q.max_results) * sizeof(Hit);
        return;
    }
    j.g = band_geometry(W, W, band_mode_of(algo), c.sm_count);
    j.area_x0 = (int32_t)((int64_t)q.center_x - q.rd_max);
    j.area_z0 = (int32_t)((int64_t)q.center_z - q.rd_max);
    j.hit_cap = (uint64_t)std::min<double>((double)(16u << 20), 2.0 * expect + 65536.0);
    const double halo = (double)(W + 16) * (double)(W + 16);
    j.rare_cap = (uint32_t)std::min<double>(1 << 20, 3.0 * halo * rare_share() + 1024.0);
    j.bytes = align256((size_t)(j.g.width_u + 16) * 8) +
              align256((size_t)j.g.ngroups * j.g.vrows_alloc * band_row_words(j.g.indep || j.g.groups > 0) * 4) +
              align256((size_t)j.hit_cap * sizeof(Hit)) + align256((size_t)j.rare_cap * sizeof(int2)) +
              align256(2 * kHistBins * sizeof(unsigned int)) + 256;
}

}  // namespace

void Server::complete(Job* j, int64_t total, bool ok) {
    if (j->mem) cudaFreeAsync(j->mem, ctx().stream);
    j->mem = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    j->total = total;
    j->state = ok ? kDone : kFailed;
    j->t_done = Clock::now();
    used -= (int64_t)j->bytes;
    active.erase(std::remove(active.begin(), active.end(), j), active.end());
    done_cv.notify_all();
}

bool Server::start(Job* j) {
    Context& c = ctx();
    cudaError_t e = cudaMallocAsync(&j->mem, j->bytes, c.stream);
    if (e != cudaSuccess) { c.set_error("server alloc", e); j->mem = nullptr; return false; }
    char* p = (char*)j->mem;
    j->ct = (uint64_t*)p; p += align256((size_t)(j->g.width_u + 16) * 8);
    j->rt = (uint32_t*)p; p += align256((size_t)j->g.ngroups * j->g.vrows_alloc * band_row_words(j->g.indep || j->g.groups > 0) * 4);
    j->hits = (Hit*)p; p += align256((size_t)j->hit_cap * sizeof(Hit));
    j->rare = (int2*)p; p += align256((size_t)j->rare_cap * sizeof(int2));
    j->hist = (unsigned int*)p; p += align256(2 * kHistBins * sizeof(unsigned int));
    j->flags = (unsigned int*)p;
    j->counts = (unsigned long long*)(p + 32);
    const SearchSpec& q = j->q;
    const BandGeom& g = j->g;
    const int64_t W = 2 * q.rd_max + 1;
    const int32_t col_first = (g.transposed ? j->area_z0 : j->area_x0) - 8;
    const int32_t row_first = (g.transposed ? j->area_x0 : j->area_z0) - 8;
    if ((e = cudaMemsetAsync(p, 0, 256, c.stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(j->hist, 0, 2 * kHistBins * sizeof(unsigned int), c.stream)) != cudaSuccess ||
        (e = launch_band_terms(j->ct, col_first, (int32_t)(g.width_u + 16), j->rt, g.vrows_alloc, g.vrows,
                               (int32_t)g.nJ, row_first, g.height_v + 16, g.stride, q.seed, g.transposed, g.indep,
                               g.groups, c.stream)) != cudaSuccess ||
        (e = launch_rare_scan(c.rare_targets.ptr, c.rare_offsets.ptr, q.seed, j->area_z0 - 8, (int32_t)(W + 16),
                              j->area_x0 - 8, (int32_t)(W + 16), j->rare, j->rare_cap, j->flags + 2,
                              c.stream)) != cudaSuccess) {
        c.set_error("server start", e);
        return false;
    }
    j->started = true;
    return true;
}

int Server::finish_band(Job* j) {
    Context& c = ctx();
    uint32_t fl[4] = {0, 0, 0, 0};
    unsigned long long cnt[2] = {0, 0};
    cudaError_t e;
    if ((e = cudaMemcpyAsync(fl, j->flags, sizeof(fl), cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(cnt, j->counts, sizeof(cnt), cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c.stream)) != cudaSuccess) {
        c.set_error("server finish", e);
        return 0;
    }
    if (fl[0] & 4u) { c.set_error("band engine: row-term copy timed out", cudaErrorLaunchTimeout); return 0; }
    j->results.assign((size_t)std::max<int32_t>(1, j->q.max_results), ExtChunkResult{});
    if ((fl[0] & 1u) || cnt[0] > j->hit_cap || fl[2] > j->rare_cap) {
        // A dense strip, a full hit slice or too many rare chunks: the single search redoes it.
        if (j->mem) cudaFreeAsync(j->mem, c.stream);
        j->mem = nullptr;
        const int64_t t = c.search(j->q, j->results.data());
        if (t < 0) return 0;
        j->total = t;
        return 1;
    }
    const uint64_t n = cnt[0];
    const uint32_t nrare = fl[2];
    std::vector<Hit> hits_h(n);
    if (n && nrare && (e = launch_filter_hits(j->hits, (int64_t)n, j->rare, (int32_t)nrare, false, c.stream)) != cudaSuccess) {
        c.set_error("server filter", e);
        return 0;
    }
    if (n && ((e = cudaMemcpyAsync(hits_h.data(), j->hits, n * sizeof(Hit), cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess ||
              (e = cudaStreamSynchronize(c.stream)) != cudaSuccess)) {
        c.set_error("server copy", e);
        return 0;
    }
    std::vector<Hit> best;
    best.reserve(n);
    for (const Hit& hit : hits_h)
        if (hit.count >= 0) best.push_back(hit);  // window holds a rare chunk: fixed below
    // Exact counts of the centres around the rare chunks, and the histogram's correction (their
    // first-draw counts out, their exact counts in).
    int* delta = reinterpret_cast<int*>(j->hist + kHistBins);
    if (nrare) {
        if ((e = c.fixed.reserve(1u << 20)) != cudaSuccess) {
            c.set_error("server fixup", e);
            return 0;
        }
        FixArgs f{};
        f.area_x0 = j->area_x0;
        f.area_z0 = j->area_z0;
        f.width = 2 * j->q.rd_max + 1;
        f.height = 2 * j->q.rd_max + 1;
        f.rd_min_sq = j->q.rd_min * j->q.rd_min;
        f.center_x = j->q.center_x;
        f.center_z = j->q.center_z;
        f.min_size = j->q.min_size;
        f.max_size = j->q.max_size;
        f.fixed = c.fixed.ptr;
        f.fixed_count = j->counts + 1;
        f.cap = c.fixed.count;
        f.error = j->flags + 1;
        f.hist_delta = delta;
        uint64_t nf = 0;
        uint32_t ferr = 0;
        if ((e = cudaMemsetAsync(j->counts + 1, 0, 8, c.stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(j->flags + 1, 0, 4, c.stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(delta, 0, kHistBins * sizeof(int), c.stream)) != cudaSuccess ||
            (e = launch_fixup(j->rare, (int32_t)nrare, j->q.seed, f, c.stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(&nf, j->counts + 1, 8, cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(&ferr, j->flags + 1, 4, cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(c.stream)) != cudaSuccess) {
            c.set_error("server fixup", e);
            return 0;
        }
        if (nf > c.fixed.count || ferr) { c.set_error("fixup overflow", cudaErrorUnknown); return 0; }
        const size_t old = best.size();
        best.resize(old + nf);
        if (nf && ((e = cudaMemcpyAsync(best.data() + old, c.fixed.ptr, nf * sizeof(Hit), cudaMemcpyDeviceToHost,
                                        c.stream)) != cudaSuccess ||
                   (e = cudaStreamSynchronize(c.stream)) != cudaSuccess)) {
            c.set_error("server copy", e);
            return 0;
        }
    }
    // Every centre in range by count, from the device histogram with the rare-chunk correction.
    std::vector<uint32_t> hd(2 * kHistBins, 0u);
    if ((e = cudaMemcpyAsync(hd.data(), j->hist, hd.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, c.stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c.stream)) != cudaSuccess) {
        c.set_error("server histogram", e);
        return 0;
    }
    std::vector<uint32_t> h(kHistBins, 0u);
    for (int i = 0; i < kHistBins; ++i) h[i] = (uint32_t)((int64_t)hd[i] + (int32_t)hd[kHistBins + i]);
    uint64_t total = 0, have = 0;
    for (int k = j->q.min_size; k <= j->q.max_size; ++k) {
        total += h[k];
        if (k >= j->emit_min) have += h[k];
    }
    const int64_t want = (j->q.biome_flags & 3) ? 2LL * j->q.max_results + 1024 : (int64_t)j->q.max_results;
    const uint64_t need = std::min<uint64_t>(total, (uint64_t)want);
    if (have < need && j->emit_min > j->q.min_size) {
        // Too few sites sent: rescan with the exact gate (the highest count whose cumulative number
        // covers need), like the single search's second pass.
        uint64_t acc = 0;
        int32_t gate = j->q.max_size;
        for (int k = j->q.max_size; k >= j->q.min_size; --k) {
            acc += h[k];
            gate = k;
            if (acc >= need) break;
        }
        j->emit_min = gate;
        j->next_tile = 0;
        if ((e = cudaMemsetAsync(j->counts, 0, 2 * sizeof(unsigned long long), c.stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(j->flags, 0, 2 * sizeof(unsigned int), c.stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(j->hist, 0, 2 * kHistBins * sizeof(unsigned int), c.stream)) != cudaSuccess) {
            c.set_error("server rescan", e);
            return 0;
        }
        return 2;
    }
    int64_t t = c.finish(j->q, best, h, j->results.data());
    if (t == kNeedMoreSites) t = c.search(j->q, j->results.data());  // biome exclusion needs more sites
    if (t < 0) return 0;
    j->total = t;
    return 1;
}

// One step over the live jobs (called with the library lock held).
bool Server::step(std::vector<Job*>& live) {
    Context& c = ctx();
    if (!c.ensure_device() || !c.ensure_band()) return false;
    // Requests for the general scan run whole, one per step, the smallest area first.
    Job* whole = nullptr;
    for (Job* j : live)
        if (!j->band && (!whole || j->q.rd_max < whole->q.rd_max)) whole = j;
    if (whole) {
        whole->results.assign((size_t)std::max<int32_t>(1, whole->q.max_results), ExtChunkResult{});
        const int64_t t = c.search(whole->q, whole->results.data());
        complete(whole, t, t >= 0);
        return true;
    }
    std::vector<Job*> band;
    for (Job* j : live) {
        if (!j->started && !start(j)) {
            complete(j, -1, false);
            continue;
        }
        band.push_back(j);
    }
    if (band.empty()) return true;
    // Work items, shortest remaining work first: each job in turn takes its remaining tiles up to
    // what is left of the step's tile budget, and at least a floor of a quarter wave, so that
    // small requests finish within a step while large ones keep moving.
    std::sort(band.begin(), band.end(), [](const Job* x, const Job* y) {
        return x->g.tiles - x->next_tile < y->g.tiles - y->next_tile;
    });
    const int64_t floor_tiles = std::max<int64_t>(1, c.sm_count / 4);
    int64_t budget = tiles_per_step;
    std::vector<BandArgs> items;
    std::vector<int64_t> take;
    for (Job* j : band) {
        const int64_t n = std::min<int64_t>(std::max<int64_t>(budget, floor_tiles), j->g.tiles - j->next_tile);
        budget = std::max<int64_t>(0, budget - n);
        take.push_back(n);
        if (n <= 0) continue;
        const SearchSpec& q = j->q;
        const BandGeom& g = j->g;
        BandArgs a{};
        a.ct = j->ct;
        a.ncols = g.width_u + 16;
        a.rt = j->rt;
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
        a.tile_begin = j->next_tile;
        a.tile_end = j->next_tile + n;
        a.min_size = q.min_size;
        a.max_size = q.max_size;
        a.rd_min_sq = q.rd_min * q.rd_min;
        a.area_x0 = j->area_x0;
        a.area_z0 = j->area_z0;
        a.center_x = q.center_x;
        a.center_z = q.center_z;
        a.transposed = g.transposed ? 1 : 0;
        a.out = j->hits;
        a.cap = j->hit_cap;
        a.emitted = j->counts;
        a.overflow = j->flags;
        a.one = 1u;
        a.mad_add = c.band_mad_add;
        a.exact = j->exact ? 1 : 0;
        a.poll_limit = c.wait_polls;
        a.indep = g.indep ? 1 : 0;
        a.groups = g.groups;
        a.row_stride = g.stride;
        a.hist = j->hist;
        a.emit_min = j->emit_min;
        items.push_back(a);
    }
    const int32_t m = (int32_t)items.size();
    cudaError_t e;
    if (m > 0) {
        if ((e = args.reserve((size_t)m)) != cudaSuccess || (e = prefix.reserve((size_t)m + 1)) != cudaSuccess ||
            (e = head.reserve(kBandClasses)) != cudaSuccess ||
            (e = run_band_items(items, args.ptr, prefix.ptr, head.ptr, c.sm_count, c.stream, nullptr)) != cudaSuccess ||
            (e = cudaStreamSynchronize(c.stream)) != cudaSuccess) {
            c.set_error("server step", e);
            return false;
        }
    }
    for (size_t k = 0; k < band.size(); ++k) {
        Job* j = band[k];
        j->next_tile += std::max<int64_t>(0, take[k]);
        if (j->next_tile < j->g.tiles) continue;
        const int r = finish_band(j);
        if (r == 2) continue;  // its tiles run again with a lower emission gate
        complete(j, r == 1 ? j->total : -1, r == 1);
    }
    return true;
}

void Server::run() {
    for (;;) {
        std::vector<Job*> live;
        {
            std::unique_lock<std::mutex> lock(mu);
            cv.wait(lock, [&] { return stop || !queued.empty() || !active.empty(); });
            if (stop) break;
            // Admission in arrival order while the device budget allows it; a request larger
            // than the whole budget can never run and fails.
            while (!queued.empty()) {
                Job* j = queued.front();
                if ((int64_t)j->bytes > budget) {
                    queued.pop_front();
                    j->state = kFailed;
                    j->t_done = Clock::now();
                    done_cv.notify_all();
                    continue;
                }
                if (used + (int64_t)j->bytes > budget) break;
                queued.pop_front();
                used += (int64_t)j->bytes;
                j->state = kRunning;
                active.push_back(j);
            }
            live = active;
        }
        {
            std::lock_guard<std::mutex> glock(ctx().mu);
            if (!step(live)) {  // a CUDA failure: fail what was in flight
                for (Job* j : live)
                    if (j->state == kRunning) complete(j, -1, false);
            }
        }
    }
    // Shutting down: release device memory of unfinished jobs.
    std::lock_guard<std::mutex> glock(ctx().mu);
    std::lock_guard<std::mutex> lock(mu);
    for (Job* j : active) {
        if (j->mem) cudaFreeAsync(j->mem, ctx().stream);
        j->mem = nullptr;
        j->state = kFailed;
    }
    active.clear();
    for (Job* j : queued) j->state = kFailed;
    queued.clear();
    if (ctx().stream) cudaStreamSynchronize(ctx().stream);
    done_cv.notify_all();
}

}  // namespace slime

using slime::Server;

extern "C" {

void* slime_b200_server_create(int64_t device_bytes, int32_t tiles_per_step) {
    if (device_bytes <= 0) return nullptr;
    {
        std::lock_guard<std::mutex> glock(slime::ctx().mu);
        if (!slime::ctx().ensure_device()) return nullptr;
    }
    auto* s = new Server();
    s->budget = device_bytes;
    s->tiles_per_step = tiles_per_step > 0 ? tiles_per_step : 4 * slime::ctx().sm_count;
    s->worker = std::thread([s] { s->run(); });
    return s;
}

int64_t slime_b200_server_submit(void* server, const SlimeBatchRequest* r) {
    auto* s = static_cast<Server*>(server);
    if (!s || !r) return -1;
    auto j = std::make_unique<slime::Job>();
    j->q = slime::SearchSpec{r->seed, r->rd_max, r->min_size, r->max_size, r->rd_min, r->center_x, r->center_z,
                             r->max_results, r->precise_afk, r->biome_flags, r->biome_version};
    std::vector<ExtChunkResult> probe(1);
    if (!slime::validate_search(j->q.rd_max, j->q.min_size, j->q.max_size, j->q.rd_min, j->q.center_x,
                                j->q.center_z, reinterpret_cast<slime::ExtChunkResult*>(probe.data()),
                                j->q.max_results) ||
        (j->q.biome_flags & ~7) != 0)
        return -1;
    slime::plan_job(*j, slime::ctx());  // reads only the device's SM count and engine thresholds
    j->t_submit = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) return -1;
    const int64_t t = s->next_ticket++;
    j->ticket = t;
    s->queued.push_back(j.get());
    s->jobs[t] = std::move(j);
    s->cv.notify_all();
    return t;
}

int32_t slime_b200_server_poll(void* server, int64_t ticket) {
    auto* s = static_cast<Server*>(server);
    if (!s) return slime::kUnknown;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(ticket);
    return it == s->jobs.end() ? slime::kUnknown : it->second->state;
}

int32_t slime_b200_server_wait(void* server, int64_t ticket, int32_t timeout_ms) {
    auto* s = static_cast<Server*>(server);
    if (!s) return slime::kUnknown;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return slime::kUnknown;
    slime::Job* j = it->second.get();
    s->done_cv.wait_for(lock, std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms),
                        [&] { return j->state == slime::kDone || j->state == slime::kFailed; });
    return j->state;
}

int64_t slime_b200_server_take(void* server, int64_t ticket, ExtChunkResult* results, int32_t capacity,
                               double* latency_ms) {
    auto* s = static_cast<Server*>(server);
    if (!s) return -2;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return -2;
    slime::Job* j = it->second.get();
    if (j->state != slime::kDone && j->state != slime::kFailed) return -2;
    if (latency_ms)
        *latency_ms = std::chrono::duration<double, std::milli>(j->t_done - j->t_submit).count();
    int64_t total = j->state == slime::kDone ? j->total : -1;
    if (total >= 0 && results && capacity > 0) {
        const int64_t n = std::min<int64_t>({total, (int64_t)capacity, (int64_t)j->q.max_results});
        std::copy(j->results.begin(), j->results.begin() + n, reinterpret_cast<slime::ExtChunkResult*>(results));
    }
    s->jobs.erase(it);
    return total;
}

void slime_b200_server_destroy(void* server) {
    auto* s = static_cast<Server*>(server);
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    {
        std::lock_guard<std::mutex> glock(slime::ctx().mu);
        s->args.free();
        s->prefix.free();
        s->head.free();
    }
    delete s;
}

}  // extern "C"
