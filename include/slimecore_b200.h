/*
 * slimecore_b200.h -- C ABI of libslime_b200.so, the B200 (sm_100a) slime-chunk cluster search.
 *
 * The first group of entry points has exactly the signatures, argument meaning, return values
 * and error behaviour of the reference GPU library `slimecore_gpu` (SlimeCoreGPU.cu, whose
 * extern "C" block spans lines 3034-3991) and of `score_candidates_precise` in the reference
 * CPU library (SlimeCore.cpp:654-726), so a frontend that binds those libraries with ctypes can
 * load this one instead. Every declaration cites the reference function it replaces.
 *
 * Conventions (as in the reference):
 *  - Coordinates passed in are chunk coordinates; results carry block coordinates 16*c + 8.
 *  - Calls are synchronous. The library serialises concurrent calls with an internal lock.
 *  - The search returns the number of centres with min_size <= count <= max_size (not the
 *    number written) and writes the first min(total, max_results) results ranked by
 *    (size desc, center_x asc, center_z asc); -1 on invalid arguments or a CUDA failure.
 *  - There is no CPU fallback: without a usable CUDA device every search returns -1.
 */
#ifndef SLIMECORE_B200_H
#define SLIMECORE_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 24-byte record, identical layout to ExtChunkResult (SlimeCoreGPU.cu:198-205). */
typedef struct ExtChunkResult {
    int32_t size;      /* slime chunks inside the 221-cell AFK window */
    int32_t center_x;  /* block x of the centre chunk: 16 * cx + 8 */
    int32_t center_z;  /* block z of the centre chunk: 16 * cz + 8 */
    int32_t obs_count; /* precise AFK score (| (y + 1024) << 20 with Y scan), else 0 */
    int32_t afk_x;     /* best AFK block x (centre when not scored) */
    int32_t afk_z;     /* best AFK block z */
} ExtChunkResult;

/* ---- search (replaces SlimeCoreGPU.cu:3927-3955) ------------------------------------------- */

/* search_slime_clusters_gpu_v1 (SlimeCoreGPU.cu:3927-3934): search centred on chunk (0, 0). */
int64_t search_slime_clusters_gpu_v1(int64_t seed, int64_t rd_max, int32_t min_size,
                                     int32_t max_size, int64_t rd_min,
                                     ExtChunkResult* results_buffer, int32_t max_results,
                                     int32_t precise_afk);

/* search_slime_clusters_gpu_v1_centered (SlimeCoreGPU.cu:3936-3944). Centres are the
 * (2*rd_max+1)^2 chunks around the search centre minus those with dx^2 + dz^2 < rd_min^2.
 * With precise_afk != 0 the best min(n, 100) results are scored (SlimeCoreGPU.cu:3882-3909). */
int64_t search_slime_clusters_gpu_v1_centered(int64_t seed, int64_t rd_max, int32_t min_size,
                                              int32_t max_size, int64_t rd_min,
                                              int32_t search_center_x, int32_t search_center_z,
                                              ExtChunkResult* results_buffer, int32_t max_results,
                                              int32_t precise_afk);

/* Legacy aliases (SlimeCoreGPU.cu:3946-3965). */
int64_t search_slime_clusters_gpu_v34(int64_t seed, int64_t rd_max, int32_t min_size,
                                      int32_t max_size, int64_t rd_min,
                                      ExtChunkResult* results_buffer, int32_t max_results,
                                      int32_t precise_afk);
int64_t search_slime_clusters_gpu_v34_centered(int64_t seed, int64_t rd_max, int32_t min_size,
                                               int32_t max_size, int64_t rd_min,
                                               int32_t search_center_x, int32_t search_center_z,
                                               ExtChunkResult* results_buffer,
                                               int32_t max_results, int32_t precise_afk);

/* ---- precise AFK scoring -------------------------------------------------------------------- */

/* refine_candidates_y (SlimeCoreGPU.cu:3958-3990): XZ offsets and every configured Y level;
 * obs_count always packs Y. Semantics of the reference CPU routine (SlimeCore.cpp:728-773). */
void refine_candidates_y(int64_t seed, ExtChunkResult* results_buffer, int32_t count);

/* score_candidates_precise (SlimeCore.cpp:654-726): `threads` is accepted for signature
 * compatibility and ignored (the work runs on the GPU). */
void score_candidates_precise(int64_t seed, ExtChunkResult* results_buffer, int32_t count,
                              int32_t threads, int32_t scan_xz);

/* set_y_scan_config (SlimeCoreGPU.cu:3123-3140): y_step <= 0 means 4. */
void set_y_scan_config(int32_t enabled, int32_t platform_y, int32_t y_min, int32_t y_max,
                       int32_t y_step);

/* ---- control and progress (SlimeCoreGPU.cu:3085-3116) --------------------------------------- */

void request_cancel(void);
void request_pause(void);
void resume_search(void);
void reset_cancel(void);
int32_t get_progress(void);
int64_t get_processed_centers(void);
int64_t get_gpu_scan_work_ns(void);

/* ---- device and diagnostics (SlimeCoreGPU.cu:3035-3083,3118-3161) --------------------------- */

int32_t get_cuda_device_count(void);
int32_t get_cuda_device_name(char* buffer, int32_t buffer_size);
int32_t get_gpu_v1_shape(void);
int32_t get_gpu_v1_algorithm(void);
int32_t get_gpu_v1_rng(void);
void set_gpu_v1_rng_override(int32_t value);
int32_t get_gpu_v34_shape(void);
int32_t get_gpu_v34_rng(void);
void set_gpu_v34_rng_override(int32_t value);
/* Releases this library's device buffers and stream. Unlike the reference
 * (SlimeCoreGPU.cu:3118-3121) it never resets the device. */
void cleanup_gpu_resources(void);
/* is_slime_chunk_c (SlimeCoreGPU.cu:3142-3161). */
bool is_slime_chunk_c(int64_t seed, int64_t cx, int64_t cz);

/* ---- additions of this library (no reference counterpart) ----------------------------------- */

/* Library version string. */
const char* slime_b200_version(void);

/* Statistics of the last search call: summed duration of its scan kernels, timed with CUDA events
 * on the library's stream, and the number of kernels it launched. */
void slime_b200_last_search_stats(double* kernel_ms, int64_t* launches);

/* Rare redraw chunks (first draw rejected by nextInt(10), redraw slime) found by the last search
 * that used the band engine; 0 otherwise. */
int64_t slime_b200_last_rare_chunks(void);

/* Engine selection: mode 0 automatic, 1 always the general scan, 2 the shared-LCG band engine,
 * 3 the independent-band engine and 6 the grouped-band engine whenever the threshold allows it
 * (min_size >= 28), 4 / 5 / 7 the shared-LCG / independent-band / grouped-band engine with
 * bit-sliced exact counts (any threshold).
 * `band_min_threshold` (28..221, other values keep the current one) is the smallest threshold
 * automatic mode sends to the shared-LCG band engine. Results are identical either way; only
 * speed differs. get_gpu_v1_algorithm() reports 100 (general), 200 (band), 300 (independent
 * bands), 220 (grouped bands), or 210 / 310 / 230 (their exact-count modes) for the last search. */
void slime_b200_set_engine(int32_t mode, int32_t band_min_threshold);

/* The automatic engine rule as 6, 8 or 12 numbers: {band_min_threshold, band_min_periods,
 * band_fast_threshold, band_fast_periods, indep_min_threshold, indep_min_centres,
 * exact_below_threshold, exact_min_centres, grouped_min_threshold, grouped_min_width,
 * grouped_max_width, exact_wide_below_threshold}. Areas 4 x 2^17 chunks wide or more use the
 * exact counts below the larger of exact_below_threshold and exact_wide_below_threshold. Thresholds below exact_below_threshold on areas of
 * exact_min_centres centres or more use the band engines with bit-sliced exact counts (shared LCG
 * on areas band_fast_periods x 2^17 chunks wide, grouped bands from 4 x 2^17 up to
 * grouped_max_width, else independent bands) while the expected
 * number of sites stays below 1e9. Otherwise grouped bands (X phase pairs with groups of Z period
 * copies) take areas grouped_min_width .. grouped_max_width chunks wide (at most 16 x 2^17) from
 * grouped_min_threshold; the shared-LCG band engine takes areas at least
 * band_min_periods x 2^17 chunks wide from band_min_threshold, or band_fast_periods x 2^17 wide
 * from band_fast_threshold; independent bands take areas of indep_min_centres centres or more from indep_min_threshold; the
 * general scan takes the rest. Thresholds 28..222 (222 disables a branch;
 * exact_below_threshold and exact_wide_below_threshold 0..222, 0 disables them;
 * grouped_min_threshold 28..222), periods 2..64,
 * widths >= 0. With n = 6 or 8 the numbers not given are kept. Returns 0, or -1 for a wrong count or a value out of range (nothing is changed).
 * slime_b200/autotune.py measures the crossovers on the local GPU and writes them; the defaults are
 * B200 measurements. */
int32_t slime_b200_set_engine_rule(const int64_t* rule, int32_t n);
int32_t slime_b200_get_engine_rule(int64_t* rule, int32_t n);

/* Generator variant of the band engine (results are identical): band_mad_add != 0 issues the
 * per-band add on the multiply pipe instead of the integer ALU. */
void slime_b200_set_tuning(int32_t band_mad_add);

/* Polls of the band kernels' bounded mbarrier waits (row-term bulk copies) before a CTA gives up:
 * it then waits, again bounded, for its copies still in flight, flags the search, and the search
 * returns -1 with the error text "row-term copy timed out"; the library stays usable. polls < 0
 * restores the default (2^22). Returns the previous value. For tests of that error path: with 0 the
 * first wait gives up at once. */
int64_t slime_b200_set_wait_limit(int64_t polls);

/* Last CUDA error text of this library ("" if none). */
const char* slime_b200_last_error(void);

/* out[i] = is_slime(seed, x[i], z[i]) for n host-resident coordinates, evaluated on the GPU.
 * Returns 0, or -1 on a CUDA failure. */
int32_t slime_b200_is_slime_batch(int64_t seed, const int64_t* x, const int64_t* z, uint8_t* out,
                                  int64_t n);

/* Integer-pipe throughput probe on the current device (the denominator of the scan's roofline).
 * kind: 0 LOP3, 1 IADD3, 2 IMAD, 3 POPC, 4 generator mix (IADD3+LOP3+IMAD+ISETP+VOTE),
 * 5 b1 tensor AND+POPC (mma.sync m16n8k256), 6 SHF, 7 ISETP+VOTE+LOP3, 8 generator mix with the
 * add as a multiply-add. Writes lane operations per second and the
 * timed milliseconds. Returns 0, or -1 on a CUDA failure. */
int32_t slime_b200_microbench(int32_t kind, int32_t iters, double* lane_ops_per_s, double* ms);

/* Search without any allocation (no counterpart in the reference). For callers that cannot
 * allocate GPU memory while they search -- an application whose own pool or caching allocator
 * owns the device memory, a service that must not take cudaMalloc's implicit device
 * synchronisation on its request path, or a program with a fixed memory budget. Same arguments,
 * return value and ranked output as search_slime_clusters_gpu_v1_centered, without precise
 * scoring. Its working memory is one fixed 4 MiB array inside the library, which every GPU that
 * loads the library holds until the process exits; the call makes no cudaMalloc, cudaFree,
 * cudaMallocHost or host heap allocation (error texts go to a fixed buffer). Limits: rd_max <= 8191
 * and max_results <= 65536; larger requests return -1 with an error text (slime_b200_last_error).
 * A call can also return -1 if a single 64-row band of the area holds more than about 327k centres
 * at or above the count gate its max_results implies (possible only with max_results near 65536
 * and a wide area). The first call on a device looks up the array's device address (set-up) and
 * caches it per device ordinal, so make that first call before any stream capture; a device
 * reset invalidates the cached address, so call cleanup_gpu_resources() after resetting a device.
 * The array exists once per process and device (per loaded module and context), and every call
 * in the process shares it: the library lock serialises calls from the threads of one process,
 * and calls that could still overlap on the GPU (another context of the same process on the same
 * device) race. Runs on the legacy default stream. */
int64_t slime_b200_search_noalloc(int64_t seed, int64_t rd_max, int32_t min_size, int32_t max_size,
                                  int64_t rd_min, int32_t search_center_x, int32_t search_center_z,
                                  ExtChunkResult* results_buffer, int32_t max_results);

/* ---- search with biome exclusion (replaces the search + mcgpu_modern_ctx_filter_candidates
 *      round trip of the reference's frontend) ---------------------------------------------- */

/* search_slime_clusters_gpu_v1_centered with the biome filter inside the call. biome_flags: bit 0
 * exclude sites whose AFK window holds a slime chunk with a Deep Dark quart (quart Y -16..0),
 * bit 1 one with a Mushroom Fields quart (quart Y 16), bit 2 large biomes; biome_version is the
 * Minecraft version code of the parameter tree (>= 1194, e.g. 2602). The return value is still
 * the number of centres in range (the filter does not change it); the results are the first
 * min(passing, max_results) ranked sites whose verdict (mcgpu_modern_ctx_filter_candidates with
 * the same flags) is 0, with precise scores of the best min(n, 100) when precise_afk != 0; the
 * records after them, up to min(total, max_results), have size -1 (the same holds for the
 * results of batches and of the server, whose requests carry the same flags). With
 * biome_flags & 3 == 0 it is exactly search_slime_clusters_gpu_v1_centered. -1 on invalid
 * arguments (including other flag bits or an unsupported version) or a CUDA failure. */
int64_t slime_b200_search_biome(int64_t seed, int64_t rd_max, int32_t min_size, int32_t max_size,
                                int64_t rd_min, int32_t search_center_x, int32_t search_center_z,
                                ExtChunkResult* results_buffer, int32_t max_results, int32_t precise_afk,
                                int32_t biome_flags, int32_t biome_version);

/* Sites the biome filter examined and excluded in the last search (0 without a filter). */
void slime_b200_last_biome_stats(int64_t* examined, int64_t* excluded);

/* ---- batched search (no reference counterpart) --------------------------------------------- */

/* One search of a batch: the arguments of slime_b200_search_biome (those of
 * search_slime_clusters_gpu_v1_centered plus the biome exclusion). 56 bytes. */
typedef struct SlimeBatchRequest {
    int64_t seed;
    int64_t rd_max;
    int64_t rd_min;
    int32_t min_size;
    int32_t max_size;
    int32_t center_x;
    int32_t center_z;
    int32_t max_results;
    int32_t precise_afk;
    int32_t biome_flags;    /* 0, or bit 0 exclude Deep Dark, bit 1 Mushroom Fields, bit 2 large biomes */
    int32_t biome_version;  /* Minecraft version code of the biome tree, e.g. 2602 */
} SlimeBatchRequest;

/* Runs n searches as one batch (each with its own biome exclusion, as slime_b200_search_biome).
 * Searches with min_size >= 28 share one persistent launch of the independent-band kernel whose CTAs take the tiles of all of them from one device queue; the
 * others (and any whose sites would not fit the batch's pool) run one by one. Request i writes
 * min(total_i, max_results_i) ranked results at results + (max_results_0 + ... +
 * max_results_{i-1}) and its total to totals[i], exactly as the single search would; totals[i]
 * is -1 when request i's arguments are invalid. Returns 0, or -1 on a CUDA failure or a null
 * buffer. No reference counterpart: the reference library runs one search per call. */
int32_t slime_b200_search_batch(const SlimeBatchRequest* requests, int32_t n, ExtChunkResult* results,
                                int64_t* totals);

/* ---- search server (no reference counterpart) ----------------------------------------------- */

/* A server runs submitted searches on a worker thread with continuous batching: each step admits
 * queued requests in arrival order while the device memory they need fits `device_bytes`, then
 * runs a quantum of tiles (about `tiles_per_step` in all; <= 0 picks 4 per SM) of every admitted
 * band-engine search in one persistent launch, finishing those whose last tile ran. Requests for
 * the general scan (thresholds below the band engines' range) run whole within a step. Results
 * are exactly those of search_slime_clusters_gpu_v1_centered for the same arguments. Returns an
 * opaque handle, or NULL without a usable device. */
void* slime_b200_server_create(int64_t device_bytes, int32_t tiles_per_step);

/* Queues one request; returns its ticket (>= 0), or -1 for invalid arguments. */
int64_t slime_b200_server_submit(void* server, const SlimeBatchRequest* request);

/* State of a ticket: 0 queued, 1 running, 2 done, -1 failed (e.g. it needs more device memory
 * than the server's budget), -2 unknown ticket. */
int32_t slime_b200_server_poll(void* server, int64_t ticket);

/* Waits up to timeout_ms for a ticket to finish; returns its state as slime_b200_server_poll. */
int32_t slime_b200_server_wait(void* server, int64_t ticket, int32_t timeout_ms);

/* For a finished ticket: writes min(total, capacity, max_results) ranked results, the time from
 * submission to completion in ms, forgets the ticket and returns the total (-1 if it failed).
 * Returns -2 (ticket kept) while it is not finished, or for an unknown ticket. */
int64_t slime_b200_server_take(void* server, int64_t ticket, ExtChunkResult* results, int32_t capacity,
                               double* latency_ms);

/* Stops the worker (unfinished tickets fail), releases the server's device memory and the handle. */
void slime_b200_server_destroy(void* server);

#ifdef __cplusplus
}
#endif

#endif /* SLIMECORE_B200_H */
