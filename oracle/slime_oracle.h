/*
 * slime_oracle.h -- CPU restatement of the reference slime-chunk cluster search.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA product is compared
 * against; the product never links, loads or calls it. Every function states the reference
 * file:line it restates (paths are inside the OvOliziOvO/slime source tree).
 *
 * Pinning: the restatement is itself checked against the reference's own compiled CPU library
 * (SlimeCore.cpp built by oracle/Makefile into oracle/_ref/) and against golden vectors that
 * were generated from that library (tests/golden/).
 */
#ifndef SLIME_ORACLE_H
#define SLIME_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same 24-byte record as the reference's ExtChunkResult (SlimeCore.cpp:182-189). */
typedef struct OracleChunkResult {
    int32_t size;
    int32_t center_x;
    int32_t center_z;
    int32_t obs_count;
    int32_t afk_x;
    int32_t afk_z;
} OracleChunkResult;

/* Java slime predicate (SlimeCore.cpp:208-232). */
int oracle_is_slime(int64_t seed, int64_t cx, int64_t cz);

/* One byte per chunk: out[j * w + i] = slime(x0 + i, z0 + j). */
void oracle_slime_bitmap(int64_t seed, int64_t x0, int64_t z0, int32_t w, int32_t h,
                         uint8_t* out);

/* Exact 221-cell AFK window count for every centre of a w x h block of centres:
 * out[j * w + i] = count(cx0 + i, cz0 + j)   (SlimeCore.cpp:399-404,526-533). */
void oracle_window_counts(int64_t seed, int64_t cx0, int64_t cz0, int32_t w, int32_t h,
                          int32_t* out);

/* Y-level configuration used by precise scoring (SlimeCore.cpp:19-27,148-180,364-371). */
typedef struct OracleYConfig {
    int32_t enabled;
    int32_t platform_y;
    int32_t y_min;
    int32_t y_max;
    int32_t y_step;
} OracleYConfig;

/* Centred search (SlimeCore.cpp:373-632). Returns the number of centres with
 * min_size <= count <= max_size (outside the rd_min disc), -1 on invalid arguments.
 * Writes the first min(total, max_results) results ranked (size desc, block x asc,
 * block z asc). If precise_afk != 0 the first min(n, precise_limit) results get the
 * precise AFK score (precise_limit is 500 in SlimeCore.cpp:573-577 and 100 in the GPU
 * library, SlimeCoreGPU.cu:3884). threads <= 0 means one thread. */
int64_t oracle_search_centered(int64_t seed, int64_t rd_max, int32_t min_size, int32_t max_size,
                               int64_t rd_min, int32_t center_x, int32_t center_z,
                               OracleChunkResult* out, int32_t max_results,
                               int32_t precise_afk, int32_t precise_limit,
                               const OracleYConfig* ycfg, int32_t threads);

/* Precise AFK scoring of arbitrary sites (SlimeCore.cpp:654-726). */
void oracle_score_candidates_precise(int64_t seed, OracleChunkResult* buf, int32_t count,
                                     int32_t scan_xz, const OracleYConfig* ycfg,
                                     int32_t threads);

/* Multi-Y refinement (SlimeCore.cpp:728-773). */
void oracle_refine_candidates_y(int64_t seed, OracleChunkResult* buf, int32_t count,
                                const OracleYConfig* ycfg, int32_t threads);

#ifdef __cplusplus
}
#endif

#endif
