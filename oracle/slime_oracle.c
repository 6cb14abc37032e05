/*
 * slime_oracle.c -- CPU restatement of the reference slime-chunk cluster search.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA product (see slime_oracle.h).
 * It is written for clarity, not speed: a plain scalar predicate, row prefix sums for the
 * 221-cell window and a sort for the ranking. Each function cites the reference lines it
 * restates (paths inside the OvOliziOvO/slime tree).
 */
#include "slime_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define LCG_MULT 0x5DEECE66DULL
#define LCG_ADD 0xBULL
#define MASK48 0xFFFFFFFFFFFFULL
#define SLIME_SCRAMBLE 0x3AD8025FULL

/* dx in [-128, 128] indexes the per-Y radius tables (SlimeCore.cpp:29-31). */
#define DX_MIN (-128)
#define DX_MAX 128
#define DX_COUNT (DX_MAX - DX_MIN + 1)

/* ---------------------------------------------------------------- predicate */

/* Java: seed + (int)(x*x*0x4c1906) + (int)(x*0x5ac0db) + (int)(z*z)*0x4307a7L
 *            + (int)(z*0x5f24f) ^ 0x3ad8025fL, with 32-bit wrap on the int products
 * (SlimeCore.cpp:209-215). */
static uint64_t seed_mix(int64_t seed, int64_t x, int64_t z) {
    const uint32_t ux = (uint32_t)(int32_t)x;
    const uint32_t uz = (uint32_t)(int32_t)z;
    const uint64_t a = (uint64_t)(int64_t)(int32_t)(ux * ux * 0x4c1906u);
    const uint64_t b = (uint64_t)(int64_t)(int32_t)(ux * 0x5ac0dbu);
    const uint64_t c = (uint64_t)(int64_t)(int32_t)(uz * uz) * 0x4307a7ull;
    const uint64_t d = (uint64_t)(int64_t)(int32_t)(uz * 0x5f24fu);
    return (uint64_t)seed + a + b + c + d;
}

/* new Random(mix).nextInt(10) == 0, with Java's rejection loop: next(31) draws are
 * rejected while bits - bits%10 + 9 overflows a signed int (SlimeCore.cpp:54-56,217-231). */
int oracle_is_slime(int64_t seed, int64_t cx, int64_t cz) {
    uint64_t state = (seed_mix(seed, cx, cz) ^ SLIME_SCRAMBLE ^ LCG_MULT) & MASK48;
    for (;;) {
        state = (state * LCG_MULT + LCG_ADD) & MASK48;
        const uint32_t bits = (uint32_t)(state >> 17);
        const uint32_t val = bits % 10u;
        if (bits - val + 9u <= 0x7FFFFFFFu) return val == 0;
    }
}

void oracle_slime_bitmap(int64_t seed, int64_t x0, int64_t z0, int32_t w, int32_t h,
                         uint8_t* out) {
    if (w <= 0 || h <= 0 || !out) return;
#pragma omp parallel for schedule(static)
    for (int32_t j = 0; j < h; ++j)
        for (int32_t i = 0; i < w; ++i)
            out[(int64_t)j * w + i] = (uint8_t)oracle_is_slime(seed, x0 + i, z0 + j);
}

/* ---------------------------------------------------------------- window */

/* Half-width of the AFK window on each row dz = -8..8: the largest k with
 * dz*dz + k*k <= 68 (SlimeCore.cpp:399-404). Rows: 2,4,5,6,7,7,8,8,8,8,8,7,7,6,5,4,2. */
static void window_half_widths(int32_t hw[17]) {
    for (int32_t d = -8; d <= 8; ++d) {
        int32_t k = 0;
        while (d * d + (k + 1) * (k + 1) <= 68) ++k;
        hw[d + 8] = k;
    }
}

/* Counts for a w x h block of centres from a (w+16) x (h+16) slime bitmap whose origin is
 * (cx0-8, cz0-8): each row's prefix sums turn a row slice into two lookups. */
static void counts_from_bitmap(const uint8_t* bm, int32_t w, int32_t h, int32_t* out,
                               int32_t* prefix /* (h+16) * (w+17) scratch */) {
    const int32_t bw = w + 16, bh = h + 16, pw = w + 17;
    int32_t hw[17];
    window_half_widths(hw);
    for (int32_t r = 0; r < bh; ++r) {
        int32_t* p = prefix + (int64_t)r * pw;
        p[0] = 0;
        for (int32_t k = 0; k < bw; ++k) p[k + 1] = p[k] + bm[(int64_t)r * bw + k];
    }
    for (int32_t j = 0; j < h; ++j) {
        for (int32_t i = 0; i < w; ++i) {
            int32_t total = 0;
            for (int32_t d = -8; d <= 8; ++d) {
                const int32_t* p = prefix + (int64_t)(j + 8 + d) * pw;
                total += p[i + 8 + hw[d + 8] + 1] - p[i + 8 - hw[d + 8]];
            }
            out[(int64_t)j * w + i] = total;
        }
    }
}

void oracle_window_counts(int64_t seed, int64_t cx0, int64_t cz0, int32_t w, int32_t h,
                          int32_t* out) {
    if (w <= 0 || h <= 0 || !out) return;
    const int64_t bw = w + 16, bh = h + 16;
    uint8_t* bm = (uint8_t*)malloc((size_t)(bw * bh));
    int32_t* prefix = (int32_t*)malloc(sizeof(int32_t) * (size_t)(bh * (w + 17)));
    if (!bm || !prefix) { free(bm); free(prefix); return; }
    oracle_slime_bitmap(seed, cx0 - 8, cz0 - 8, (int32_t)bw, (int32_t)bh, bm);
    counts_from_bitmap(bm, w, h, out, prefix);
    free(bm);
    free(prefix);
}

/* ---------------------------------------------------------------- ranking */

/* (size desc, center_x asc, center_z asc) on the 32-bit block coordinates
 * (SlimeCore.cpp:191-206; ResultGreater, SlimeCoreGPU.cu:213-220). */
static int result_cmp(const void* pa, const void* pb) {
    const OracleChunkResult* a = (const OracleChunkResult*)pa;
    const OracleChunkResult* b = (const OracleChunkResult*)pb;
    if (a->size != b->size) return a->size > b->size ? -1 : 1;
    if (a->center_x != b->center_x) return a->center_x < b->center_x ? -1 : 1;
    if (a->center_z != b->center_z) return a->center_z < b->center_z ? -1 : 1;
    return 0;
}

typedef struct ResultList {
    OracleChunkResult* v;
    int64_t n, cap;
} ResultList;

static int list_push(ResultList* l, OracleChunkResult r) {
    if (l->n == l->cap) {
        int64_t cap = l->cap ? l->cap * 2 : 1024;
        OracleChunkResult* v = (OracleChunkResult*)realloc(l->v, sizeof(*v) * (size_t)cap);
        if (!v) return 0;
        l->v = v;
        l->cap = cap;
    }
    l->v[l->n++] = r;
    return 1;
}

/* Keep only the best `keep` entries (sorted). */
static void list_trim(ResultList* l, int64_t keep) {
    qsort(l->v, (size_t)l->n, sizeof(OracleChunkResult), result_cmp);
    if (l->n > keep) l->n = keep;
}

/* ---------------------------------------------------------------- precise scoring */

static int32_t isqrt_floor(int32_t v) {
    if (v < 0) return -1;
    int32_t r = 0;
    for (int32_t bit = 1 << 15; bit; bit >>= 1) {
        const int32_t t = r | bit;
        if ((int64_t)t * t <= v) r = t;
    }
    return r;
}

static int64_t floor_div16(int64_t v) {
    return v >= 0 ? v / 16 : -((-v + 15) / 16);
}

typedef struct YTables {
    int32_t count;
    int32_t* values;
    int16_t* outer; /* count x DX_COUNT, -1 where dy^2 + dx^2 > 128^2 */
    int16_t* inner; /* count x DX_COUNT, -1 where dy^2 + dx^2 > 24^2 */
    int32_t platform_y;
    int32_t scan_y;
} YTables;

/* rebuild_y_radius_tables (SlimeCore.cpp:148-180) after set_y_scan_config's own
 * normalisation of the step (y_step <= 0 becomes 4, SlimeCore.cpp:364-371). A NULL config
 * is the library's initial state: Y scan off, platform Y -64. */
static int build_y_tables(const OracleYConfig* cfg, YTables* t) {
    OracleYConfig c = {0, -64, -64, 64, 4};
    if (cfg) c = *cfg;
    if (c.y_step <= 0) c.y_step = 4;
    const int enabled = c.enabled != 0;
    int32_t y0 = enabled ? c.y_min : c.platform_y;
    int32_t y1 = enabled ? c.y_max : c.platform_y;
    int32_t step = enabled ? c.y_step : 1;
    if (y1 < y0) { int32_t s = y0; y0 = y1; y1 = s; }
    int32_t count = (y1 - y0) / step + 1;
    if (count <= 0) count = 1;
    t->count = count;
    t->platform_y = c.platform_y;
    t->scan_y = enabled;
    t->values = (int32_t*)malloc(sizeof(int32_t) * (size_t)count);
    t->outer = (int16_t*)malloc(sizeof(int16_t) * (size_t)count * DX_COUNT);
    t->inner = (int16_t*)malloc(sizeof(int16_t) * (size_t)count * DX_COUNT);
    if (!t->values || !t->outer || !t->inner) return 0;
    for (int32_t yi = 0; yi < count; ++yi) {
        const int32_t y = y0 + yi * step;
        const int32_t dy = c.platform_y - y;
        const int32_t dy2 = dy * dy;
        t->values[yi] = y;
        for (int32_t dx = DX_MIN; dx <= DX_MAX; ++dx) {
            const int64_t k = (int64_t)yi * DX_COUNT + (dx - DX_MIN);
            const int32_t o = 16384 - dy2 - dx * dx;
            const int32_t n = 576 - dy2 - dx * dx;
            t->outer[k] = (int16_t)(o >= 0 ? isqrt_floor(o) : -1);
            t->inner[k] = (int16_t)(n >= 0 ? isqrt_floor(n) : -1);
        }
    }
    return 1;
}

static void free_y_tables(YTables* t) {
    free(t->values);
    free(t->outer);
    free(t->inner);
}

static int32_t interval_len(int32_t a, int32_t b) { return b >= a ? b - a + 1 : 0; }
static int64_t max64(int64_t a, int64_t b) { return a > b ? a : b; }
static int64_t min64(int64_t a, int64_t b) { return a < b ? a : b; }
static int32_t max32(int32_t a, int32_t b) { return a > b ? a : b; }
static int32_t min32(int32_t a, int32_t b) { return a < b ? a : b; }

/* Number of block columns of slime chunks within the horizontal annulus
 * 24^2 < dx^2 + dy^2 + dz^2 <= 128^2 around block (ox, oz), for one Y level
 * (build_chunk_cache + count_spawnable_cached_table, SlimeCore.cpp:234-246,291-331). */
static int32_t spawnable_count(int64_t ox, int64_t oz, const int16_t* outer,
                               const int16_t* inner, const uint8_t cache[21][21],
                               int64_t base_cx, int64_t base_cz) {
    int32_t count = 0;
    for (int32_t i = 0; i < 21; ++i) {
        const int64_t x0 = (base_cx + i) * 16;
        const int32_t rx0 = (int32_t)max64(DX_MIN, x0 - ox);
        const int32_t rx1 = (int32_t)min64(DX_MAX, x0 + 15 - ox);
        if (rx0 > rx1) continue;
        for (int32_t j = 0; j < 21; ++j) {
            if (!cache[i][j]) continue;
            const int64_t z0 = (base_cz + j) * 16;
            const int32_t rz0 = (int32_t)max64(DX_MIN, z0 - oz);
            const int32_t rz1 = (int32_t)min64(DX_MAX, z0 + 15 - oz);
            if (rz0 > rz1) continue;
            for (int32_t dx = rx0; dx <= rx1; ++dx) {
                const int32_t ro = outer[dx - DX_MIN];
                if (ro < 0) continue;
                const int32_t zl = max32(rz0, -ro), zr = min32(rz1, ro);
                int32_t add = interval_len(zl, zr);
                if (!add) continue;
                const int32_t ri = inner[dx - DX_MIN];
                if (ri >= 0) add -= interval_len(max32(zl, -ri), min32(zr, ri));
                count += add;
            }
        }
    }
    return count;
}

static int32_t pack_obs_y(int32_t obs, int32_t y) {
    return (int32_t)((uint32_t)obs | ((uint32_t)(y + 1024) << 20));
}

/* Best (strict >, first in dx-major, dz, Y order) over the offsets around one site
 * (SlimeCore.cpp:667-717). */
static void score_site(int64_t seed, OracleChunkResult* r, int32_t scan_xz, const YTables* t) {
    const int64_t bx = r->center_x, bz = r->center_z;
    int32_t best = 0, best_y = t->platform_y;
    int64_t best_x = bx, best_z = bz;
    const int32_t lo = scan_xz ? -16 : 0, hi = scan_xz ? 16 : 0, step = scan_xz ? 4 : 1;
    const int32_t ycount = t->scan_y ? t->count : 1;
    for (int32_t dx = lo; dx <= hi; dx += step) {
        for (int32_t dz = lo; dz <= hi; dz += step) {
            const int64_t ox = bx + dx, oz = bz + dz;
            const int64_t base_cx = floor_div16(ox) - 10, base_cz = floor_div16(oz) - 10;
            uint8_t cache[21][21];
            for (int32_t i = 0; i < 21; ++i)
                for (int32_t j = 0; j < 21; ++j)
                    cache[i][j] = (uint8_t)oracle_is_slime(seed, base_cx + i, base_cz + j);
            for (int32_t yi = 0; yi < ycount; ++yi) {
                const int32_t obs = spawnable_count(ox, oz, t->outer + (int64_t)yi * DX_COUNT,
                                                    t->inner + (int64_t)yi * DX_COUNT, cache,
                                                    base_cx, base_cz);
                if (obs > best) {
                    best = obs;
                    best_x = ox;
                    best_z = oz;
                    best_y = t->values[yi];
                }
            }
        }
    }
    r->obs_count = t->scan_y ? pack_obs_y(best, best_y) : best;
    r->afk_x = (int32_t)best_x;
    r->afk_z = (int32_t)best_z;
}

void oracle_score_candidates_precise(int64_t seed, OracleChunkResult* buf, int32_t count,
                                     int32_t scan_xz, const OracleYConfig* ycfg,
                                     int32_t threads) {
    if (!buf || count <= 0) return;
    YTables t;
    if (!build_y_tables(ycfg, &t)) { free_y_tables(&t); return; }
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
#pragma omp parallel for schedule(dynamic)
    for (int32_t i = 0; i < count; ++i) score_site(seed, &buf[i], scan_xz, &t);
    free_y_tables(&t);
}

/* refine_candidates_y (SlimeCore.cpp:728-773): XZ offsets always, every Y of the table,
 * the result always packs Y. */
void oracle_refine_candidates_y(int64_t seed, OracleChunkResult* buf, int32_t count,
                                const OracleYConfig* ycfg, int32_t threads) {
    if (!buf || count <= 0) return;
    YTables t;
    if (!build_y_tables(ycfg, &t)) { free_y_tables(&t); return; }
    t.scan_y = 1;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
#pragma omp parallel for schedule(dynamic)
    for (int32_t i = 0; i < count; ++i) score_site(seed, &buf[i], 1, &t);
    free_y_tables(&t);
}

/* ---------------------------------------------------------------- search */

#define TILE 256

int64_t oracle_search_centered(int64_t seed, int64_t rd_max, int32_t min_size, int32_t max_size,
                               int64_t rd_min, int32_t center_x, int32_t center_z,
                               OracleChunkResult* out, int32_t max_results,
                               int32_t precise_afk, int32_t precise_limit,
                               const OracleYConfig* ycfg, int32_t threads) {
    /* Argument checks of SlimeCore.cpp:378-384. */
    if (!out || max_results <= 0 || rd_max < 0 || rd_max > (INT32_MAX - 17LL) / 2LL ||
        rd_min < 0 || rd_min > rd_max || min_size < 0 || min_size > 221 || max_size < min_size)
        return -1;
    if ((int64_t)center_x - rd_max - 8 < INT32_MIN || (int64_t)center_x + rd_max + 8 > INT32_MAX ||
        (int64_t)center_z - rd_max - 8 < INT32_MIN || (int64_t)center_z + rd_max + 8 > INT32_MAX)
        return -1;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    const int64_t width = 2 * rd_max + 1;
    const int64_t min_x = (int64_t)center_x - rd_max, min_z = (int64_t)center_z - rd_max;
    const int64_t tiles_x = (width + TILE - 1) / TILE;
    const int64_t tiles = tiles_x * tiles_x;
    const int64_t rd_min_sq = rd_min * rd_min;
    int64_t total = 0;
    ResultList merged = {0, 0, 0};
    int failed = 0;

#pragma omp parallel
    {
        ResultList local = {0, 0, 0};
        int64_t local_total = 0;
        uint8_t* bm = (uint8_t*)malloc((TILE + 16) * (TILE + 16));
        int32_t* prefix = (int32_t*)malloc(sizeof(int32_t) * (TILE + 16) * (TILE + 17));
        int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * TILE * TILE);
        int local_failed = !bm || !prefix || !counts;
#pragma omp for schedule(dynamic, 1)
        for (int64_t t = 0; t < tiles; ++t) {
            if (local_failed) continue;
            const int64_t x0 = min_x + (t % tiles_x) * TILE;
            const int64_t z0 = min_z + (t / tiles_x) * TILE;
            const int32_t w = (int32_t)min64(TILE, min_x + width - x0);
            const int32_t h = (int32_t)min64(TILE, min_z + width - z0);
            for (int32_t j = 0; j < h + 16; ++j)
                for (int32_t i = 0; i < w + 16; ++i)
                    bm[(int64_t)j * (w + 16) + i] =
                        (uint8_t)oracle_is_slime(seed, x0 - 8 + i, z0 - 8 + j);
            counts_from_bitmap(bm, w, h, counts, prefix);
            for (int32_t j = 0; j < h; ++j) {
                for (int32_t i = 0; i < w; ++i) {
                    const int64_t cx = x0 + i, cz = z0 + j;
                    if (rd_min > 0) {
                        const int64_t dx = cx - center_x, dz = cz - center_z;
                        if (dx * dx + dz * dz < rd_min_sq) continue;
                    }
                    const int32_t c = counts[(int64_t)j * w + i];
                    if (c < min_size || c > max_size) continue;
                    ++local_total;
                    OracleChunkResult r = {c, (int32_t)(cx * 16 + 8), (int32_t)(cz * 16 + 8), 0,
                                           0, 0};
                    r.afk_x = r.center_x;
                    r.afk_z = r.center_z;
                    if (!list_push(&local, r)) { local_failed = 1; break; }
                    if (local.n > 2 * (int64_t)max_results + 4096) list_trim(&local, max_results);
                }
            }
        }
        if (!local_failed) list_trim(&local, max_results);
#pragma omp critical
        {
            if (local_failed) failed = 1;
            total += local_total;
            for (int64_t k = 0; k < local.n && !failed; ++k)
                if (!list_push(&merged, local.v[k])) failed = 1;
        }
        free(local.v);
        free(bm);
        free(prefix);
        free(counts);
    }
    if (failed) { free(merged.v); return -1; }
    list_trim(&merged, max_results);
    memcpy(out, merged.v, sizeof(OracleChunkResult) * (size_t)merged.n);
    const int32_t n = (int32_t)merged.n;
    free(merged.v);

    if (precise_afk && n > 0) {
        YTables t;
        if (build_y_tables(ycfg, &t)) {
            const int32_t limit = precise_limit < n ? precise_limit : n;
#pragma omp parallel for schedule(dynamic)
            for (int32_t i = 0; i < limit; ++i) score_site(seed, &out[i], 1, &t);
        }
        free_y_tables(&t);
    }
    return total;
}
