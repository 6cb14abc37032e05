/*
 * biome_oracle.c -- plain-C restatement of the reference's FP64 biome filter.
 *
 * TEST INFRASTRUCTURE ONLY: a checker for the CUDA biome filter, never part of the product. Each
 * function cites the part of the reference (gpu_noise/MinecraftGPUNoise.cu) whose algorithm it
 * restates. Compiled with -ffp-contract=off: every double/float operation is one IEEE operation
 * in source order, as the reference's code reads. The data (octave and climate hashes, octave
 * amplitudes, depth-spline control points, the biome parameter trees of 1.18 to 26.2) comes from
 * slime_b200/csrc/biome_data.h; the pin against the reference's own code compiled for the CPU
 * (oracle/_ref/libmcgpu_host_ref.so, golden vectors in tests/golden/biome.npz) checks both the
 * arithmetic and that data.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "../slime_b200/csrc/biome_data.h"

/* ---- Xoroshiro128++ (MinecraftGPUNoise.cu:15-73) --------------------------------------------- */

typedef struct { uint64_t lo, hi; } Xr;

static uint64_t rotl(uint64_t x, unsigned b) { return (x << b) | (x >> (64u - b)); }

static uint64_t mix13(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* 64-bit seed to the 128-bit state: lo = seed ^ 0x6a09e667f3bcc909, hi = lo + golden ratio. */
static Xr xr_seed(uint64_t seed) {
    const uint64_t lo = seed ^ 0x6a09e667f3bcc909ull;
    const uint64_t hi = lo + 0x9e3779b97f4a7c15ull;
    Xr r = {mix13(lo), mix13(hi)};
    return r;
}

static uint64_t xr_next(Xr* s) {
    const uint64_t l = s->lo;
    uint64_t h = s->hi;
    const uint64_t out = rotl(l + h, 17) + l;
    h ^= l;
    s->lo = rotl(l, 49) ^ h ^ (h << 21);
    s->hi = rotl(h, 28);
    return out;
}

/* Java nextInt(bound): Lemire's multiply with rejection of the low word. */
static uint32_t xr_next_int(Xr* s, uint32_t n) {
    uint64_t r = (xr_next(s) & 0xffffffffull) * (uint64_t)n;
    if ((uint32_t)r < n) {
        const uint32_t bound = (uint32_t)(-n) % n;
        while ((uint32_t)r < bound) r = (xr_next(s) & 0xffffffffull) * (uint64_t)n;
    }
    return (uint32_t)(r >> 32);
}

static double xr_next_double(Xr* s) { return (double)(xr_next(s) >> 11) * 0x1.0p-53; }

/* ---- improved Perlin noise (MinecraftGPUNoise.cu:75-190) -------------------------------------- */

typedef struct {
    uint8_t perm[257];
    uint8_t y_cell;   /* cell and fraction of the y offset, for samples at y = 0 */
    double ox, oy, oz;
    double y_frac, y_fade;
} Perlin;

static double fade(double t) { return t * t * t * (t * (t * 6.0 - 15.0) + 10.0); }

static void perlin_init(Perlin* p, Xr xr) {
    p->ox = xr_next_double(&xr) * 256.0;
    p->oy = xr_next_double(&xr) * 256.0;
    p->oz = xr_next_double(&xr) * 256.0;
    for (int i = 0; i < 256; ++i) p->perm[i] = (uint8_t)i;
    for (int i = 0; i < 256; ++i) {
        const int j = (int)xr_next_int(&xr, (uint32_t)(256 - i)) + i;
        const uint8_t t = p->perm[i];
        p->perm[i] = p->perm[j];
        p->perm[j] = t;
    }
    p->perm[256] = p->perm[0];
    const double cell = floor(p->oy);
    p->y_cell = (uint8_t)(int)cell;
    p->y_frac = p->oy - cell;
    p->y_fade = fade(p->y_frac);
}

/* Gradient dot product for hash h: two of (x, y, z) with signs. Columns: first operand (0 x,
 * 1 y, 2 z), its sign, second operand, its sign -- the 16 gradient directions of improved noise
 * (12 edges of the cube, 4 repeated). */
static const int8_t GRAD[16][4] = {
    {0, 1, 1, 1}, {0, -1, 1, 1}, {0, 1, 1, -1}, {0, -1, 1, -1},
    {0, 1, 2, 1}, {0, -1, 2, 1}, {0, 1, 2, -1}, {0, -1, 2, -1},
    {1, 1, 2, 1}, {1, -1, 2, 1}, {1, 1, 2, -1}, {1, -1, 2, -1},
    {0, 1, 1, 1}, {1, -1, 2, 1}, {0, -1, 1, 1}, {1, -1, 2, -1},
};

static double grad(uint8_t h, double x, double y, double z) {
    const int8_t* g = GRAD[h & 15];
    const double v[3] = {x, y, z};
    const double a = g[1] > 0 ? v[g[0]] : -v[g[0]];
    const double b = g[3] > 0 ? v[g[2]] : -v[g[2]];
    return a + b;
}

static double lerp(double t, double a, double b) { return a + t * (b - a); }

static double perlin_sample(const Perlin* p, double x, double y, double z) {
    uint8_t hy;
    double ty;
    if (y == 0.0) {
        y = p->y_frac;
        hy = p->y_cell;
        ty = p->y_fade;
    } else {
        y += p->oy;
        const double cy = floor(y);
        y -= cy;
        hy = (uint8_t)(int)cy;
        ty = fade(y);
    }
    x += p->ox;
    z += p->oz;
    const double cx = floor(x), cz = floor(z);
    x -= cx;
    z -= cz;
    const uint8_t hx = (uint8_t)(int)cx, hz = (uint8_t)(int)cz;
    const double tx = fade(x), tz = fade(z);
    const uint8_t* d = p->perm;
    const uint8_t a1 = (uint8_t)(d[hx] + hy), b1 = (uint8_t)(d[hx + 1] + hy);
    const uint8_t a2 = (uint8_t)(d[a1] + hz), b2 = (uint8_t)(d[b1] + hz);
    const uint8_t a3 = (uint8_t)(d[a1 + 1] + hz), b3 = (uint8_t)(d[b1 + 1] + hz);
    double l1 = grad(d[a2], x, y, z), l2 = grad(d[b2], x - 1.0, y, z);
    double l3 = grad(d[a3], x, y - 1.0, z), l4 = grad(d[b3], x - 1.0, y - 1.0, z);
    double l5 = grad(d[a2 + 1], x, y, z - 1.0), l6 = grad(d[b2 + 1], x - 1.0, y, z - 1.0);
    double l7 = grad(d[a3 + 1], x, y - 1.0, z - 1.0), l8 = grad(d[b3 + 1], x - 1.0, y - 1.0, z - 1.0);
    l1 = lerp(tx, l1, l2);
    l3 = lerp(tx, l3, l4);
    l5 = lerp(tx, l5, l6);
    l7 = lerp(tx, l7, l8);
    l1 = lerp(ty, l1, l3);
    l5 = lerp(ty, l5, l7);
    return lerp(tz, l1, l5);
}

/* ---- octaves and climate (MinecraftGPUNoise.cu:196-422) --------------------------------------- */

typedef struct {
    Perlin p;
    double amp, lac;
} Octave;

typedef struct {
    int32_t first, na, nb;
    double amp;
} Noise;

typedef struct {
    Noise n[6];
    Octave oct[46];
} Climate;

enum { SHIFT = 0, TEMP = 1, HUMID = 2, CONT = 3, EROS = 4, WEIRD = 5 };

/* One octave set: two seeds from the parent, then per non-zero amplitude an octave seeded with
 * the hash of "octave_<k>"; lacunarity 2^k, amplitude amp_i * 2^(n-1-i) / (2^n - 1). */
static int octaves_init(Octave* out, Xr* parent, const double* amp, int first, int n) {
    double lac = ldexp(1.0, first);
    double persist = ldexp(1.0, n - 1) / (ldexp(1.0, n) - 1.0);
    const uint64_t lo = xr_next(parent), hi = xr_next(parent);
    int m = 0;
    for (int i = 0; i < n; ++i, lac *= 2.0, persist *= 0.5) {
        if (amp[i] == 0.0) continue;
        const int k = 16 + first + i;
        Xr o = {lo ^ BD_OCTAVE_HASH[k][0], hi ^ BD_OCTAVE_HASH[k][1]};
        perlin_init(&out[m].p, o);
        out[m].amp = amp[i] * persist;
        out[m].lac = lac;
        ++m;
    }
    return m;
}

/* A double-Perlin noise: two octave sets of the same parameters; its amplitude factor
 * 5n / (3(n + 1)) for the n octaves between the first and last non-zero amplitude. */
static void climate_init(Climate* c, uint64_t world_seed, int large) {
    Xr base = xr_seed(world_seed);
    const uint64_t lo = xr_next(&base), hi = xr_next(&base);
    int off = 0;
    for (int s = 0; s < 6; ++s) {
        const BdClimateNoise* d = &BD_CLIMATE[s];
        const int li = large ? 1 : 0;
        Xr xr = {lo ^ d->hash[li][0], hi ^ d->hash[li][1]};
        const int first = d->first_octave[li];
        c->n[s].first = off;
        c->n[s].na = octaves_init(c->oct + off, &xr, d->amp, first, d->octaves);
        c->n[s].nb = octaves_init(c->oct + off + c->n[s].na, &xr, d->amp, first, d->octaves);
        off += c->n[s].na + c->n[s].nb;
        int lead = 0, last = d->octaves;
        while (last > 0 && d->amp[last - 1] == 0.0) --last;
        while (lead < last && d->amp[lead] == 0.0) ++lead;
        const int span = last - lead;
        c->n[s].amp = (double)(5 * span) / (double)(3 * (span + 1));
    }
}

static double octaves_sample(const Octave* o, int n, double x, double y, double z) {
    double v = 0.0;
    for (int i = 0; i < n; ++i) {
        const double f = o[i].lac;
        const double s = perlin_sample(&o[i].p, x * f, y * f, z * f);
        v += o[i].amp * s;
    }
    return v;
}

static double noise_sample(const Climate* c, int s, double x, double y, double z) {
    const Noise* n = &c->n[s];
    const double f = 337.0 / 331.0;
    double v = octaves_sample(c->oct + n->first, n->na, x, y, z);
    v += octaves_sample(c->oct + n->first + n->na, n->nb, x * f, y * f, z * f);
    return v * n->amp;
}

/* ---- depth spline (spline_generated.cuh: a spline of splines over c, e, pv, w) ---------------- */

static float fbits(int32_t b) {
    float f;
    memcpy(&f, &b, 4);
    return f;
}

static float spline_eval(int s, const float* v);

static float spline_value(const int32_t* pt, const float* v) {
    return pt[3] < 0 ? fbits(pt[2]) : spline_eval(pt[3], v);
}

/* Cubic Hermite segments between control points, linear extension outside: with k the position
 * in the segment, value lerp(k, v0, v1) + k(1-k) lerp(k, p, q), the lerps in double. */
static float spline_eval(int s, const float* v) {
    const int32_t* head = BD_SPLINE_HEAD[s];
    const int32_t (*pts)[4] = &BD_SPLINE_PTS[head[1]];
    const int n = head[2];
    const float f = v[head[0]];
    if (f <= fbits(pts[0][0])) return spline_value(pts[0], v) + fbits(pts[0][1]) * (f - fbits(pts[0][0]));
    for (int i = 1; i < n; ++i) {
        const float h = fbits(pts[i][0]);
        if (f > h) continue;
        const float g = fbits(pts[i - 1][0]);
        const float k = (f - g) / (h - g);
        const float l = fbits(pts[i - 1][1]), m = fbits(pts[i][1]);
        const float v0 = spline_value(pts[i - 1], v), v1 = spline_value(pts[i], v);
        const float p = l * (h - g) - (v1 - v0);
        const float q = -m * (h - g) + (v1 - v0);
        const double a = lerp((double)k, (double)v0, (double)v1);
        const float kk = k * (1.0f - k);
        const double b = lerp((double)k, (double)p, (double)q);
        return (float)(a + (double)kk * b);
    }
    return spline_value(pts[n - 1], v) + fbits(pts[n - 1][1]) * (f - fbits(pts[n - 1][0]));
}

static float peaks_valleys(float w) { return -(fabsf(fabsf(w) - 0.6666667f) - 0.33333334f) * 3.0f; }

/* The six quantised climate parameters of quart (x, y, z): {T, H, C, E, depth, W} (x 1e4,
 * truncated), as biome_modern_at computes them (MinecraftGPUNoise.cu:868-913). */
static void climate6(const Climate* c, int32_t xi, int32_t yi, int32_t zi, int32_t np[6]) {
    const double x = (double)xi, z = (double)zi;
    const double px = x + noise_sample(c, SHIFT, x, 0.0, z) * 4.0;
    const double pz = z + noise_sample(c, SHIFT, z, x, 0.0) * 4.0;
    const float cc = (float)noise_sample(c, CONT, px, 0.0, pz);
    const float e = (float)noise_sample(c, EROS, px, 0.0, pz);
    const float w = (float)noise_sample(c, WEIRD, px, 0.0, pz);
    const float in[4] = {cc, e, peaks_valleys(w), w};
    const float off = spline_eval(0, in) + 0.015f;
    const double d0 = 1.0 - ((double)(yi * 4)) / 128.0 - 83.0 / 160.0 + (double)off;
    const float d = (float)d0;
    const float t = (float)noise_sample(c, TEMP, px, 0.0, pz);
    const float h = (float)noise_sample(c, HUMID, px, 0.0, pz);
    np[0] = (int32_t)(10000.0f * t);
    np[1] = (int32_t)(10000.0f * h);
    np[2] = (int32_t)(10000.0f * cc);
    np[3] = (int32_t)(10000.0f * e);
    np[4] = (int32_t)(10000.0f * d);
    np[5] = (int32_t)(10000.0f * w);
}

/* ---- biome parameter tree (MinecraftGPUNoise.cu:650-809) -------------------------------------- */

/* A tree with its patches applied (node words of the tree in `node`). */
typedef struct {
    const BdTree* t;
    uint64_t node[BD_TREE_MAX_NODES];
} Tree;

static Tree g_trees[BD_TREES];

static const Tree* tree_for(int32_t version) {
    int k = -1;
    for (int i = 0; i < BD_TREES; ++i)
        if (version >= BD_TREE[i].version_from) k = i;
    if (k < 0) return 0;
    Tree* t = &g_trees[k];
    if (!t->t) {
        const BdTree* b = &BD_TREE[k];
        memcpy(t->node, b->node, sizeof(uint64_t) * (size_t)b->nnodes);
        for (int i = 0; i < b->npatch; ++i) t->node[b->patch[i][0]] = b->patch[i][1];
        t->t = b;
    }
    return t;
}

static uint64_t node_dist(const Tree* tr, const int32_t np[6], int idx) {
    const BdTree* t = tr->t;
    const uint64_t node = tr->node[idx];
    uint64_t ds = 0;
    for (int i = 0; i < 6; ++i) {
        const int pi = (int)((node >> (8 * i)) & 0xff);
        const int64_t lo = t->param[pi][0], hi = t->param[pi][1], v = np[i];
        const int64_t d = v > hi ? v - hi : v < lo ? lo - v : 0;
        ds += (uint64_t)(d * d);
    }
    return ds;
}

/* Branch-and-bound nearest leaf: children of the node at idx are `order` nodes steps[depth]
 * apart (a subtree that would run past the end descends in place), visited in order; a subtree
 * is entered when its box is strictly closer than the best leaf so far, and a leaf replaces the
 * best only when strictly closer. Returns the leaf's index. */
static int tree_search(const Tree* tr, const int32_t np[6], int depth, int idx, int best, uint64_t ds) {
    const BdTree* t = tr->t;
    if (depth >= t->depth) return idx;
    const int step = t->steps[depth];
    if (idx + step >= t->nnodes) return tree_search(tr, np, depth + 1, idx, best, ds);
    int child = (int)((tr->node[idx] >> 48) & 0xffff);
    for (int k = 0; k < t->order && child < t->nnodes; ++k, child += step) {
        const uint64_t dc = node_dist(tr, np, child);
        if (dc >= ds) continue;
        const int leaf = tree_search(tr, np, depth + 1, child, best, ds);
        const uint64_t dl = leaf == child ? dc : node_dist(tr, np, leaf);
        if (dl < ds) {
            ds = dl;
            best = leaf;
        }
    }
    return best;
}

static int tree_biome(const Tree* t, const int32_t np[6]) {
    const int leaf = tree_search(t, np, 0, 0, 0, ~0ull);
    return (int)((t->node[leaf] >> 48) & 0xff);
}

/* ---- slime test (MinecraftGPUNoise.cu:942-968; Java Random nextInt(10) == 0) ----------------- */

static int is_slime(uint64_t seed, int32_t cx, int32_t cz) {
    const uint32_t x = (uint32_t)cx, z = (uint32_t)cz;
    const uint64_t mix = seed + (uint64_t)(int64_t)(int32_t)(x * x * 0x4c1906u) +
                         (uint64_t)(int64_t)(int32_t)(x * 0x5ac0dbu) +
                         (uint64_t)(int64_t)(int32_t)(z * z) * 0x4307a7ull +
                         (uint64_t)(int64_t)(int32_t)(z * 0x5f24fu);
    uint64_t r = (mix ^ 0x3ad8025full ^ 0x5deece66dull) & 0xffffffffffffull;
    for (;;) {
        r = (r * 0x5deece66dull + 0xb) & 0xffffffffffffull;
        const uint32_t bits = (uint32_t)(r >> 17), val = bits % 10u;
        if (bits - val + 9u <= 0x7fffffffu) return val == 0u;
    }
}

/* ---- exported checkers ---------------------------------------------------------------------- */

void bo_xoroshiro_nextlong(const uint64_t* seeds, int32_t n, int32_t steps, uint64_t* out) {
    for (int32_t i = 0; i < n; ++i) {
        Xr s = xr_seed(seeds[i]);
        for (int32_t j = 0; j < steps; ++j) out[(size_t)i * steps + j] = xr_next(&s);
    }
}

void bo_xperlin_sample(const uint64_t* seeds, const double* xs, const double* ys, const double* zs,
                       int32_t n, double* out) {
    for (int32_t i = 0; i < n; ++i) {
        Perlin p;
        perlin_init(&p, xr_seed(seeds[i]));
        out[i] = perlin_sample(&p, xs[i], ys[i], zs[i]);
    }
}

float bo_depth_spline(const float* v4) { return spline_eval(0, v4); }

void bo_climate6(uint64_t world_seed, int32_t large, const int32_t* xs, const int32_t* ys,
                 const int32_t* zs, int32_t n, int32_t* out6) {
    static Climate c;
    climate_init(&c, world_seed, large);
    for (int32_t i = 0; i < n; ++i) climate6(&c, xs[i], ys[i], zs[i], out6 + (size_t)i * 6);
}

int32_t bo_biome_at(int32_t version, uint64_t world_seed, int32_t large, const int32_t* xs,
                    const int32_t* ys, const int32_t* zs, int32_t n, int32_t* out) {
    const Tree* t = tree_for(version);
    if (!t) return -1;
    static Climate c;
    climate_init(&c, world_seed, large);
    for (int32_t i = 0; i < n; ++i) {
        int32_t np[6];
        climate6(&c, xs[i], ys[i], zs[i], np);
        out[i] = tree_biome(t, np);
    }
    return 0;
}

/* Verdict mask of each candidate centre chunk: bit 0 if a quart of a slime chunk of its 221-cell
 * window is Deep Dark (biome 183) at quart Y -16..0, bit 1 if one is Mushroom Fields (14) at quart
 * Y 16 (MinecraftGPUNoise.cu:978-1074). */
int32_t bo_filter(int32_t version, uint64_t world_seed, int32_t large, const int32_t* ccx,
                  const int32_t* ccz, int32_t n, int32_t flags, int32_t* mask) {
    const Tree* t = tree_for(version);
    if (!t) return -1;
    static Climate c;
    climate_init(&c, world_seed, large);
#pragma omp parallel for schedule(dynamic, 1)
    for (int32_t i = 0; i < n; ++i) {
        int32_t m = 0;
        for (int dx = -8; dx <= 8; ++dx)
            for (int dz = -8; dz <= 8; ++dz) {
                if (dx * dx + dz * dz > 68 || !is_slime(world_seed, ccx[i] + dx, ccz[i] + dz)) continue;
                for (int q = 0; q < 16; ++q) {
                    const int32_t qx = (ccx[i] + dx) * 4 + q / 4, qz = (ccz[i] + dz) * 4 + q % 4;
                    int32_t np[6];
                    if ((flags & 1) && !(m & 1))
                        for (int y = -16; y <= 0; ++y) {
                            climate6(&c, qx, y, qz, np);
                            if (tree_biome(t, np) == 183) {
                                m |= 1;
                                break;
                            }
                        }
                    if ((flags & 2) && !(m & 2)) {
                        climate6(&c, qx, 16, qz, np);
                        if (tree_biome(t, np) == 14) m |= 2;
                    }
                }
            }
        mask[i] = m;
    }
    return 0;
}
