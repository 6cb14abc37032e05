// engine.h -- host-side interface between the C-ABI driver (api.cu) and the kernels.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "slime_core.cuh"

namespace slime {

constexpr int kHistBins = 222;  // window counts 0..221

// One launch of the general scan over rows [slab_z0, slab_z0 + slab_h) of a search area.
struct ScanArgs {
    const uint64_t* xt;    // xt[i] = x_term(area_x0 - 8 + i), i < width + 16
    const uint64_t* zt;    // zt[j] = z_term(area_z0 - 8 + j) + seed, j < height + 16
    int32_t area_x0, area_z0;  // chunk coordinates of the first centre of the area
    int32_t width, height;     // centres per axis
    int32_t slab_z0, slab_h;   // centre rows of this launch
    int32_t band_h;            // centre rows per tile
    int32_t tiles_x, tiles_z;
    int32_t min_size, max_size, emit_min;
    int64_t rd_min_sq;
    int32_t center_x, center_z;
    Hit* out;
    uint64_t cap;
    unsigned long long* emitted;  // number of hits with count >= emit_min (may exceed cap)
    unsigned int* hist;           // kHistBins counters of every kept centre by count
};

// Tile geometry of the general scan: `narrow` = 256-chunk input tiles, else 1024.
int general_out_width(bool narrow);
cudaError_t launch_general_scan(const ScanArgs& a, bool narrow, int grid, cudaStream_t s);
int general_max_grid(bool narrow);

// Fills xt/zt for an area (x terms, and z terms with the seed folded in).
cudaError_t launch_terms(uint64_t* xt, int32_t x0, int32_t nx, uint64_t* zt, int32_t z0,
                         int32_t nz, int64_t seed, cudaStream_t s);

// Precise AFK scoring (SlimeCore.cpp:654-726 semantics).
struct PreciseArgs {
    int64_t seed;
    ExtChunkResult* sites;
    int32_t n;
    int32_t scan_xz;
    int32_t y_count;           // Y levels scored (1 when Y scan is off)
    const int32_t* y_values;   // y_count
    const uint16_t* weights;   // [16][16][21][21][y_count] block columns per (alignment, chunk, y)
    int32_t platform_y;
    int32_t pack_y;            // obs_count = obs | (y + 1024) << 20
};
cudaError_t launch_precise(const PreciseArgs& a, cudaStream_t s);

// Weight table for precise scoring from per-Y outer/inner radius tables ([y][257], -1 = none).
cudaError_t launch_weight_table(uint16_t* weights, const int16_t* outer, const int16_t* inner,
                                int32_t y_count, cudaStream_t s);

// Fills out[i] = is_slime(seed, x[i], z[i]).
cudaError_t launch_predicate(int64_t seed, const int64_t* x, const int64_t* z, uint8_t* out,
                             int64_t n, cudaStream_t s);

// ---- band engine (scan_band.cu) ------------------------------------------------------------

// One launch of the band engine over tiles [tile_begin, tile_end) of one band group.
// The phase axis (u) is x, or z when `transposed`; the band axis (v) is the other one.
struct BandArgs {
    const uint64_t* ct;      // column terms (phase axis, no seed), ncols = width_u + 16 entries
    int64_t ncols;
    const uint32_t* rt;      // row-term records of this band group (see row_terms_kernel)
    int32_t vrows;           // base input rows = vbase + 16
    int32_t vbase;           // base centre rows = min(2^17, height_v)
    int32_t ubase;           // base centre columns owned = min(2^17, width_u)
    int64_t width_u, height_v;
    int32_t j0, nb;          // first band of the group and bands in it (<= 32)
    int32_t u_tiles, v_tiles;
    int32_t band_h;
    int64_t tile_begin, tile_end;
    int32_t min_size, max_size;
    int64_t rd_min_sq;
    int32_t area_x0, area_z0, center_x, center_z;
    int32_t transposed;
    Hit* out;
    uint64_t cap;
    unsigned long long* emitted;
    unsigned int* overflow;
    uint32_t one;            // the value 1 (run time): band adds as multiply-adds when mad_add
    int32_t mad_add;
    int32_t indep;           // 1: independent bands (no shared LCG work, one X phase)
    int32_t exact;           // 1: bit-sliced exact counts of every centre (no bounds)
    uint32_t poll_limit;     // polls of a row-term mbarrier before the CTA gives up (bit 4 of overflow)
    unsigned int* hist;      // if set: kHistBins counters of every centre in range, by count
    int32_t emit_min;        // centres in range are appended to `out` only from this count on
    int64_t row_stride;      // input rows between band j and band j + 1 (2^17 with the shared LCG;
                             // grouped bands: between group g and group g + 1)
    int32_t groups;          // grouped bands (G > 0): band m = copy * G + group, copies 2^17 apart
    int32_t pad_;
};

// Tiling of one band search (band_driver.cu): axes (u = phase axis, v = band axis), phases,
// bands, base sizes and tiles, as the band kernels expect them.
struct BandGeom {
    bool indep, transposed;
    int32_t groups;  // grouped bands: G groups of nJ / G copies (0 otherwise)
    int64_t width_u, height_v, nI, nJ, stride, ngroups;
    int32_t ubase, vbase, vrows, vrows_alloc, band_h;
    int64_t u_tiles, v_tiles, pairs, tiles;
};
// Band modes of band_geometry.
constexpr int kBandShared = 0, kBandIndep = 1, kBandGrouped = 2;
BandGeom band_geometry(int64_t W, int64_t H, int mode, int sm_count);

size_t band_smem_bytes();
int band_tile_out_w();
int band_max_bands();
cudaError_t band_prepare();
cudaError_t launch_band_scan(const BandArgs& a, int grid, cudaStream_t s);
// Tiles of many band searches of one launch class (band_class: band mode, survivor lists, exact
// counts; kBandClasses of them) in one persistent launch: args[i] (device) describes search i,
// prefix[i] (device, nsearch + 1 entries, increasing from any start) is its first tile in the
// launch, *head (device, zeroed) is the tile queue. Item i runs tiles tile_begin .. tile_begin +
// prefix[i+1] - prefix[i] - 1 of its search (tile_end is unused).
constexpr int kBandClasses = 9;
int band_class(const BandArgs& a);
cudaError_t launch_band_batch(const BandArgs* args, const int64_t* prefix, int32_t nsearch,
                              unsigned long long* head, int cls, int grid, cudaStream_t s);
// Uploads band work items of any classes (reordered by class in place) and runs them: one
// persistent launch per class present. args_dev / prefix_dev hold items.size() (+1) entries,
// heads_dev kBandClasses counters. Adds the launches made to *launches.
cudaError_t run_band_items(std::vector<BandArgs>& items, BandArgs* args_dev, int64_t* prefix_dev,
                           unsigned long long* heads_dev, int grid, cudaStream_t s, int64_t* launches);
// Words of a row-term record: per-band low bits (independent and grouped bands) or shared ones.
int band_row_words(bool split);
cudaError_t launch_band_terms(uint64_t* ct, int32_t col_first, int32_t ncols, uint32_t* rt,
                              int32_t vrows_alloc, int32_t vrows, int32_t nj, int32_t row_first,
                              int64_t row_limit, int64_t row_stride, int64_t seed, bool transposed,
                              bool indep, int32_t groups, cudaStream_t s);

// ---- rare redraw correction (rare_fix.cu) ------------------------------------------------

struct FixArgs {
    int32_t area_x0, area_z0;
    int64_t width, height;
    int64_t rd_min_sq;
    int32_t center_x, center_z;
    int32_t min_size, max_size;
    Hit* fixed;
    unsigned long long* fixed_count;
    uint64_t cap;
    unsigned int* error;
    // If set: per count, the change the fix-up makes to a scan histogram of first-draw counts
    // (-1 at a fixed centre's first-draw count, +1 at its exact count, each when in range).
    int* hist_delta;
};

void rare_target_table(std::vector<uint64_t>& targets, std::vector<uint32_t>& offsets);
cudaError_t launch_rare_scan(const uint64_t* targets, const uint32_t* offsets, int64_t seed,
                             int32_t z_first, int32_t nz, int32_t x_first, int32_t nx, int2* out,
                             uint32_t cap, unsigned int* count, cudaStream_t s);
cudaError_t launch_fixup(const int2* rare, int32_t nrare, int64_t seed, const FixArgs& f,
                         cudaStream_t s);
// Marks hits whose window holds a rare chunk (count -1). With `sorted_by_x` the rare list is in
// ascending x and each hit binary-searches it; otherwise every hit scans the whole list.
cudaError_t launch_filter_hits(Hit* hits, int64_t n, const int2* rare, int32_t nrare, bool sorted_by_x,
                               cudaStream_t s);

}  // namespace slime
