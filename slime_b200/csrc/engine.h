// engine.h -- host-side interface between the C-ABI driver (api.cu) and the kernels.
#pragma once

#include <cstdint>
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

}  // namespace slime
