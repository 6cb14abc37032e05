/*
 * mcgpu_b200.h -- the biome module's C ABI in libslime_b200.so: the FP64 climate noise, biome
 * lookup and Deep Dark / Mushroom Fields candidate filter on B200 (sm_100a).
 *
 * Same names, signatures, argument meaning and return codes as the reference's biome module
 * (gpu_noise/MinecraftGPUNoise.cu, extern "C" functions at lines 1076-2018; five of them are
 * declared in gpu_noise/mcgpu.h). A frontend that binds that module with ctypes loads this
 * library instead. Every declaration cites the reference function it replaces.
 *
 * Results are bit-exact with the reference's arithmetic: every floating-point operation is one
 * IEEE operation in the reference's source order (the library is built without multiply-add
 * contraction). Biome parameter trees are vendored for every version code the reference accepts,
 * from 1180 (1.18, 1.19.2, 1.19.4, 1.20.6, 1.21.4, 1.21.5 and 26.2); a context for an older
 * version code cannot be created (NULL), as in the reference.
 *
 * Calls are synchronous and serialised with the library's other entry points.
 */
#ifndef MCGPU_B200_H
#define MCGPU_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes (mcgpu.h:14-19). */
enum { MCGPU_OK = 0, MCGPU_ERR_ARG = -1, MCGPU_ERR_CUDA = -2, MCGPU_ERR_ALLOC = -3 };

/* mcgpu_api_version (MinecraftGPUNoise.cu:1076): 1. */
int mcgpu_api_version(void);

/* mcgpu_build_name (MinecraftGPUNoise.cu:1102): a descriptive string. */
const char* mcgpu_build_name(void);

/* mcgpu_modern_recommended_filter_batch (MinecraftGPUNoise.cu:1081): candidates per filter call
 * that fill the current device, a multiple of 32 in [32, 1024]. */
int32_t mcgpu_modern_recommended_filter_batch(void);

/* mcgpu_xoroshiro_nextlong_batch (MinecraftGPUNoise.cu:1107): out[i*steps + j] = the j-th nextLong
 * of Xoroshiro128++ seeded (Minecraft's upgradeSeedTo128bit) with seeds[i]. */
int mcgpu_xoroshiro_nextlong_batch(const uint64_t* seeds, int32_t count, int32_t steps, uint64_t* out);

/* mcgpu_xperlin_sample_batch (MinecraftGPUNoise.cu:1153): one improved-noise sample per (seed,
 * x, y, z), the noise initialised from each seed. */
int mcgpu_xperlin_sample_batch(const uint64_t* seeds, const double* xs, const double* ys, const double* zs,
                               int32_t count, double* out);

/* mcgpu_xperlin_sample_fixed_seed (MinecraftGPUNoise.cu:1207): one noise, many points. */
int mcgpu_xperlin_sample_fixed_seed(uint64_t seed, const double* xs, const double* ys, const double* zs,
                                    int32_t count, double* out);

/* mcgpu_continentalness_noise_fixed_seed (MinecraftGPUNoise.cu:1259): the continentalness
 * double-Perlin noise of a world seed at (x, 0, z). */
int mcgpu_continentalness_noise_fixed_seed(uint64_t world_seed, const double* xs, const double* zs,
                                           int32_t count, double* out);

/* mcgpu_climate5_fixed_seed (MinecraftGPUNoise.cu:1307): {T, H, C, E, W} noise values at shifted
 * (x, z), as doubles. */
int mcgpu_climate5_fixed_seed(uint64_t world_seed, const double* xs, const double* zs, int32_t count,
                              double* out5);

/* mcgpu_climate5_quant_fixed_seed (MinecraftGPUNoise.cu:1356): the same, quantised
 * (int32)(10000.0f * (float)v). */
int mcgpu_climate5_quant_fixed_seed(uint64_t world_seed, const double* xs, const double* zs, int32_t count,
                                    int32_t* out5);

/* mcgpu_climate5_i32_fixed_seed (MinecraftGPUNoise.cu:1405): quantised, integer quart inputs. */
int mcgpu_climate5_i32_fixed_seed(uint64_t world_seed, const int32_t* xs, const int32_t* zs, int32_t count,
                                  int32_t* out5);

/* mcgpu_climate_ctx_create / _query_i32 / _destroy (MinecraftGPUNoise.cu:1461-1542): the
 * climate5_i32 sampling of one world seed behind an opaque handle (NULL on failure). */
void* mcgpu_climate_ctx_create(uint64_t world_seed, int32_t capacity);
int mcgpu_climate_ctx_query_i32(void* handle, const int32_t* xs, const int32_t* zs, int32_t count, int32_t* out5);
void mcgpu_climate_ctx_destroy(void* handle);

/* mcgpu_climate6_i32_fixed_seed (MinecraftGPUNoise.cu:1544): {T, H, C, E, depth, W} of quarts
 * (x, y, z), the depth from the terrain spline and y. */
int mcgpu_climate6_i32_fixed_seed(uint64_t world_seed, const int32_t* xs, const int32_t* ys, const int32_t* zs,
                                  int32_t count, int32_t* out6);

/* mcgpu_climate6_i32_fixed_seed_ex (MinecraftGPUNoise.cu:1988): large != 0 for large biomes. */
int mcgpu_climate6_i32_fixed_seed_ex(uint64_t world_seed, int32_t large, const int32_t* xs, const int32_t* ys,
                                     const int32_t* zs, int32_t count, int32_t* out6);

/* mcgpu_biome20_i32_fixed_seed (MinecraftGPUNoise.cu:1597) and the biome20 context
 * (:1678-1775): biome ids of quarts with the 1.20.6 parameter tree. */
int mcgpu_biome20_i32_fixed_seed(uint64_t world_seed, const int32_t* xs, const int32_t* ys, const int32_t* zs,
                                 int32_t count, int32_t* biome_out);
void* mcgpu_biome20_ctx_create(uint64_t world_seed, int32_t capacity);
int mcgpu_biome20_ctx_query(void* handle, const int32_t* xs, const int32_t* ys, const int32_t* zs, int32_t count,
                            int32_t* biome_out);
void mcgpu_biome20_ctx_destroy(void* handle);

/* mcgpu_modern_ctx_create (MinecraftGPUNoise.cu:1837): a biome context of a Minecraft version
 * code (e.g. 2602 for 26.2) and world seed, for up to `capacity` points per call. NULL for a
 * version code below 1180, capacity <= 0 or no usable device. */
void* mcgpu_modern_ctx_create(int32_t version_code, uint64_t world_seed, int32_t capacity);

/* mcgpu_modern_ctx_create_ex (MinecraftGPUNoise.cu:1966): flags bit 0 = large biomes; other bits
 * give NULL. */
void* mcgpu_modern_ctx_create_ex(int32_t version_code, uint64_t world_seed, int32_t flags, int32_t capacity);

/* mcgpu_modern_ctx_query (MinecraftGPUNoise.cu:1891): biome ids of quarts (x, y, z). */
int mcgpu_modern_ctx_query(void* handle, const int32_t* xs, const int32_t* ys, const int32_t* zs, int32_t count,
                           int32_t* biome_out);

/* mcgpu_modern_ctx_filter_candidates (MinecraftGPUNoise.cu:1923): for each candidate centre chunk,
 * over the slime chunks of its 221-cell AFK window and their 16 quarts each, mask_out bit 0 = a
 * quart is Deep Dark (183) at some quart Y in -16..0 (flags bit 0), bit 1 = a quart is Mushroom
 * Fields (14) at quart Y 16 (flags bit 1). flags must be 1, 2 or 3; count <= capacity. */
int mcgpu_modern_ctx_filter_candidates(void* handle, const int32_t* center_chunk_x, const int32_t* center_chunk_z,
                                       int32_t count, int32_t flags, int32_t* mask_out);

/* mcgpu_modern_ctx_destroy (MinecraftGPUNoise.cu:1952). */
void mcgpu_modern_ctx_destroy(void* handle);

/* Device time of the last filter call on a context (CUDA events on the library's stream) and the
 * number of distinct slime chunks it evaluated. No reference counterpart. */
void slime_b200_biome_last_stats(void* handle, double* kernel_ms, int64_t* unique_chunks);

#ifdef __cplusplus
}
#endif

#endif /* MCGPU_B200_H */
