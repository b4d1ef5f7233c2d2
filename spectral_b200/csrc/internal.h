// Internal interface between the host runtime (capi.cu, batch.cu, server.cu)
// and the kernel files.  Not part of the public ABI.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"

namespace sc {

// One forward photon pass over photons [photon_base, photon_base + photon_count).
struct alignas(16) PhotonParams {
    // what every haze sample reads, in 16-byte groups
    float hz_hw, hz_hh, hz_w, hz_h;   // film width and height halves, film width and height
    float hz_kexp, g, hz_m2g, hz_g2;  // -sigma_t * log2(e); HG g; -2 g; 1 + g^2
    uint32_t width, height, tiles_x, channels;
    unsigned long long* film;         // tile-major int64 film
    uint32_t* flags;                  // per-tile dirty flags, nullable
    const float* zbuf;                // device, nullable
    uint32_t estimator, spectral;
    f3 corner, bu, bv, bdir;          // Beam (lighttrace.rs:116-121)
    Proj proj;                        // Camera::project basis
    uint32_t photon_base, photon_count, seed, max_bounces;
    float sigma_s, sigma_t, max_dist;
    float lambda_min, lambda_range, bin_min, bin_inv_width;
    float scale;
    uint32_t bins;
    const sc_primitive* prims; const sc_plane* planes; const sc_material* mats;
    uint32_t n_prims, n_planes, n_mats;
    const float* cmf;                 // device 3x71 (xbar, ybar, zbar)
    sc_debug_photon* debug;           // debug launches only
    const uint32_t* order;            // nullable: photon i of the launch is photon_base + order[i]
    uint32_t haze_exact;              // 1: haze samples in the CPU crate's operation order (per-photon kernel)
    // Launch constants of the fast haze samples, filled by set_haze_consts()
    // from the fields above just before a launch.
    float hz_sx, hz_sy;               // W / |horizontal|, -H / |vertical|
    float hz_k, hz_kiso;              // sigma_s * 2^scale / 4 * HG numerator / (4 pi); isotropic estimator's
    float hz_inv_sigma_t;             // 1 / sigma_t
};

// Fills the hz_* launch constants of `p` (host side, before every launch).
void set_haze_consts(PhotonParams& p);

// Photon launch: CTAs of 256 threads, `grid` CTAs (grid-stride), warp
// aggregation on/off, register bound (minimum CTAs per SM: 4 or 5), the
// warp-split transport (segments buffered per warp, haze samples processed as
// one converged list) on/off, and the wavelength-ordered dispatch (0 never,
// 1 for spectral films larger than L2, 2 for every spectral film; its scratch
// comes from `pool`, and without a pool it is off).
struct LaunchShape {
    uint32_t block, grid;
    int aggregate;
    int minb;
    int split = 1;
    int order = 1;
    cudaMemPool_t pool = nullptr;
};

// Dirty-tile masks up to this many 32-bit words (16 KB, 524288 tiles) are
// accumulated in shared memory by each photon CTA.
constexpr uint32_t kMaxSmemMaskWords = 4096;
// Dirty-tile mask: one bit per 8x8 tile, 32-bit words.
__host__ __device__ __forceinline__ uint32_t flag_words(uint32_t width, uint32_t height) {
    return (((width + 7u) / 8u) * ((height + 7u) / 8u) + 31u) / 32u;
}

size_t scene_smem_bytes(uint32_t n_prims, uint32_t n_planes, uint32_t n_mats);
uint32_t photon_mask_words(const PhotonParams& p);
cudaError_t launch_photons(const PhotonParams& p, const LaunchShape& shape, cudaStream_t s);
cudaError_t launch_photon_debug(const PhotonParams& p, cudaStream_t s);
cudaError_t launch_photon_count(const PhotonParams& p, unsigned long long* out, uint32_t grid, cudaStream_t s);
// Resident CTAs per SM of kernel `fn` with `block` threads and `smem` bytes of
// dynamic shared memory on the current device; the kernel's shared-memory
// limit is raised the first time a size above 48 KB is asked for, and answers
// are cached per (device, kernel, block, size).
int occupancy_blocks(const void* fn, int block, size_t smem);
int photon_occupancy_blocks(const LaunchShape& shape, bool spectral, size_t smem);

// Photon-beam estimator (beam.cu): same transport, each segment marched in
// deterministic steps with an energy-conserving transverse tent splat.
cudaError_t launch_beam(const PhotonParams& p, const LaunchShape& shape, cudaStream_t s);
int beam_occupancy_blocks(const LaunchShape& shape, bool spectral, size_t smem);
// Instrumented beam pass: out[0..4] += photons, segments, steps, in-frame steps, deposits.
cudaError_t launch_beam_count(const PhotonParams& p, unsigned long long* out, uint32_t grid, cudaStream_t s);

// Host-side scene validation shared by every entry point that uploads a scene.
int check_scene(uint32_t n_prims, uint32_t n_planes, uint32_t n_mats, const sc_primitive* prims,
                const sc_plane* planes, const sc_material* mats);

struct RimParams {
    sc_camera cam;
    uint32_t width, height;
    const sc_primitive* prims; const sc_plane* planes; const sc_material* mats;
    uint32_t n_prims, n_planes, n_mats;
    float* out;                       // 3*w*h
};
cudaError_t launch_rim(const RimParams& p, cudaStream_t s);
cudaError_t launch_rng_draws(uint32_t key, uint32_t seed, uint32_t n, uint32_t* out, cudaStream_t s);
cudaError_t launch_glass_n(uint32_t glass, const float* lambda_nm, uint32_t n, float* out, cudaStream_t s);

// Film reduction: tile-major int64 film -> interleaved f32 XYZ (3*w*h).
struct ReduceParams {
    unsigned long long* film;
    uint32_t* flags;                  // nullable: every tile is read
    float* xyz;
    uint32_t width, height, tiles_x, tiles_y, channels;
    const float* binw;                // 3*channels bin-averaged CMF (spectral films)
    double inv_scale;
};
cudaError_t launch_reduce(const ReduceParams& p, bool drain, cudaStream_t s);

// Up to 8 films of the same geometry (one per GPU of a split scene, peers'
// films mapped into this process); the reduction of their exact sum for tiles
// [tile_begin, tile_end) into p.xyz (p.film and p.flags unused).
constexpr uint32_t kMaxPeerFilms = 8;
struct PeerFilms {
    const unsigned long long* film[kMaxPeerFilms];
    uint32_t n;
};
cudaError_t launch_reduce_peers(const ReduceParams& p, const PeerFilms& films, uint32_t tile_begin, uint32_t tile_end,
                                cudaStream_t s);

// Batched reduction over many films described in device memory.
struct FilmDesc {
    unsigned long long* film; uint32_t* flags; float* xyz; const float* binw;
    uint32_t width, height, tiles_x, tiles_y, channels;
    uint32_t word_begin;  // prefix over films of their dirty-mask words
    uint32_t keep;        // 1: a draining pass leaves this film and its mask as they are (it accumulates)
    double inv_scale;
};
struct DirtyTile { uint32_t film, tile; };
// Two launches after zeroing `count`: a scan of every film's dirty-mask words
// that writes zeros into the images of clean tiles and lists the dirty ones
// (clearing their mask words when draining, except for films marked `keep`),
// then the pipelined reduction of the listed tiles only.  Scratch: `list` with room for every tile of the
// films, one counter.
cudaError_t launch_reduce_many(const FilmDesc* descs, uint32_t n_films, uint32_t total_words, bool drain,
                               uint32_t max_channels, DirtyTile* list, uint32_t* count, cudaStream_t s);

cudaError_t launch_composite_max_y(const float* xyz, const float* surface, uint32_t n_pixels,
                                   uint32_t* out_bits, cudaStream_t s);
cudaError_t launch_composite_select(const float* xyz, const float* surface, uint32_t n_pixels,
                                    uint32_t k, uint32_t* work /*260 u32*/, cudaStream_t s);
cudaError_t launch_to_rgb8(const float* xyz, const float* surface, uint32_t n_pixels, float exposure,
                           uint8_t* out, cudaStream_t s);
cudaError_t launch_gather_rgba8(const float* xyz, const float* surface, uint32_t w, uint32_t h,
                                float k, float kradius, float exposure, uint8_t* out, cudaStream_t s);
cudaError_t launch_synthetic_splat(uint32_t* film, uint32_t w, uint32_t h, uint32_t seed, uint32_t n,
                                   cudaStream_t s);
cudaError_t launch_atomic_resolve(uint32_t* film, float* accum, size_t n, cudaStream_t s);

// Host helpers shared by the runtime objects.
void bin_weights(const float* tables_5x71, uint32_t bins, float lambda_min, float lambda_max, float* out_3xbins);
Proj make_proj(const sc_camera& c);

}  // namespace sc
