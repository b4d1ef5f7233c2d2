/*
 * spectral_cuda.h -- C ABI of the B200 (sm_100a) spectral forward / volumetric /
 * camera-tracer path.
 *
 * This is the drop-in boundary for the reference renderer's `spectral-gpu` crate
 * (TSavo/spectral, Rust + wgpu).  Every entry point names the reference item it
 * replaces (file:line in the reference checkout).  Conventions:
 *   - every call returns an int status: SC_OK (0) or a negative SC_E_* code;
 *     sc_last_error() returns a thread-local message for the last failure;
 *   - handles are opaque; each handle owns one CUDA stream; calls on one handle
 *     are serialised by a mutex, different handles may be used concurrently;
 *   - host buffers are caller-allocated; sizes are in elements unless stated;
 *   - no C++ exception crosses the ABI;
 *   - the library never falls back to a CPU path: without a usable sm_100 device
 *     sc_ctx_create fails with SC_E_NODEVICE.
 *
 * Films are 64-bit fixed point (value = count / 2^scale_log2): exact and
 * independent of the order in which splats land.
 */
#ifndef SPECTRAL_CUDA_H
#define SPECTRAL_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SC_OK 0
#define SC_E_INVALID (-1)   /* bad argument (null pointer, size, range) */
#define SC_E_CUDA (-2)      /* CUDA runtime error (message has the CUDA string) */
#define SC_E_NOMEM (-3)     /* device allocation failed or HBM budget exceeded */
#define SC_E_LIMIT (-4)     /* scene or film exceeds a documented compile-time limit */
#define SC_E_TIMEOUT (-5)   /* a bounded device-side wait gave up */
#define SC_E_STATE (-6)     /* call not valid in the handle's current state */
#define SC_E_NODEVICE (-7)  /* no usable device: none present, none at that index, or not sm_100 */

/* ---- limits ------------------------------------------------------------ */
#define SC_MAX_PRIMS 64
#define SC_MAX_PLANES 256
#define SC_MAX_BINS 256

/* ---- plain data records ------------------------------------------------ */
/* Scene records, byte-identical to spectral-gpu/src/upload.rs:7-32
 * (GpuPrimitive 32 B, GpuMaterial 16 B, GpuPlane 16 B). */
typedef struct { float center[3]; float radius; uint32_t plane_start, plane_count, kind, material; } sc_primitive; /* kind 0 sphere, 1 convex solid */
typedef struct { float reflectance; uint32_t glass, kind, pad; } sc_material; /* kind 0 Lambertian, 1 dielectric; glass 0 BK7, 1 SF11, 2 water, 3 fused silica */
typedef struct { float normal[3]; float d; } sc_plane;

/* spectral-core/src/lighttrace.rs:116-121 (Beam). */
typedef struct { float corner[3], u[3], v[3], dir[3]; } sc_beam;
/* spectral-core/src/camera.rs:5-10 (Camera, the view_basis of camera.rs:36-38). */
typedef struct { float origin[3], lower_left[3], horizontal[3], vertical[3]; } sc_camera;
/* spectral-gpu/src/vol_photons.rs:256-267 (VolWeights). */
typedef struct { float sigma_s, sigma_t, g; } sc_vol_weights;
/* spectral-gpu/src/vol_photons.rs:85-93 (DebugPhotonGpu, 304 bytes). */
typedef struct { uint32_t num_states; float lambda; uint32_t pad0, pad1; float states[18][4]; } sc_debug_photon;

/* Film options beyond the reference: spectral binning and band.  Zero-initialise
 * and set what you need; zeros select the reference's film (XYZ, 380-730 nm,
 * 8 bounces, the point estimator). */
typedef struct {
    uint32_t bins;          /* 0: XYZ film (3 channels, the reference film); N>0: N spectral bins */
    float lambda_min;       /* emission band start, nm (0 -> 380) */
    float lambda_max;       /* emission band end, nm (0 -> 730) */
    uint32_t max_bounces;   /* bounce loop length (0 -> 8, volume.rs:126) */
    uint32_t scale_log2;    /* fixed-point scale 2^k (0 -> 32) */
    uint32_t estimator;     /* 0 point estimator (volume.rs:99-168), 1 legacy isotropic (volume.rs:22-85),
                               2 photon-beam estimator (volume.rs:170-329; photon films and the
                               device-pointer trace only; deposits are small: use scale_log2 >= 40),
                               3 point estimator with free-flight sampling (no counterpart in the
                               reference): the 4 distances of a segment follow sigma_t exp(-sigma_t t)
                               restricted to the segment, weighted by 1/pdf: the same integral */
    uint32_t haze_exact;    /* 0: haze samples (camera projection, distance, transmittance, phase) in
                               fast f32 arithmetic, within 2e-3 relative L1 of the CPU crate's film
                               (the bar the tests hold it to);
                               1: in the CPU crate's operation order (volume.rs:130-150), film cells
                               within a few fixed-point quanta of it, slower.  Photon paths, the RNG
                               stream and the film's integer sums are the same either way.  Photon
                               films and the device-pointer and allocation-free traces only: batches
                               and the server run the fast samples. */
} sc_film_options;

typedef struct sc_batch sc_batch;
typedef struct sc_server sc_server;

/* ---- errors / context (spectral-gpu/src/lib.rs:21-41 GpuContext::new) ---- */
const char* sc_last_error(void);
const char* sc_version(void);
typedef struct sc_ctx sc_ctx;
/* tables: the 5x71 sensor table [xbar;71][ybar;71][zbar;71][d65;71][a;71]
 * (spectral-gpu/src/data.rs:12-22 sample_tables). */
int sc_ctx_create(int device, const float* tables_5x71, sc_ctx** out);
int sc_ctx_destroy(sc_ctx* ctx);
int sc_ctx_synchronize(sc_ctx* ctx);
/* Parse the 5-column sensor CSV shipped with the library into a 5x71 table. */
int sc_load_sensor_tables(const char* csv_path, float* out_5x71);

/* ---- host helpers that mirror spectral-core constructors ---------------- */
/* Camera::look_at (spectral-core/src/camera.rs:15-27). */
int sc_camera_look_at(const float origin[3], const float target[3], const float up[3],
                      float vfov_deg, float aspect, sc_camera* out);
/* camera_proj_params (spectral-gpu/src/vol_photons.rs:100-115): out[16] =
 * (origin, 0), (horizontal unit, |horizontal|), (vertical unit, |vertical|),
 * (origin - horizontal/2 - vertical/2 - lower_left, 0). */
int sc_camera_proj_params(const sc_camera* cam, float out[16]);
/* Glass::n (spectral-core/src/sellmeier.rs:28-44), f64 internally. */
float sc_glass_n(uint32_t glass, float lambda_nm);
/* Glass::n over an array on the host: out[i] = sc_glass_n(glass, lambda_nm[i]).
 * glass 0 BK7, 1 SF11, 2 water, 3 fused silica; others return SC_E_INVALID. */
int sc_glass_n_many(uint32_t glass, const float* lambda_nm, size_t n, float* out);
/* The same with the kernels' own device code over device arrays, on `stream`
 * (asynchronous; n <= 2^31). */
int sc_glass_n_device(sc_ctx* ctx, uint32_t glass, const float* lambda_nm_dev, size_t n, float* out_dev,
                      void* stream);
/* Device RNG stream: n draws of PathRng(key, seed).next_u32() computed on the GPU
 * into host `out` (the kernel of spectral-gpu/tests/rng_parity.rs:4-16). */
int sc_rng_draws(sc_ctx* ctx, uint32_t key, uint32_t seed, uint32_t n, uint32_t* out);
/* dsotm_scene (spectral-gpu/src/vol_photons.rs:188-222): writes 1 primitive,
 * 5 planes, 1 material, the beam and the camera for the given aspect. */
int sc_dsotm_scene(float aspect, sc_primitive* prim, sc_plane* planes5, sc_material* mat,
                   sc_beam* beam, sc_camera* cam);

/* ---- photon film: GpuPhotonFilm (spectral-gpu/src/vol_photons.rs:228-851) */
typedef struct sc_photon_film sc_photon_film;
/* GpuPhotonFilm::new (vol_photons.rs:275-573).  zbuffer: host, width*height
 * floats, or NULL for no occlusion.  opts may be NULL (reference XYZ film). */
int sc_photon_film_create(sc_ctx* ctx, const sc_primitive* prims, uint32_t n_prims,
                          const sc_plane* planes, uint32_t n_planes,
                          const sc_material* mats, uint32_t n_mats, float background,
                          const sc_camera* cam, const sc_beam* beam, uint32_t width,
                          uint32_t height, uint32_t n_photons, uint32_t seed, float max_dist,
                          const sc_vol_weights* weights, const float* zbuffer,
                          const sc_film_options* opts, sc_photon_film** out);
int sc_photon_film_destroy(sc_photon_film* f);
/* trace_and_resolve (vol_photons.rs:582-585): photons [0, n_photons). */
int sc_photon_film_trace_and_resolve(sc_photon_film* f, uint32_t n_photons, uint32_t seed);
/* trace_chunked (vol_photons.rs:590-598). */
int sc_photon_film_trace_chunked(sc_photon_film* f, uint32_t total_photons, uint32_t seed);
/* dispatch_photons (vol_photons.rs:633-635): photons [photon_base, n_photons), asynchronous. */
int sc_photon_film_dispatch(sc_photon_film* f, uint32_t photon_base, uint32_t n_photons, uint32_t seed);
/* trace_debug (vol_photons.rs:727-779): records photons [0, debug_count); the
 * film is not touched.  out: debug_count records. */
int sc_photon_film_trace_debug(sc_photon_film* f, uint32_t n_photons, uint32_t seed,
                               uint32_t debug_count, sc_debug_photon* out);
/* set_spectral / spectral (vol_photons.rs:658-666). */
int sc_photon_film_set_spectral(sc_photon_film* f, int on);
int sc_photon_film_get_spectral(sc_photon_film* f, int* on);
/* set the camera used by the next trace and by the rim pass. */
int sc_photon_film_set_camera(sc_photon_film* f, const sc_camera* cam);
/* recompute_surface (vol_photons.rs:685-714): rim pass for `cam` (NULL: current camera). */
int sc_photon_film_recompute_surface(sc_photon_film* f, const sc_camera* cam);
/* surface (vol_photons.rs:717-719): out 3*w*h interleaved XYZ. */
int sc_photon_film_read_surface(sc_photon_film* f, float* out);
/* accum (vol_photons.rs:807-809): out 3*w*h interleaved XYZ f32 (film / 2^scale,
 * sensor-reduced for spectral films). */
int sc_photon_film_read_accum(sc_photon_film* f, float* out);
/* raw film: int64 in row-major [h][w][channels] (channels = 3 or bins). */
int sc_photon_film_read_raw(sc_photon_film* f, int64_t* out);
/* clear_film (vol_photons.rs:800-804): zero the 64-bit film (it is the accumulator). */
int sc_photon_film_clear(sc_photon_film* f);
/* auto_expose, auto_expose_p997, to_rgb8 (vol_photons.rs:823-850), on the device. */
int sc_photon_film_auto_expose(sc_photon_film* f, float scale, float* exposure);
int sc_photon_film_auto_expose_p997(sc_photon_film* f, float* exposure);
int sc_photon_film_to_rgb8(sc_photon_film* f, float exposure, uint8_t* out_rgb);
/* Viewer reconstruction (spectral-viewer/src/main.rs:132-173): normalized
 * Gaussian gather of radius kradius over the accumulated film scaled by
 * target_n / total_photons, plus the rim surface, XYZ->sRGB, Reinhard,
 * gamma 1/2.2.  out: w*h RGBA8. */
int sc_photon_film_gather_rgba8(sc_photon_film* f, uint64_t total_photons, float target_n,
                                float kradius, float exposure, uint8_t* out_rgba);
int sc_photon_film_dims(sc_photon_film* f, uint32_t* width, uint32_t* height, uint32_t* channels);
/* Replace the scene records, camera and beam (host -> device upload on the
 * film's stream); the film keeps accumulating.  Same limits as create. */
int sc_photon_film_set_scene(sc_photon_film* f, const sc_primitive* prims, uint32_t n_prims,
                             const sc_plane* planes, uint32_t n_planes, const sc_material* mats,
                             uint32_t n_mats, const sc_camera* cam, const sc_beam* beam);
/* Device buffers of the film (tile-major int64 cells and the dirty-tile mask),
 * for collectives over several GPUs: films of disjoint photon ranges add up
 * exactly.  Valid until the film is destroyed. */
int sc_photon_film_device_buffers(sc_photon_film* f, void** film_dev, size_t* film_bytes, void** flags_dev,
                                  size_t* flag_bytes, void** stream);
/* Mark every tile as lit (after another process added its film into this one). */
int sc_photon_film_mark_all_dirty(sc_photon_film* f);
/* Work counters of photons [photon_base, photon_base+count) without touching
 * the film: out[0..3] = photons, path segments, in-frame haze samples (film
 * splats), surface scatters. */
int sc_photon_film_trace_stats(sc_photon_film* f, uint32_t photon_base, uint32_t count, uint32_t seed,
                               uint64_t out[4]);

/* ---- camera tracer: GpuTracer (spectral-gpu/src/lib.rs:165-389) -------- */
typedef struct sc_tracer sc_tracer;
/* Extensions beyond the reference (zero = reference behaviour). */
typedef struct {
    uint32_t max_depth;        /* 0 -> 8 (tracer.rs:26) */
    uint32_t rr_start;         /* Russian roulette once this many scatters happened (0 = off) */
    float emitter_center[3];   /* spherical emitter (radius 0 = none) */
    float emitter_radius;
    float emitter_scale;       /* emitted radiance = scale * illuminant(lambda) */
    uint32_t wave_bounces;     /* bounces run as compacted wavefront stages before the in-place tail
                                  (0 -> 2); the image is the same for any value */
    uint32_t chains;           /* waves in flight at once, one stream each (0 -> 3, at most 4) */
    uint32_t wave_paths_log2;  /* paths per wave 2^k (0 -> 22; 12..24); scheduling only, as above */
} sc_tracer_options;
/* GpuTracer::new (lib.rs:179-187), CpuTracer::new (tracer.rs:20-37).
 * illuminant 0 D65, 1 A; has_horizon/horizon: Scene::horizon (scene.rs:25-28). */
int sc_tracer_create(sc_ctx* ctx, const sc_primitive* prims, uint32_t n_prims,
                     const sc_plane* planes, uint32_t n_planes, const sc_material* mats,
                     uint32_t n_mats, float background, int has_horizon, float horizon,
                     const sc_camera* cam, uint32_t width, uint32_t height,
                     uint32_t illuminant, uint32_t seed, const sc_tracer_options* opts,
                     sc_tracer** out);
int sc_tracer_destroy(sc_tracer* t);
/* accumulate (lib.rs:307-321): spp more samples per pixel; sample indices
 * continue across calls as in CpuTracer::accumulate (tracer.rs:115-141).
 * Asynchronous. */
int sc_tracer_accumulate(sc_tracer* t, uint32_t spp);
/* read_xyz (lib.rs:324-357): per-pixel mean XYZ, out 3*w*h. */
int sc_tracer_read_xyz(sc_tracer* t, float* out);
/* set_camera (lib.rs:376-383). */
int sc_tracer_set_camera(sc_tracer* t, const sc_camera* cam);
/* clear_accum (lib.rs:386-389): zero the sum and the sample count. */
int sc_tracer_clear_accum(sc_tracer* t);
int sc_tracer_dims(sc_tracer* t, uint32_t* width, uint32_t* height);
/* set_spectral (lib.rs:369-372): on (the default) refracts at the hero
 * wavelength; off uses n(550 nm) for every path (trace.wgsl:477-480).  The
 * accumulation is kept, as in the reference. */
int sc_tracer_set_spectral(sc_tracer* t, int on);
/* Trace only image rows [row_begin, row_end) in later accumulate calls (all
 * rows by default; no counterpart in the reference).  A pixel's samples are
 * keyed by the pixel and sample index, so a row renders the same whichever
 * rows are traced with it: GPUs that own bands of rows gather their bands into
 * the full image with no reduction.  Rows outside the range keep their sums. */
int sc_tracer_set_rows(sc_tracer* t, uint32_t row_begin, uint32_t row_end);
/* The CUDA stream (cudaStream_t) all of this tracer's work runs on, for callers
 * that order or time their own work against it.  Owned by the tracer. */
int sc_tracer_stream(sc_tracer* t, void** stream);
/* paths of the last accumulate and path segments traced since creation. */
int sc_tracer_last_stats(sc_tracer* t, uint64_t* paths, uint64_t* segments);

/* ---- atomic film: AtomicFilm (spectral-gpu/src/film.rs:40-305) --------- */
typedef struct sc_atomic_film sc_atomic_film;
int sc_atomic_film_create(sc_ctx* ctx, uint32_t width, uint32_t height, sc_atomic_film** out);
int sc_atomic_film_destroy(sc_atomic_film* f);
/* splat (film.rs:174-192): vol_splat.wgsl semantics (u32, x4096, truncation). */
int sc_atomic_film_splat(sc_atomic_film* f, uint32_t seed, uint32_t n_splats);
/* read_film_raw (film.rs:197-214): out 3*w*h u32. */
int sc_atomic_film_read_raw(sc_atomic_film* f, uint32_t* out);
/* resolve (film.rs:218-224) + accum (film.rs:239-241). */
int sc_atomic_film_resolve(sc_atomic_film* f);
int sc_atomic_film_read_accum(sc_atomic_film* f, float* out);
int sc_atomic_film_clear_film(sc_atomic_film* f);
int sc_atomic_film_clear_accum(sc_atomic_film* f);
/* auto_expose_accum (film.rs:262-270): max(scale / max(max Y, 1e-6), 1). */
int sc_atomic_film_auto_expose_accum(sc_atomic_film* f, float scale, float* exposure);
/* to_rgb8 (film.rs:243-258): XYZ -> linear sRGB -> tonemap_to_u8, out 3*w*h bytes. */
int sc_atomic_film_to_rgb8(sc_atomic_film* f, float exposure, uint8_t* out);
/* The CUDA stream (cudaStream_t) this film's work runs on, for callers that
 * order or time their own work against it.  Owned by the film. */
int sc_atomic_film_stream(sc_atomic_film* f, void** stream);
/* check_determinism (film.rs:282-305): returns SC_OK and *first_diff=-1 when identical. */
int sc_atomic_film_check_determinism(sc_ctx* ctx, uint32_t width, uint32_t height, uint32_t seed,
                                     uint32_t n_splats, int64_t* first_diff);

/* ---- screen caustics and z-buffer (spectral-core/src/lighttrace.rs) ----- */
/* Screen rectangle corner + s*u + r*v, s and r in [0,1) (lighttrace.rs:27-34). */
typedef struct { float corner[3], u[3], v[3]; } sc_screen;
/* lighttrace::trace (lighttrace.rs:157-166): photons [0, n_photons) from the
 * beam, wavelengths uniform over [lambda_min, lambda_max) (opts; NULL = the
 * visible band, 8 bounces), bilinear XYZ deposit into Screen::sum.  out_sum:
 * 3*width*height floats, row 0 at the top (r = 1). */
int sc_lighttrace(sc_ctx* ctx, const sc_primitive* prims, uint32_t n_prims, const sc_plane* planes,
                  uint32_t n_planes, const sc_material* mats, uint32_t n_mats, const sc_screen* screen,
                  uint32_t width, uint32_t height, const sc_beam* beam, uint32_t n_photons, uint32_t seed,
                  const sc_film_options* opts, float* out_sum);
/* Z-buffer of spectral-core/examples/prism_on_plane.rs:125-160: per pixel the
 * ray distance of the nearer of the scene hit and the floor rectangle hit
 * (floor may be NULL) along the primary ray through the pixel centre, +INF
 * where nothing is hit.  out: width*height floats, the zbuffer input of
 * sc_photon_film_create. */
int sc_scene_zbuffer(sc_ctx* ctx, const sc_primitive* prims, uint32_t n_prims, const sc_plane* planes,
                     uint32_t n_planes, const sc_material* mats, uint32_t n_mats, const sc_screen* floor,
                     const sc_camera* cam, uint32_t width, uint32_t height, float* out);

/* ---- device-pointer entry points (zero-copy; caller owns device memory) -- */
/* One plain launch of the forward photon + haze kernel over photons
 * [photon_base, photon_base+count) into a device film the caller allocated
 * with sc_film_bytes().  All pointers are device pointers; stream may be 0.
 * Films hold at most 2^28 pixels, as film objects do (SC_E_LIMIT). */
typedef struct {
    const sc_primitive* prims; uint32_t n_prims;
    const sc_plane* planes; uint32_t n_planes;
    const sc_material* mats; uint32_t n_mats;
    sc_camera cam; sc_beam beam; sc_vol_weights weights;
    uint32_t width, height, seed, spectral;
    float max_dist;
    sc_film_options opts;
    const float* zbuffer;   /* device, or NULL */
} sc_trace_desc;
size_t sc_film_bytes(uint32_t width, uint32_t height, uint32_t channels);
size_t sc_film_flag_bytes(uint32_t width, uint32_t height);
int sc_trace_photons_device(sc_ctx* ctx, const sc_trace_desc* desc, uint32_t photon_base,
                            uint32_t count, void* film_dev, uint32_t* flags_dev, void* stream);
/* Work counters for a device-pointer desc, accumulated into out_dev (device
 * uint64, zero it first): point / isotropic estimators 4 counters (photons,
 * segments, in-frame haze samples, scatters; see sc_photon_film_trace_stats),
 * beam estimator 5 (photons, segments, march steps, in-frame steps, footprint
 * pixels deposited). */
int sc_trace_stats_device(sc_ctx* ctx, const sc_trace_desc* desc, uint32_t photon_base, uint32_t count,
                          uint64_t* out_dev, void* stream);
/* Sensor reduction of a device film to interleaved f32 XYZ (3*w*h, device);
 * drain != 0 also zeroes the film and its tile flags (ready for the next pass). */
int sc_sensor_reduce_device(sc_ctx* ctx, uint32_t width, uint32_t height, uint32_t channels,
                            float lambda_min, float lambda_max, uint32_t scale_log2,
                            void* film_dev, uint32_t* flags_dev, float* xyz_dev, int drain,
                            void* stream);

/* ---- one scene split over GPUs (no counterpart in the reference, which runs
 * one GPU) --------------------------------------------------------------- */
/* Every GPU traces its range of photons into its own device film
 * (sc_trace_photons_device); each then reduces its own band of image rows
 * from the SUM of all the films, reading the other GPUs' films as peer memory
 * (NVLink), so no film is summed into one or sent whole: a GPU reads 1/N of
 * every film, and the XYZ bands (a few MB) are gathered.  The int64 sum is
 * exact: each band is bit-identical to the same rows of the image of one film
 * that traced every photon.
 *
 * sc_ipc_export: a CUDA IPC handle (64 bytes) of the allocation holding
 * dev_ptr (e.g. a torch tensor's storage) and dev_ptr's offset in it, to pass
 * to the other processes.  sc_ipc_import: map another process's allocation
 * into this context (peer access enabled as needed); *dev_ptr = its base +
 * offset.  sc_ipc_close: unmap it (the same offset).  The exporting process
 * must keep the memory alive until every importer has closed it. */
int sc_ipc_export(sc_ctx* ctx, const void* dev_ptr, unsigned char handle[64], size_t* offset);
int sc_ipc_import(sc_ctx* ctx, const unsigned char handle[64], size_t offset, void** dev_ptr);
int sc_ipc_close(sc_ctx* ctx, void* dev_ptr, size_t offset);
/* The sensor reduction (as sc_sensor_reduce_device, without draining) of the
 * sum of n_films device films of the same geometry (films_dev: a host array
 * of 1..8 device pointers, this GPU's own film and mapped peer films, 16-byte
 * aligned) for image rows [row_begin, row_end) only: row_begin a multiple of
 * 8, row_end a multiple of 8 or the height.  Writes those rows of the full
 * interleaved XYZ image at xyz_dev (3*w*h floats).  Every film must be
 * complete (all ranks' traces finished) before the call is ordered; the films
 * are read, not changed. */
int sc_sensor_reduce_peers(sc_ctx* ctx, uint32_t width, uint32_t height, uint32_t channels,
                           float lambda_min, float lambda_max, uint32_t scale_log2,
                           const int64_t* const* films_dev, uint32_t n_films, uint32_t row_begin,
                           uint32_t row_end, float* xyz_dev, void* stream);

/* ---- allocation-free render (no counterpart in the reference) ----------
 * For callers that cannot allocate device memory: hosts whose framework owns
 * all device memory through its own pool (a raw cudaMalloc would bypass it and
 * cudaFree synchronises the whole device) and render loops that must never
 * block on an allocation.  Traces photons [photon_base, photon_base+count) of
 * the scene in `desc` (scene records in device memory, as for
 * sc_trace_photons_device) and writes the f32 XYZ image (3*w*h floats) to the
 * caller's device buffer `xyz_dev` on `stream`.  It calls no cudaMalloc /
 * cudaFree: its scratch (64-bit film, tile mask, colour-matching table, bin
 * weights) lives in static device arrays that every GPU loading this library
 * holds until the process exits; the table and bin weights travel as a kernel
 * parameter, so `tables_5x71` is read only during the call.  Estimators 0
 * (point), 1 (isotropic) and 3 (free-flight); others return SC_E_INVALID.
 * Limit: (width padded to 8) * (height padded to 8) * channels <=
 * SC_NOALLOC_MAX_FILM_CELLS (16 MiB of int64 cells; e.g. 640x360 XYZ, or
 * 256x256 with 32 bins); larger films return SC_E_LIMIT.  The first call on a
 * device looks up the arrays' device addresses (once per device); make that
 * first call before any stream capture.  Every call clears the scratch it
 * reads, but all calls share it: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised. */
#define SC_NOALLOC_MAX_FILM_CELLS (1u << 21)
#define SC_NOALLOC_MAX_MASK_WORDS 4096u
int sc_trace_xyz_noalloc(const float* tables_5x71, const sc_trace_desc* desc, uint32_t photon_base,
                         uint32_t count, float* xyz_dev, void* stream);

/* ---- batched uneven workload (no counterpart in the reference) ----------
 * Many independent scenes with different photon budgets, film sizes and bins
 * traced by ONE persistent launch (warps steal photon chunks, largest scene
 * first), then one persistent drain + sensor reduction over every film; the
 * pair is captured in a CUDA graph and replayed.  Photon i of a scene is keyed
 * by its index inside that scene, so each film is bit-identical to the film of
 * a plain per-scene launch. */
#define SC_BATCH_MAX_PRIMS 4
#define SC_BATCH_MAX_PLANES 16
typedef struct {
    uint32_t n_prims, n_planes, n_mats, spectral;   /* spectral: 1 n(lambda), 0 n(550 nm) */
    sc_primitive prims[SC_BATCH_MAX_PRIMS];
    sc_plane planes[SC_BATCH_MAX_PLANES];
    sc_material mats[SC_BATCH_MAX_PRIMS];
    sc_camera cam;
    sc_beam beam;
    sc_vol_weights weights;
    uint32_t width, height, n_photons, seed;
    float max_dist;
    sc_film_options opts;                           /* bins must be >= 1 */
} sc_scene_job;
/* Tuning knobs, 0 = default: photons per work chunk (queue granularity),
 * register bound (minimum CTAs per SM, 4 or 5), warp-aggregated splats, grid,
 * per_photon = 1 to run each photon's haze samples in its own lane instead
 * of the default warp-split transport (segments buffered per warp, samples
 * processed as one converged list), and threads per CTA (128 or 256). */
typedef struct { uint32_t chunk_photons, minb, aggregate, grid, per_photon, block; } sc_batch_tuning;
int sc_batch_create(sc_ctx* ctx, const sc_scene_job* jobs, uint32_t n_jobs,
                    const sc_batch_tuning* tuning, sc_batch** out);
int sc_batch_destroy(sc_batch* b);
/* Time every candidate tuning on this batch and keep the fastest. */
int sc_batch_autotune(sc_batch* b, sc_batch_tuning* chosen);
int sc_batch_set_tuning(sc_batch* b, const sc_batch_tuning* tuning);
int sc_batch_get_tuning(sc_batch* b, sc_batch_tuning* tuning);
/* New cameras / beams / seeds / weights for the same films and budgets. */
int sc_batch_update_jobs(sc_batch* b, const sc_scene_job* jobs, uint32_t n_jobs);
/* One pass over every job (graph replay); stream NULL = the batch's stream.
 * Asynchronous; afterwards each job's XYZ image is ready and its film drained. */
int sc_batch_run(sc_batch* b, void* stream);
/* The same work as plain per-scene launches (trace + drain/reduce per job),
 * with the transport of the batch's tuning (per_photon). */
int sc_batch_run_plain(sc_batch* b, void* stream);
int sc_batch_synchronize(sc_batch* b);
int sc_batch_read_xyz(sc_batch* b, uint32_t job, float* out);
/* All jobs' XYZ images concatenated in job order (sum of 3*w*h floats). */
int sc_batch_read_all_xyz(sc_batch* b, float* out, size_t capacity, void* stream);
/* The same copy without waiting for it: ordered after the last pass, on
 * `stream` (NULL: the batch's own copy stream).  The next pass traces while the
 * copy runs and starts its drain only after the copy ends, and the next
 * sc_batch_update_jobs waits for the last pass; `out` must stay valid (and
 * should be pinned) until sc_batch_synchronize or the stream is synchronised. */
int sc_batch_read_all_xyz_async(sc_batch* b, float* out, size_t capacity, void* stream);
/* job_table_bytes: bytes uploaded host -> device by sc_batch_update_jobs. */
int sc_batch_info(sc_batch* b, uint64_t* total_photons, uint64_t* film_bytes, uint64_t* xyz_floats,
                  uint64_t* job_table_bytes);
/* Work of one pass, measured by an instrumented pass (not timed work):
 * out[0..5] = photons, path segments, in-frame haze samples, scatters, film
 * tiles that received light, bytes of those tiles. */
int sc_batch_stats(sc_batch* b, uint64_t out[6]);
int sc_batch_device_xyz(sc_batch* b, uint32_t job, const float** xyz_dev);

/* ---- serving loop: continuous batching (no counterpart in the reference) -
 * Requests are admitted against a device-memory budget (one arena allocated
 * at creation), and each sc_server_step traces the current frame of every
 * admitted request in one persistent launch.  A request's photons are keyed by
 * its own photon index, so its image is the same alone or in any mix. */
typedef struct {
    uint64_t hbm_budget_bytes;  /* arena for films, masks and images of admitted requests */
    uint32_t max_slots;         /* requests on the device at once (0 -> 256) */
    uint32_t chunk_photons;     /* work-chunk size of the batched launch (0 -> 2048) */
    uint32_t warp_split;        /* 0: one photon per lane (the default, as the batch autotuner picks
                                   on uneven scenes); 1: the warp-split transport */
} sc_server_config;
typedef struct {
    sc_scene_job job;           /* scene, film (bins >= 1), photons per frame (n_photons), seed, camera */
    uint32_t frames;            /* 1: a single render; F > 1: a session of F frames.  Frame f traces
                                   photons [f*N, (f+1)*N) of the request's stream.  With orbit_deg == 0
                                   the session is progressive (spectral-viewer/src/main.rs:395-419): the
                                   frames add into the request's film on the device and its image is
                                   that film over all frames so far times 1/frames (one frame's
                                   brightness); with orbit_deg != 0 the camera moves every frame, the
                                   film restarts, and the image is the last frame's */
    float orbit_deg;            /* camera azimuth step per frame around orbit_target (about +y) */
    float orbit_target[3];
    float orbit_up[3];
    float vfov_deg;             /* camera of frame f rebuilt with Camera::look_at */
} sc_request;
int sc_server_create(sc_ctx* ctx, const sc_server_config* cfg, sc_server** out);
int sc_server_destroy(sc_server* s);
/* Queue a request; SC_E_NOMEM when it could never fit the budget. */
int sc_server_submit(sc_server* s, const sc_request* r, uint64_t* id);
/* Admit what fits and queue one frame of every admitted request (one batched
 * launch and one drain) on the server's stream; returns once at most one step
 * (two while requests wait for admission) is queued ahead of it.  Requests
 * whose last frame was queued become pollable once their image is in host
 * memory.  With nothing left to trace, a step waits for the queued work.
 * `active` counts admitted requests plus those whose images are still on their
 * way (sc_server_stats too), so a loop "while queued or active: step" ends
 * with every result pollable. */
int sc_server_step(sc_server* s, uint32_t* active);
/* Pop a finished request: its last frame's XYZ image (3*w*h floats) and the
 * steady-clock times [submit, admit, first frame done, done] in seconds (the
 * last two as seen by the host).  SC_E_STATE when nothing is finished.
 * Finished images wait in a 256 MB pinned host ring until polled; while it is
 * full, further finished images stay on the device (holding their share of
 * the budget) and are copied as polls make room, so poll as results come. */
int sc_server_poll(sc_server* s, uint64_t* id, float* xyz_out, size_t capacity, uint32_t* width,
                   uint32_t* height, double times[4]);
/* The current image of an active request (3*w*h floats): for a progressive
 * session the accumulated film so far (times 1/frames_done), for an orbit
 * session its latest frame.  Waits for the frames already queued on the
 * server's stream; *frames_done = frames in that image.  SC_E_STATE when the
 * request is not on the device or has no frame yet (a finished one is polled). */
int sc_server_peek(sc_server* s, uint64_t id, float* xyz_out, size_t capacity, uint32_t* frames_done);
/* Drop a queued or active request (frames of it already queued still run;
 * its device memory is reused only behind them). */
int sc_server_cancel(sc_server* s, uint64_t id);
int sc_server_stats(sc_server* s, uint64_t* photons_traced, uint64_t* bytes_in_use, uint32_t* queued,
                    uint32_t* active, uint32_t* finished);

#ifdef __cplusplus
}
#endif
#endif
