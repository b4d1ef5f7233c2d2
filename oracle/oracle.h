/*
 * CPU oracle for the spectral forward / volumetric / camera-tracer hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * renderer's CPU crate (spectral-core, Rust) used to check the CUDA path.  It
 * is never linked into or called by the product library; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Each function cites the reference file:line it restates.  Arithmetic is f32
 * in the reference's operation order (glam 0.29 scalar Vec3 semantics:
 * dot = (x*x + y*y) + z*z, normalize = v * (1/len)), Sellmeier in f64, built
 * with -ffp-contract=off so no multiply-add is fused.
 */
#ifndef SPECTRAL_ORACLE_H
#define SPECTRAL_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Flat scene records: same layout as the reference's GPU upload PODs
 * (spectral-gpu/src/upload.rs:7-32). */
typedef struct { float center[3]; float radius; uint32_t plane_start, plane_count, kind, material; } or_prim;
typedef struct { float reflectance; uint32_t glass, kind, pad; } or_mat;
typedef struct { float normal[3]; float d; } or_plane;

typedef struct {
    const or_prim* prims; uint32_t n_prims;
    const or_plane* planes; uint32_t n_planes;
    const or_mat* mats; uint32_t n_mats;
    float background;
    int32_t has_horizon;
    float horizon;
} or_scene;

typedef struct { float corner[3], u[3], v[3], dir[3]; } or_beam;
typedef struct { float origin[3], lower_left[3], horizontal[3], vertical[3]; } or_camera;

typedef struct {
    uint32_t width, height, seed, max_bounces;
    float sigma_s, sigma_t, g, max_dist;
    float lambda_min, lambda_range;   /* emission band */
    uint32_t spectral;                /* 1: n(lambda); 0: n(550 nm) for every photon */
    uint32_t bins;                    /* spectral film bins */
    float bin_min, bin_inv_width;     /* bin = floor((lambda - bin_min) * bin_inv_width) */
    float scale;                      /* fixed-point scale of the int64 films */
    uint32_t estimator;               /* 0 point (HG + transmittance), 1 legacy isotropic, 3 point with
                                         free-flight distances (truncated exponential, 1/pdf weights) */
} or_vol_params;

/* rng.rs */
uint32_t or_pcg32(uint32_t x);
uint32_t or_mix2(uint32_t a, uint32_t b);
void or_rng_draws_u32(uint32_t key, uint32_t seed, uint32_t n, uint32_t* out);
void or_rng_draws_f32(uint32_t key, uint32_t seed, uint32_t n, float* out);

/* sellmeier.rs (+ fused silica, glass id 3) */
float or_glass_n(uint32_t glass, float nm);
/* Planted faults for the gate-sensitivity test only (0 = none; see oracle.c). */
void or_set_fault(int fault);
/* or_glass_n of every element of nm[0..n). */
void or_glass_n_many(uint32_t glass, const float* nm, size_t n, float* out);

/* cie.rs */
int or_load_tables_csv(const char* path);
void or_get_tables(float* out_5x71);
void or_cmf(float nm, float out[3]);
float or_illuminant(uint32_t which, float nm);
void or_integrate_illuminant(uint32_t which, float out[3]);
void or_xyz_to_linear_srgb(const float xyz[3], float out[3]);
void or_tonemap_to_u8(const float lin[3], float exposure, uint8_t out[3]);

/* optics.rs / geom.rs / material.rs */
void or_reflect(const float d[3], const float n[3], float out[3]);
int or_refract(const float d[3], const float n[3], float n1, float n2, float out[3]);
float or_fresnel(float cos_i, float n1, float n2);
int or_scene_intersect(const or_scene* sc, const float o[3], const float d[3],
                       float* t, float point[3], float normal[3], int* front_face, uint32_t* mat);

/* camera.rs */
void or_camera_look_at(const float origin[3], const float target[3], const float up[3],
                       float vfov_deg, float aspect, or_camera* out);
void or_camera_primary_ray(const or_camera* c, float s, float t, float o[3], float d[3]);
int or_camera_project(const or_camera* c, const float p[3], float out_std[3]);
/* camera_proj_params (spectral-gpu/src/vol_photons.rs:100-115), 16 floats. */
void or_camera_proj_params(const or_camera* c, float out[16]);

/* volume.rs */
float or_phase_hg(float g, float cos_theta);

/* Per-photon path (spectral-gpu/src/vol_photons.rs:932-991). states: 2*max_pairs float4. */
uint32_t or_simulate_photon(const or_scene* sc, const or_beam* beam, const or_vol_params* p,
                            uint32_t photon_idx, uint32_t max_pairs, float* states4,
                            float* lambda, uint32_t* tir_count);

/* Point estimator (volume.rs:99-168) over photons [begin, end).  Any output may be NULL:
 * img_f32  3*w*h f32 accumulated in photon order (the reference's own film),
 * film_xyz 3*w*h int64 fixed point, film_spec w*h*bins int64 fixed point.
 * zbuf may be NULL (no occlusion). */
void or_render_point(const or_scene* sc, const or_camera* cam, const or_beam* beam,
                     const or_vol_params* p, const float* zbuf, uint32_t begin, uint32_t end,
                     float* img_f32, int64_t* film_xyz, int64_t* film_spec);

/* Same, photon-parallel over nthreads POSIX threads (int64 films only, exact merge). */
void or_render_point_mt(const or_scene* sc, const or_camera* cam, const or_beam* beam,
                        const or_vol_params* p, const float* zbuf, uint32_t begin, uint32_t end,
                        int64_t* film_xyz, int64_t* film_spec, int nthreads);

/* Photon-beam estimator (volume.rs:178-329), f32 image, serial. */
void or_render_beam(const or_scene* sc, const or_camera* cam, const or_beam* beam,
                    const or_vol_params* p, const float* zbuf, uint32_t begin, uint32_t end,
                    float* img_f32);

/* Screen-caustic light tracer (lighttrace.rs:157-166). screen: corner,u,v (9 floats). */
void or_lighttrace(const or_scene* sc, const float screen_cuv[9], uint32_t w, uint32_t h,
                   const or_beam* beam, const or_vol_params* p, uint32_t n, float* sum_xyz);

/* Camera-tracer extensions with no counterpart in the reference (all zero =
 * reference behaviour): a spherical emitter whose radiance is
 * emitter_scale * illuminant(lambda), and Russian roulette after rr_start
 * scatters (survival p = min(throughput, 0.95), throughput /= p). */
typedef struct { float center[3]; float radius; float scale; uint32_t rr_start; } or_tracer_ext;
void or_tracer_set_ext(const or_tracer_ext* ext);
/* GpuTracer::set_spectral (spectral-gpu/src/lib.rs:369-372; trace.wgsl:477-480):
 * 0 makes every dielectric hit use n(550 nm) instead of n(hero wavelength). */
void or_tracer_set_spectral(int on);

/* Hero-wavelength camera tracer (tracer.rs:44-141). Accumulates spp samples starting
 * at sample index `base` into sum_xyz (3*w*h); rows [row0,row1). */
void or_tracer_accumulate(const or_scene* sc, const or_camera* cam, uint32_t w, uint32_t h,
                          uint32_t illuminant, uint32_t seed, uint32_t spp, uint32_t base,
                          uint32_t max_bounces, uint32_t row0, uint32_t row1, float* sum_xyz);
void or_tracer_accumulate_mt(const or_scene* sc, const or_camera* cam, uint32_t w, uint32_t h,
                             uint32_t illuminant, uint32_t seed, uint32_t spp, uint32_t base,
                             uint32_t max_bounces, float* sum_xyz, int nthreads);
void or_tracer_sample(const or_scene* sc, const or_camera* cam, uint32_t w, uint32_t h,
                      uint32_t illuminant, uint32_t seed, uint32_t px, uint32_t py,
                      uint32_t sample_idx, uint32_t max_bounces, float out[3]);

/* Material::scatter (material.rs:30-66) for one (wo, hit) with PathRng(key, seed). */
int or_scatter(uint32_t kind, float reflectance, const float wo[3], const float normal[3], int front_face,
               float n_hero, uint32_t key, uint32_t seed, float dir_out[3], float* weight);

/* vol_photons.rs:1048-1095: like or_simulate_photon but the path uses `fixed_lambda`
 * (the lambda draw is still consumed). */
uint32_t or_simulate_photon_fixed(const or_scene* sc, const or_beam* beam, const or_vol_params* p,
                                  uint32_t photon_idx, float fixed_lambda, uint32_t max_pairs, float* states4);

/* lighttrace.rs tests (mean_landing, lighttrace.rs:406-416): mean (s, r) of the
 * photons 0..n that land, with PathRng(i, seed) and a fixed wavelength.
 * Returns the number landed. */
uint32_t or_mean_landing(const or_scene* sc, const float screen_cuv[9], const or_beam* beam,
                         float lambda, uint32_t n, uint32_t seed, float out_sr[2]);

/* Surface rim pass (vol_photons.rs:1517-1538). out: 3*w*h. */
void or_surface_rim(const or_scene* sc, const or_camera* cam, uint32_t w, uint32_t h, float* out);
/* prism_on_plane.rs:125-160 z-buffer; floor9 (corner,u,v) may be NULL. */
void or_scene_zbuffer(const or_scene* sc, const float* floor9, const or_camera* cam, uint32_t w, uint32_t h,
                      float* out);

/* Synthetic atomic-film splat (spectral-gpu/src/shaders/vol_splat.wgsl:58-79), u32 film. */
void or_synthetic_splat(uint32_t w, uint32_t h, uint32_t seed, uint32_t n_splats, uint32_t* film);

/* Viewer gather (spectral-viewer/src/main.rs:132-173) on an f32 XYZ image, RGBA8 out. */
void or_gather_tonemap(const float* xyz, const float* surface, uint32_t w, uint32_t h,
                       float k, float kradius, float exposure, uint8_t* rgba);

#ifdef __cplusplus
}
#endif
#endif
