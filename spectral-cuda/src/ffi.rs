//! Raw bindings of `include/spectral_cuda.h`, the C ABI of the sm_100a library
//! `libspectral_cuda.so`: one `extern "C"` declaration per entry point and one
//! `#[repr(C)]` record per struct, field for field.  Every call returns a
//! status (`SC_OK` or a negative `SC_E_*`); `sc_last_error()` gives the
//! thread's last message.  The scene records have the layouts of the
//! reference's upload records (spectral-gpu/src/upload.rs:7-32).
//!
//! Unverified: written without a Rust toolchain (none exists where this
//! library is built); `tests/test_rust_binding.py` checks every declaration
//! here against the header and the library's exported symbols.
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_int, c_void};

pub const SC_OK: c_int = 0;
pub const SC_E_INVALID: c_int = -1;
pub const SC_E_CUDA: c_int = -2;
pub const SC_E_NOMEM: c_int = -3;
pub const SC_E_LIMIT: c_int = -4;
pub const SC_E_TIMEOUT: c_int = -5;
pub const SC_E_STATE: c_int = -6;
pub const SC_E_NODEVICE: c_int = -7;

pub const SC_MAX_PRIMS: usize = 64;
pub const SC_MAX_PLANES: usize = 256;
pub const SC_MAX_BINS: usize = 256;
pub const SC_BATCH_MAX_PRIMS: usize = 4;
pub const SC_BATCH_MAX_PLANES: usize = 16;
pub const SC_NOALLOC_MAX_FILM_CELLS: u32 = 1 << 21;

/// GpuPrimitive (upload.rs): kind 0 sphere, 1 convex solid.
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScPrimitive { pub center: [f32; 3], pub radius: f32, pub plane_start: u32, pub plane_count: u32,
                         pub kind: u32, pub material: u32 }
/// GpuMaterial (upload.rs): kind 0 Lambertian, 1 dielectric; glass 0 BK7, 1 SF11, 2 water, 3 fused silica.
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScMaterial { pub reflectance: f32, pub glass: u32, pub kind: u32, pub pad: u32 }
/// GpuPlane (upload.rs): half-space normal . x + d <= 0.
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScPlane { pub normal: [f32; 3], pub d: f32 }
/// lighttrace::Beam.
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScBeam { pub corner: [f32; 3], pub u: [f32; 3], pub v: [f32; 3], pub dir: [f32; 3] }
/// Camera::view_basis.
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScCamera { pub origin: [f32; 3], pub lower_left: [f32; 3], pub horizontal: [f32; 3], pub vertical: [f32; 3] }
/// VolWeights (vol_photons.rs:256-267).
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScVolWeights { pub sigma_s: f32, pub sigma_t: f32, pub g: f32 }
/// DebugPhotonGpu (vol_photons.rs:85-93), 304 bytes.
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct ScDebugPhoton { pub num_states: u32, pub lambda: f32, pub pad0: u32, pub pad1: u32, pub states: [[f32; 4]; 18] }
/// Film options beyond the reference; zeros select the reference's film.
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScFilmOptions { pub bins: u32, pub lambda_min: f32, pub lambda_max: f32, pub max_bounces: u32,
                           pub scale_log2: u32, pub estimator: u32, pub haze_exact: u32 }
/// Camera-tracer extensions (zero = the reference's tracer).
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScTracerOptions { pub max_depth: u32, pub rr_start: u32, pub emitter_center: [f32; 3],
                             pub emitter_radius: f32, pub emitter_scale: f32, pub wave_bounces: u32,
                             pub chains: u32, pub wave_paths_log2: u32 }
/// lighttrace::Screen rectangle.
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScScreen { pub corner: [f32; 3], pub u: [f32; 3], pub v: [f32; 3] }
/// One trace through the device-pointer entry points (all pointers device memory).
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct ScTraceDesc {
    pub prims: *const ScPrimitive, pub n_prims: u32,
    pub planes: *const ScPlane, pub n_planes: u32,
    pub mats: *const ScMaterial, pub n_mats: u32,
    pub cam: ScCamera, pub beam: ScBeam, pub weights: ScVolWeights,
    pub width: u32, pub height: u32, pub seed: u32, pub spectral: u32,
    pub max_dist: f32,
    pub opts: ScFilmOptions,
    pub zbuffer: *const f32,
}
/// One scene of a batch (or one request's scene).
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct ScSceneJob {
    pub n_prims: u32, pub n_planes: u32, pub n_mats: u32, pub spectral: u32,
    pub prims: [ScPrimitive; SC_BATCH_MAX_PRIMS],
    pub planes: [ScPlane; SC_BATCH_MAX_PLANES],
    pub mats: [ScMaterial; SC_BATCH_MAX_PRIMS],
    pub cam: ScCamera, pub beam: ScBeam, pub weights: ScVolWeights,
    pub width: u32, pub height: u32, pub n_photons: u32, pub seed: u32,
    pub max_dist: f32,
    pub opts: ScFilmOptions,
}
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScBatchTuning { pub chunk_photons: u32, pub minb: u32, pub aggregate: u32, pub grid: u32,
                           pub per_photon: u32, pub block: u32 }
#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct ScServerConfig { pub hbm_budget_bytes: u64, pub max_slots: u32, pub chunk_photons: u32,
                            pub warp_split: u32 }
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct ScRequest { pub job: ScSceneJob, pub frames: u32, pub orbit_deg: f32, pub orbit_target: [f32; 3],
                       pub orbit_up: [f32; 3], pub vfov_deg: f32 }

/// Opaque handles.
#[repr(C)] pub struct ScCtx { _private: [u8; 0] }
#[repr(C)] pub struct ScPhotonFilm { _private: [u8; 0] }
#[repr(C)] pub struct ScTracer { _private: [u8; 0] }
#[repr(C)] pub struct ScAtomicFilm { _private: [u8; 0] }
#[repr(C)] pub struct ScBatch { _private: [u8; 0] }
#[repr(C)] pub struct ScServer { _private: [u8; 0] }

extern "C" {
    pub fn sc_last_error() -> *const c_char;
    pub fn sc_version() -> *const c_char;
    pub fn sc_ctx_create(device: c_int, tables_5x71: *const f32, out: *mut *mut ScCtx) -> c_int;
    pub fn sc_ctx_destroy(ctx: *mut ScCtx) -> c_int;
    pub fn sc_ctx_synchronize(ctx: *mut ScCtx) -> c_int;
    pub fn sc_load_sensor_tables(csv_path: *const c_char, out_5x71: *mut f32) -> c_int;
    pub fn sc_camera_look_at(origin: *const f32, target: *const f32, up: *const f32, vfov_deg: f32, aspect: f32, out: *mut ScCamera) -> c_int;
    pub fn sc_camera_proj_params(cam: *const ScCamera, out: *mut f32) -> c_int;
    pub fn sc_glass_n(glass: u32, lambda_nm: f32) -> f32;
    pub fn sc_glass_n_many(glass: u32, lambda_nm: *const f32, n: usize, out: *mut f32) -> c_int;
    pub fn sc_glass_n_device(ctx: *mut ScCtx, glass: u32, lambda_nm_dev: *const f32, n: usize, out_dev: *mut f32, stream: *mut c_void) -> c_int;
    pub fn sc_rng_draws(ctx: *mut ScCtx, key: u32, seed: u32, n: u32, out: *mut u32) -> c_int;
    pub fn sc_dsotm_scene(aspect: f32, prim: *mut ScPrimitive, planes5: *mut ScPlane, mat: *mut ScMaterial, beam: *mut ScBeam, cam: *mut ScCamera) -> c_int;
    pub fn sc_photon_film_create(ctx: *mut ScCtx, prims: *const ScPrimitive, n_prims: u32, planes: *const ScPlane, n_planes: u32, mats: *const ScMaterial, n_mats: u32, background: f32, cam: *const ScCamera, beam: *const ScBeam, width: u32, height: u32, n_photons: u32, seed: u32, max_dist: f32, weights: *const ScVolWeights, zbuffer: *const f32, opts: *const ScFilmOptions, out: *mut *mut ScPhotonFilm) -> c_int;
    pub fn sc_photon_film_destroy(f: *mut ScPhotonFilm) -> c_int;
    pub fn sc_photon_film_trace_and_resolve(f: *mut ScPhotonFilm, n_photons: u32, seed: u32) -> c_int;
    pub fn sc_photon_film_trace_chunked(f: *mut ScPhotonFilm, total_photons: u32, seed: u32) -> c_int;
    pub fn sc_photon_film_dispatch(f: *mut ScPhotonFilm, photon_base: u32, n_photons: u32, seed: u32) -> c_int;
    pub fn sc_photon_film_trace_debug(f: *mut ScPhotonFilm, n_photons: u32, seed: u32, debug_count: u32, out: *mut ScDebugPhoton) -> c_int;
    pub fn sc_photon_film_set_spectral(f: *mut ScPhotonFilm, on: c_int) -> c_int;
    pub fn sc_photon_film_get_spectral(f: *mut ScPhotonFilm, on: *mut c_int) -> c_int;
    pub fn sc_photon_film_set_camera(f: *mut ScPhotonFilm, cam: *const ScCamera) -> c_int;
    pub fn sc_photon_film_recompute_surface(f: *mut ScPhotonFilm, cam: *const ScCamera) -> c_int;
    pub fn sc_photon_film_read_surface(f: *mut ScPhotonFilm, out: *mut f32) -> c_int;
    pub fn sc_photon_film_read_accum(f: *mut ScPhotonFilm, out: *mut f32) -> c_int;
    pub fn sc_photon_film_read_raw(f: *mut ScPhotonFilm, out: *mut i64) -> c_int;
    pub fn sc_photon_film_clear(f: *mut ScPhotonFilm) -> c_int;
    pub fn sc_photon_film_auto_expose(f: *mut ScPhotonFilm, scale: f32, exposure: *mut f32) -> c_int;
    pub fn sc_photon_film_auto_expose_p997(f: *mut ScPhotonFilm, exposure: *mut f32) -> c_int;
    pub fn sc_photon_film_to_rgb8(f: *mut ScPhotonFilm, exposure: f32, out_rgb: *mut u8) -> c_int;
    pub fn sc_photon_film_gather_rgba8(f: *mut ScPhotonFilm, total_photons: u64, target_n: f32, kradius: f32, exposure: f32, out_rgba: *mut u8) -> c_int;
    pub fn sc_photon_film_dims(f: *mut ScPhotonFilm, width: *mut u32, height: *mut u32, channels: *mut u32) -> c_int;
    pub fn sc_photon_film_set_scene(f: *mut ScPhotonFilm, prims: *const ScPrimitive, n_prims: u32, planes: *const ScPlane, n_planes: u32, mats: *const ScMaterial, n_mats: u32, cam: *const ScCamera, beam: *const ScBeam) -> c_int;
    pub fn sc_photon_film_device_buffers(f: *mut ScPhotonFilm, film_dev: *mut *mut c_void, film_bytes: *mut usize, flags_dev: *mut *mut c_void, flag_bytes: *mut usize, stream: *mut *mut c_void) -> c_int;
    pub fn sc_photon_film_mark_all_dirty(f: *mut ScPhotonFilm) -> c_int;
    pub fn sc_photon_film_trace_stats(f: *mut ScPhotonFilm, photon_base: u32, count: u32, seed: u32, out: *mut u64) -> c_int;
    pub fn sc_tracer_create(ctx: *mut ScCtx, prims: *const ScPrimitive, n_prims: u32, planes: *const ScPlane, n_planes: u32, mats: *const ScMaterial, n_mats: u32, background: f32, has_horizon: c_int, horizon: f32, cam: *const ScCamera, width: u32, height: u32, illuminant: u32, seed: u32, opts: *const ScTracerOptions, out: *mut *mut ScTracer) -> c_int;
    pub fn sc_tracer_destroy(t: *mut ScTracer) -> c_int;
    pub fn sc_tracer_accumulate(t: *mut ScTracer, spp: u32) -> c_int;
    pub fn sc_tracer_read_xyz(t: *mut ScTracer, out: *mut f32) -> c_int;
    pub fn sc_tracer_set_camera(t: *mut ScTracer, cam: *const ScCamera) -> c_int;
    pub fn sc_tracer_clear_accum(t: *mut ScTracer) -> c_int;
    pub fn sc_tracer_dims(t: *mut ScTracer, width: *mut u32, height: *mut u32) -> c_int;
    pub fn sc_tracer_set_spectral(t: *mut ScTracer, on: c_int) -> c_int;
    pub fn sc_tracer_set_rows(t: *mut ScTracer, row_begin: u32, row_end: u32) -> c_int;
    pub fn sc_tracer_stream(t: *mut ScTracer, stream: *mut *mut c_void) -> c_int;
    pub fn sc_tracer_last_stats(t: *mut ScTracer, paths: *mut u64, segments: *mut u64) -> c_int;
    pub fn sc_atomic_film_create(ctx: *mut ScCtx, width: u32, height: u32, out: *mut *mut ScAtomicFilm) -> c_int;
    pub fn sc_atomic_film_destroy(f: *mut ScAtomicFilm) -> c_int;
    pub fn sc_atomic_film_splat(f: *mut ScAtomicFilm, seed: u32, n_splats: u32) -> c_int;
    pub fn sc_atomic_film_read_raw(f: *mut ScAtomicFilm, out: *mut u32) -> c_int;
    pub fn sc_atomic_film_resolve(f: *mut ScAtomicFilm) -> c_int;
    pub fn sc_atomic_film_read_accum(f: *mut ScAtomicFilm, out: *mut f32) -> c_int;
    pub fn sc_atomic_film_clear_film(f: *mut ScAtomicFilm) -> c_int;
    pub fn sc_atomic_film_clear_accum(f: *mut ScAtomicFilm) -> c_int;
    pub fn sc_atomic_film_auto_expose_accum(f: *mut ScAtomicFilm, scale: f32, exposure: *mut f32) -> c_int;
    pub fn sc_atomic_film_to_rgb8(f: *mut ScAtomicFilm, exposure: f32, out: *mut u8) -> c_int;
    pub fn sc_atomic_film_stream(f: *mut ScAtomicFilm, stream: *mut *mut c_void) -> c_int;
    pub fn sc_atomic_film_check_determinism(ctx: *mut ScCtx, width: u32, height: u32, seed: u32, n_splats: u32, first_diff: *mut i64) -> c_int;
    pub fn sc_lighttrace(ctx: *mut ScCtx, prims: *const ScPrimitive, n_prims: u32, planes: *const ScPlane, n_planes: u32, mats: *const ScMaterial, n_mats: u32, screen: *const ScScreen, width: u32, height: u32, beam: *const ScBeam, n_photons: u32, seed: u32, opts: *const ScFilmOptions, out_sum: *mut f32) -> c_int;
    pub fn sc_scene_zbuffer(ctx: *mut ScCtx, prims: *const ScPrimitive, n_prims: u32, planes: *const ScPlane, n_planes: u32, mats: *const ScMaterial, n_mats: u32, floor: *const ScScreen, cam: *const ScCamera, width: u32, height: u32, out: *mut f32) -> c_int;
    pub fn sc_film_bytes(width: u32, height: u32, channels: u32) -> usize;
    pub fn sc_film_flag_bytes(width: u32, height: u32) -> usize;
    pub fn sc_trace_photons_device(ctx: *mut ScCtx, desc: *const ScTraceDesc, photon_base: u32, count: u32, film_dev: *mut c_void, flags_dev: *mut u32, stream: *mut c_void) -> c_int;
    pub fn sc_trace_stats_device(ctx: *mut ScCtx, desc: *const ScTraceDesc, photon_base: u32, count: u32, out_dev: *mut u64, stream: *mut c_void) -> c_int;
    pub fn sc_sensor_reduce_device(ctx: *mut ScCtx, width: u32, height: u32, channels: u32, lambda_min: f32, lambda_max: f32, scale_log2: u32, film_dev: *mut c_void, flags_dev: *mut u32, xyz_dev: *mut f32, drain: c_int, stream: *mut c_void) -> c_int;

    // One scene split over GPUs: IPC mapping of the peers' films and the
    // band reduction of their sum.
    pub fn sc_ipc_export(ctx: *mut ScCtx, dev_ptr: *const c_void, handle: *mut u8, offset: *mut usize) -> c_int;
    pub fn sc_ipc_import(ctx: *mut ScCtx, handle: *const u8, offset: usize, dev_ptr: *mut *mut c_void) -> c_int;
    pub fn sc_ipc_close(ctx: *mut ScCtx, dev_ptr: *mut c_void, offset: usize) -> c_int;
    pub fn sc_sensor_reduce_peers(ctx: *mut ScCtx, width: u32, height: u32, channels: u32, lambda_min: f32, lambda_max: f32, scale_log2: u32, films_dev: *const *const i64, n_films: u32, row_begin: u32, row_end: u32, xyz_dev: *mut f32, stream: *mut c_void) -> c_int;
    pub fn sc_trace_xyz_noalloc(tables_5x71: *const f32, desc: *const ScTraceDesc, photon_base: u32, count: u32, xyz_dev: *mut f32, stream: *mut c_void) -> c_int;
    pub fn sc_batch_create(ctx: *mut ScCtx, jobs: *const ScSceneJob, n_jobs: u32, tuning: *const ScBatchTuning, out: *mut *mut ScBatch) -> c_int;
    pub fn sc_batch_destroy(b: *mut ScBatch) -> c_int;
    pub fn sc_batch_autotune(b: *mut ScBatch, chosen: *mut ScBatchTuning) -> c_int;
    pub fn sc_batch_set_tuning(b: *mut ScBatch, tuning: *const ScBatchTuning) -> c_int;
    pub fn sc_batch_get_tuning(b: *mut ScBatch, tuning: *mut ScBatchTuning) -> c_int;
    pub fn sc_batch_update_jobs(b: *mut ScBatch, jobs: *const ScSceneJob, n_jobs: u32) -> c_int;
    pub fn sc_batch_run(b: *mut ScBatch, stream: *mut c_void) -> c_int;
    pub fn sc_batch_run_plain(b: *mut ScBatch, stream: *mut c_void) -> c_int;
    pub fn sc_batch_synchronize(b: *mut ScBatch) -> c_int;
    pub fn sc_batch_read_xyz(b: *mut ScBatch, job: u32, out: *mut f32) -> c_int;
    pub fn sc_batch_read_all_xyz(b: *mut ScBatch, out: *mut f32, capacity: usize, stream: *mut c_void) -> c_int;
    pub fn sc_batch_read_all_xyz_async(b: *mut ScBatch, out: *mut f32, capacity: usize, stream: *mut c_void) -> c_int;
    pub fn sc_batch_info(b: *mut ScBatch, total_photons: *mut u64, film_bytes: *mut u64, xyz_floats: *mut u64, job_table_bytes: *mut u64) -> c_int;
    pub fn sc_batch_stats(b: *mut ScBatch, out: *mut u64) -> c_int;
    pub fn sc_batch_device_xyz(b: *mut ScBatch, job: u32, xyz_dev: *mut *const f32) -> c_int;
    pub fn sc_server_create(ctx: *mut ScCtx, cfg: *const ScServerConfig, out: *mut *mut ScServer) -> c_int;
    pub fn sc_server_destroy(s: *mut ScServer) -> c_int;
    pub fn sc_server_submit(s: *mut ScServer, r: *const ScRequest, id: *mut u64) -> c_int;
    pub fn sc_server_step(s: *mut ScServer, active: *mut u32) -> c_int;
    pub fn sc_server_poll(s: *mut ScServer, id: *mut u64, xyz_out: *mut f32, capacity: usize, width: *mut u32, height: *mut u32, times: *mut f64) -> c_int;
    pub fn sc_server_peek(s: *mut ScServer, id: u64, xyz_out: *mut f32, capacity: usize, frames_done: *mut u32) -> c_int;
    pub fn sc_server_cancel(s: *mut ScServer, id: u64) -> c_int;
    pub fn sc_server_stats(s: *mut ScServer, photons_traced: *mut u64, bytes_in_use: *mut u64, queued: *mut u32, active: *mut u32, finished: *mut u32) -> c_int;
}
