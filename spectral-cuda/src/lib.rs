//! spectral-cuda: the B200 (sm_100a) backend of the spectral renderer, with
//! the shapes of the reference's `spectral-gpu` crate -- `GpuPhotonFilm`
//! (spectral-gpu/src/vol_photons.rs:228-851), `GpuTracer`
//! (spectral-gpu/src/lib.rs:165-389) and `AtomicFilm`
//! (spectral-gpu/src/film.rs:40-305) -- over the C ABI of `libspectral_cuda.so`
//! (`ffi`).  Scenes, cameras and beams are spectral-core's own types.  Errors
//! panic with the library's message, as the reference panics on GPU errors;
//! `CudaContext::new` returns `None` without a usable device, as
//! `GpuContext::new` does.
//!
//! Unverified: written without a Rust toolchain (none exists where the CUDA
//! library is built).  `tests/test_rust_binding.py` checks `ffi` against the
//! header and the library's exports; the wrappers below call nothing else.

pub mod ffi;

use std::ffi::CStr;
use std::os::raw::c_int;

use spectral_core::camera::Camera;
use spectral_core::cie::{Illuminant, Sensor};
use spectral_core::lighttrace::Beam;
use spectral_core::material::Material;
use spectral_core::scene::{Scene, Shape};
use spectral_core::sellmeier::Glass;

fn check(rc: c_int) {
    if rc != ffi::SC_OK {
        let msg = unsafe { CStr::from_ptr(ffi::sc_last_error()) }.to_string_lossy().into_owned();
        panic!("spectral_cuda error {rc}: {msg}");
    }
}

/// The 5x71 sensor table [xbar;71][ybar;71][zbar;71][d65;71][a;71] at 5 nm
/// from 380 nm, sampled from spectral-core's sensor (the layout of
/// spectral-gpu/src/data.rs:12-22).
pub fn sample_tables() -> Vec<f32> {
    let s = Sensor::new();
    let nm = |i: usize| 380.0 + 5.0 * i as f32;
    let mut t = vec![0.0f32; 5 * 71];
    for i in 0..71 {
        let (x, y, z) = s.cmf(nm(i));
        t[i] = x;
        t[71 + i] = y;
        t[142 + i] = z;
        t[213 + i] = s.illuminant(Illuminant::D65, nm(i));
        t[284 + i] = s.illuminant(Illuminant::A, nm(i));
    }
    t
}

/// Scene records in the upload layout (one material per primitive, solids'
/// half-spaces in order), as the reference's flatten_scene lays them out
/// (spectral-gpu/src/lib.rs:91-158), without its padding elements: the ABI
/// takes counts, and empty arrays are allowed.
pub fn flatten_scene(scene: &Scene) -> (Vec<ffi::ScPrimitive>, Vec<ffi::ScPlane>, Vec<ffi::ScMaterial>) {
    let mut prims = Vec::new();
    let mut planes = Vec::new();
    let mut mats = Vec::new();
    for p in &scene.primitives {
        let material = mats.len() as u32;
        mats.push(match p.material {
            Material::Lambertian { reflectance } => ffi::ScMaterial { reflectance, glass: 0, kind: 0, pad: 0 },
            Material::Dielectric { glass } => ffi::ScMaterial {
                reflectance: 0.0,
                glass: match glass {
                    Glass::Bk7 => 0,
                    Glass::Sf11 => 1,
                    Glass::Water => 2,
                },
                kind: 1,
                pad: 0,
            },
        });
        match &p.shape {
            Shape::Sphere(s) => prims.push(ffi::ScPrimitive {
                center: s.center.to_array(),
                radius: s.radius,
                plane_start: 0,
                plane_count: 0,
                kind: 0,
                material,
            }),
            Shape::Solid(solid) => {
                let plane_start = planes.len() as u32;
                for pl in &solid.planes {
                    planes.push(ffi::ScPlane { normal: pl.normal.to_array(), d: pl.d });
                }
                prims.push(ffi::ScPrimitive {
                    center: [0.0; 3],
                    radius: 0.0,
                    plane_start,
                    plane_count: solid.planes.len() as u32,
                    kind: 1,
                    material,
                });
            }
        }
    }
    (prims, planes, mats)
}

pub fn camera_record(camera: &Camera) -> ffi::ScCamera {
    let (o, ll, h, v) = camera.view_basis();
    ffi::ScCamera { origin: o.to_array(), lower_left: ll.to_array(), horizontal: h.to_array(), vertical: v.to_array() }
}

pub fn beam_record(beam: &Beam) -> ffi::ScBeam {
    ffi::ScBeam { corner: beam.corner.to_array(), u: beam.u.to_array(), v: beam.v.to_array(), dir: beam.dir.to_array() }
}

/// Single-scatter weights (spectral-gpu/src/vol_photons.rs:256-267).
#[derive(Clone, Copy, Debug)]
pub struct VolWeights {
    pub sigma_s: f32,
    pub sigma_t: f32,
    pub g: f32,
}

impl Default for VolWeights {
    /// DSOTM defaults: sigma_s 0.5, sigma_t 0.06, g 0.5.
    fn default() -> Self {
        VolWeights { sigma_s: 0.5, sigma_t: 0.06, g: 0.5 }
    }
}

/// One CUDA device and the sensor tables (GpuContext, spectral-gpu/src/lib.rs:21-62).
pub struct CudaContext {
    raw: *mut ffi::ScCtx,
}

impl CudaContext {
    /// The context on device 0, or None without a usable sm_100 device.
    pub fn new() -> Option<Self> {
        Self::on_device(0)
    }

    pub fn on_device(device: i32) -> Option<Self> {
        let tables = sample_tables();
        let mut raw = std::ptr::null_mut();
        let rc = unsafe { ffi::sc_ctx_create(device, tables.as_ptr(), &mut raw) };
        if rc == ffi::SC_E_NODEVICE {
            return None;
        }
        check(rc);
        Some(CudaContext { raw })
    }

    pub fn synchronize(&self) {
        check(unsafe { ffi::sc_ctx_synchronize(self.raw) });
    }
}

impl Drop for CudaContext {
    fn drop(&mut self) {
        unsafe { ffi::sc_ctx_destroy(self.raw) };
    }
}

/// Forward photon tracing with single-scatter haze into a 64-bit fixed-point
/// film (GpuPhotonFilm, spectral-gpu/src/vol_photons.rs:228-851).  `accum` is
/// the interleaved XYZ image (3 * width * height).
pub struct GpuPhotonFilm<'ctx> {
    raw: *mut ffi::ScPhotonFilm,
    _ctx: &'ctx CudaContext,
    pub width: usize,
    pub height: usize,
    accum: Vec<f32>,
    surface: Vec<f32>,
}

impl<'ctx> GpuPhotonFilm<'ctx> {
    /// GpuPhotonFilm::new (vol_photons.rs:275-287).
    #[allow(clippy::too_many_arguments)]
    pub fn new(ctx: &'ctx CudaContext, scene: Scene, camera: &Camera, beam: &Beam, width: usize, height: usize,
               n_photons: u32, seed: u32, max_dist: f32, weights: VolWeights, zbuffer: Option<&[f32]>) -> Self {
        Self::with_options(ctx, scene, camera, beam, width, height, n_photons, seed, max_dist, weights, zbuffer,
                           ffi::ScFilmOptions::default())
    }

    /// The same with the film options beyond the reference (spectral bins,
    /// band, bounce count, estimator, haze arithmetic).
    #[allow(clippy::too_many_arguments)]
    pub fn with_options(ctx: &'ctx CudaContext, scene: Scene, camera: &Camera, beam: &Beam, width: usize,
                        height: usize, n_photons: u32, seed: u32, max_dist: f32, weights: VolWeights,
                        zbuffer: Option<&[f32]>, opts: ffi::ScFilmOptions) -> Self {
        let (prims, planes, mats) = flatten_scene(&scene);
        if let Some(z) = zbuffer {
            assert_eq!(z.len(), width * height, "zbuffer length");
        }
        let cam = camera_record(camera);
        let b = beam_record(beam);
        let w = ffi::ScVolWeights { sigma_s: weights.sigma_s, sigma_t: weights.sigma_t, g: weights.g };
        let mut raw = std::ptr::null_mut();
        check(unsafe {
            ffi::sc_photon_film_create(ctx.raw, prims.as_ptr(), prims.len() as u32, planes.as_ptr(),
                                       planes.len() as u32, mats.as_ptr(), mats.len() as u32, scene.background, &cam,
                                       &b, width as u32, height as u32, n_photons, seed, max_dist, &w,
                                       zbuffer.map_or(std::ptr::null(), |z| z.as_ptr()), &opts, &mut raw)
        });
        GpuPhotonFilm { raw, _ctx: ctx, width, height, accum: vec![0.0; 3 * width * height],
                        surface: vec![0.0; 3 * width * height] }
    }

    fn resolve(&mut self) {
        check(unsafe { ffi::sc_photon_film_read_accum(self.raw, self.accum.as_mut_ptr()) });
    }

    /// trace_and_resolve (vol_photons.rs:582-585): photons [0, n).
    pub fn trace_and_resolve(&mut self, n_photons: u32, seed: u32) {
        check(unsafe { ffi::sc_photon_film_trace_and_resolve(self.raw, n_photons, seed) });
        self.resolve();
    }

    /// trace_chunked (vol_photons.rs:590-598).
    pub fn trace_chunked(&mut self, total: u32, seed: u32) {
        check(unsafe { ffi::sc_photon_film_trace_chunked(self.raw, total, seed) });
        self.resolve();
    }

    /// dispatch_photons (vol_photons.rs:633-635): photons [base, n_photons), asynchronous;
    /// `accum` catches up at the next resolve or clear.
    pub fn dispatch_photons(&mut self, base: u32, n_photons: u32, seed: u32) {
        check(unsafe { ffi::sc_photon_film_dispatch(self.raw, base, n_photons, seed) });
    }

    /// trace_debug (vol_photons.rs:727-779): per-photon records, film untouched.
    pub fn trace_debug(&mut self, n_photons: u32, seed: u32, debug_count: u32) -> Vec<ffi::ScDebugPhoton> {
        let blank = ffi::ScDebugPhoton { num_states: 0, lambda: 0.0, pad0: 0, pad1: 0, states: [[0.0; 4]; 18] };
        let mut out = vec![blank; debug_count as usize];
        check(unsafe { ffi::sc_photon_film_trace_debug(self.raw, n_photons, seed, debug_count, out.as_mut_ptr()) });
        out
    }

    /// set_spectral / spectral (vol_photons.rs:658-666).
    pub fn set_spectral(&mut self, on: bool) {
        check(unsafe { ffi::sc_photon_film_set_spectral(self.raw, on as c_int) });
    }

    pub fn spectral(&self) -> bool {
        let mut on: c_int = 0;
        check(unsafe { ffi::sc_photon_film_get_spectral(self.raw, &mut on) });
        on != 0
    }

    /// recompute_surface (vol_photons.rs:685-714): the rim pass for `camera`.
    pub fn recompute_surface(&mut self, camera: &Camera) {
        let cam = camera_record(camera);
        check(unsafe { ffi::sc_photon_film_recompute_surface(self.raw, &cam) });
        check(unsafe { ffi::sc_photon_film_read_surface(self.raw, self.surface.as_mut_ptr()) });
    }

    pub fn surface(&self) -> &[f32] {
        &self.surface
    }

    /// accum (vol_photons.rs:807-809).
    pub fn accum(&mut self) -> &[f32] {
        self.resolve();
        &self.accum
    }

    /// clear_film (vol_photons.rs:800-804): the 64-bit film is the accumulator.
    pub fn clear_film(&mut self) {
        check(unsafe { ffi::sc_photon_film_clear(self.raw) });
        self.accum.iter_mut().for_each(|v| *v = 0.0);
    }

    /// auto_expose / auto_expose_p997 / to_rgb8 (vol_photons.rs:823-850).
    pub fn auto_expose(&self, scale: f32) -> f32 {
        let mut e = 0.0f32;
        check(unsafe { ffi::sc_photon_film_auto_expose(self.raw, scale, &mut e) });
        e
    }

    pub fn auto_expose_p997(&self) -> f32 {
        let mut e = 0.0f32;
        check(unsafe { ffi::sc_photon_film_auto_expose_p997(self.raw, &mut e) });
        e
    }

    pub fn to_rgb8(&self, exposure: f32) -> Vec<u8> {
        let mut out = vec![0u8; 3 * self.width * self.height];
        check(unsafe { ffi::sc_photon_film_to_rgb8(self.raw, exposure, out.as_mut_ptr()) });
        out
    }

    /// Device buffers of the film for a collective across GPUs (films of
    /// disjoint photon ranges add up exactly): (film, film bytes, stream).
    pub fn device_film(&self) -> (*mut std::os::raw::c_void, usize, *mut std::os::raw::c_void) {
        let (mut f, mut fb, mut g, mut gb, mut s) =
            (std::ptr::null_mut(), 0usize, std::ptr::null_mut(), 0usize, std::ptr::null_mut());
        check(unsafe { ffi::sc_photon_film_device_buffers(self.raw, &mut f, &mut fb, &mut g, &mut gb, &mut s) });
        (f, fb, s)
    }
}

impl Drop for GpuPhotonFilm<'_> {
    fn drop(&mut self) {
        unsafe { ffi::sc_photon_film_destroy(self.raw) };
    }
}

/// Hero-wavelength camera path tracer (GpuTracer, spectral-gpu/src/lib.rs:165-389).
pub struct GpuTracer<'ctx> {
    raw: *mut ffi::ScTracer,
    _ctx: &'ctx CudaContext,
    width: usize,
    height: usize,
}

impl<'ctx> GpuTracer<'ctx> {
    /// GpuTracer::new (lib.rs:179-187).
    pub fn new(ctx: &'ctx CudaContext, scene: Scene, camera: Camera, width: usize, height: usize,
               illuminant: Illuminant, seed: u32) -> Self {
        let (prims, planes, mats) = flatten_scene(&scene);
        let cam = camera_record(&camera);
        let ill = match illuminant {
            Illuminant::D65 => 0u32,
            Illuminant::A => 1u32,
        };
        let mut raw = std::ptr::null_mut();
        check(unsafe {
            ffi::sc_tracer_create(ctx.raw, prims.as_ptr(), prims.len() as u32, planes.as_ptr(), planes.len() as u32,
                                  mats.as_ptr(), mats.len() as u32, scene.background,
                                  scene.horizon.is_some() as c_int, scene.horizon.unwrap_or(0.0), &cam,
                                  width as u32, height as u32, ill, seed, std::ptr::null(), &mut raw)
        });
        GpuTracer { raw, _ctx: ctx, width, height }
    }

    /// accumulate (lib.rs:307-321).
    pub fn accumulate(&mut self, spp: u32) {
        check(unsafe { ffi::sc_tracer_accumulate(self.raw, spp) });
    }

    /// read_xyz (lib.rs:324-357): mean XYZ per pixel, as (x, y, z) triples.
    pub fn read_xyz(&self) -> Vec<[f32; 3]> {
        let mut flat = vec![0.0f32; 3 * self.width * self.height];
        check(unsafe { ffi::sc_tracer_read_xyz(self.raw, flat.as_mut_ptr()) });
        flat.chunks_exact(3).map(|c| [c[0], c[1], c[2]]).collect()
    }

    pub fn set_spectral(&mut self, on: bool) {
        check(unsafe { ffi::sc_tracer_set_spectral(self.raw, on as c_int) });
    }

    pub fn set_camera(&mut self, camera: &Camera) {
        let cam = camera_record(camera);
        check(unsafe { ffi::sc_tracer_set_camera(self.raw, &cam) });
    }

    pub fn clear_accum(&mut self) {
        check(unsafe { ffi::sc_tracer_clear_accum(self.raw) });
    }

    pub fn dims(&self) -> (usize, usize) {
        (self.width, self.height)
    }
}

impl Drop for GpuTracer<'_> {
    fn drop(&mut self) {
        unsafe { ffi::sc_tracer_destroy(self.raw) };
    }
}

/// The synthetic atomic film (AtomicFilm, spectral-gpu/src/film.rs:40-305).
pub struct AtomicFilm<'ctx> {
    raw: *mut ffi::ScAtomicFilm,
    _ctx: &'ctx CudaContext,
    width: usize,
    height: usize,
}

impl<'ctx> AtomicFilm<'ctx> {
    pub fn new(ctx: &'ctx CudaContext, width: usize, height: usize) -> Self {
        let mut raw = std::ptr::null_mut();
        check(unsafe { ffi::sc_atomic_film_create(ctx.raw, width as u32, height as u32, &mut raw) });
        AtomicFilm { raw, _ctx: ctx, width, height }
    }

    pub fn splat(&mut self, seed: u32, n: u32) {
        check(unsafe { ffi::sc_atomic_film_splat(self.raw, seed, n) });
    }

    pub fn read_film_raw(&self) -> Vec<u32> {
        let mut out = vec![0u32; 3 * self.width * self.height];
        check(unsafe { ffi::sc_atomic_film_read_raw(self.raw, out.as_mut_ptr()) });
        out
    }

    pub fn resolve(&mut self) {
        check(unsafe { ffi::sc_atomic_film_resolve(self.raw) });
    }

    pub fn clear_film(&mut self) {
        check(unsafe { ffi::sc_atomic_film_clear_film(self.raw) });
    }

    pub fn clear_accum(&mut self) {
        check(unsafe { ffi::sc_atomic_film_clear_accum(self.raw) });
    }

    pub fn accum(&self) -> Vec<f32> {
        let mut out = vec![0.0f32; 3 * self.width * self.height];
        check(unsafe { ffi::sc_atomic_film_read_accum(self.raw, out.as_mut_ptr()) });
        out
    }

    pub fn auto_expose_accum(&self, scale: f32) -> f32 {
        let mut e = 0.0f32;
        check(unsafe { ffi::sc_atomic_film_auto_expose_accum(self.raw, scale, &mut e) });
        e
    }

    pub fn to_rgb8(&self, exposure: f32) -> Vec<u8> {
        let mut out = vec![0u8; 3 * self.width * self.height];
        check(unsafe { ffi::sc_atomic_film_to_rgb8(self.raw, exposure, out.as_mut_ptr()) });
        out
    }

    pub fn dims(&self) -> (usize, usize) {
        (self.width, self.height)
    }
}

impl Drop for AtomicFilm<'_> {
    fn drop(&mut self) {
        unsafe { ffi::sc_atomic_film_destroy(self.raw) };
    }
}

/// check_determinism (film.rs:282-305): Ok when two splat runs give the same
/// film, else the first differing index.
pub fn check_determinism(ctx: &CudaContext, width: u32, height: u32, seed: u32, n: u32) -> Result<(), usize> {
    let mut first: i64 = -1;
    check(unsafe { ffi::sc_atomic_film_check_determinism(ctx.raw, width, height, seed, n, &mut first) });
    if first < 0 { Ok(()) } else { Err(first as usize) }
}

/// One scene split over GPUs without an all-reduce: every process traces its
/// photon range into its own device film (`ffi::sc_trace_photons_device`),
/// maps the other processes' films with `ipc_import`, and reduces its band of
/// whole tile rows from the exact sum of all of them (`reduce_band_peers`);
/// the XYZ bands are then gathered by the caller's transport.
pub mod split {
    use super::{check, ffi, CudaContext};
    use std::os::raw::c_void;

    /// A CUDA IPC handle of the allocation holding `dev_ptr`, and the offset of
    /// `dev_ptr` in it, to send to the other processes.
    pub fn ipc_export(ctx: &CudaContext, dev_ptr: *const c_void) -> ([u8; 64], usize) {
        let mut handle = [0u8; 64];
        let mut offset = 0usize;
        check(unsafe { ffi::sc_ipc_export(ctx.raw, dev_ptr, handle.as_mut_ptr(), &mut offset) });
        (handle, offset)
    }

    /// Another process's device memory mapped into this context (close it with
    /// `ipc_close` before that process frees it).
    pub fn ipc_import(ctx: &CudaContext, handle: &[u8; 64], offset: usize) -> *mut c_void {
        let mut p = std::ptr::null_mut();
        check(unsafe { ffi::sc_ipc_import(ctx.raw, handle.as_ptr(), offset, &mut p) });
        p
    }

    pub fn ipc_close(ctx: &CudaContext, dev_ptr: *mut c_void, offset: usize) {
        check(unsafe { ffi::sc_ipc_close(ctx.raw, dev_ptr, offset) });
    }

    /// Rows [row_begin, row_end) of the XYZ image of the sum of `films` (device
    /// pointers, this GPU's and mapped peers'), written into `xyz_dev`.
    #[allow(clippy::too_many_arguments)]
    pub fn reduce_band_peers(ctx: &CudaContext, films: &[*const i64], width: u32, height: u32, channels: u32,
                             lambda_min: f32, lambda_max: f32, scale_log2: u32, row_begin: u32, row_end: u32,
                             xyz_dev: *mut f32, stream: *mut c_void) {
        check(unsafe {
            ffi::sc_sensor_reduce_peers(ctx.raw, width, height, channels, lambda_min, lambda_max, scale_log2,
                                        films.as_ptr(), films.len() as u32, row_begin, row_end, xyz_dev, stream)
        });
    }
}
