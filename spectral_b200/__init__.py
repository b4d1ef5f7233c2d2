"""spectral_b200: B200-native (sm_100a) forward light tracing, volumetric single
scatter and hero-wavelength camera tracing behind the C ABI in
``include/spectral_cuda.h``.

This package is the Python side of that ABI: thin classes with the names and
argument meaning of the reference renderer's ``spectral-gpu`` crate
(``GpuContext``, ``GpuPhotonFilm``, ``GpuTracer``, ``AtomicFilm``,
``VolWeights``, ``dsotm_scene``), scene builders, and numpy views of results.
All compute runs in ``libspectral_cuda.so``; there is no CPU fallback.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib

BK7, SF11, WATER, FUSED_SILICA = 0, 1, 2, 3
D65, ILLUMINANT_A = 0, 1


def _f3(v):
    return _lib.F3(*[float(x) for x in v])


def f32_normalize(v):
    """glam Vec3::normalize in f32: v * (1 / sqrt((x*x + y*y) + z*z))."""
    x, y, z = (np.float32(c) for c in v)
    ln = np.sqrt(x * x + y * y + z * z, dtype=np.float32)
    r = np.float32(1.0) / ln
    return (x * r, y * r, z * r)


def f32_scale(v, s):
    s = np.float32(s)
    return tuple(np.float32(c) * s for c in v)


def sample_tables(path=_lib.TABLES_CSV):
    """The 5x71 sensor table [xbar;71][ybar;71][zbar;71][d65;71][a;71]
    (spectral-gpu/src/data.rs:12-22)."""
    out = (C.c_float * (5 * 71))()
    check(lib.sc_load_sensor_tables(path.encode(), out))
    return np.ctypeslib.as_array(out).copy()


class Lambertian:
    def __init__(self, reflectance):
        self.reflectance = float(reflectance)


class Dielectric:
    def __init__(self, glass):
        self.glass = int(glass)


class Scene:
    """Primitives + materials + background (spectral-core/src/scene.rs:17-32),
    flattened exactly like spectral-gpu's flatten_scene (vol_photons.rs:118-183)."""

    def __init__(self, background=1.0, horizon=None):
        self.background = float(background)
        self.horizon = horizon
        self.prims, self.planes, self.mats = [], [], []

    def _mat(self, material):
        m = _lib.sc_material()
        if isinstance(material, Lambertian):
            m.kind, m.reflectance, m.glass = 0, material.reflectance, 0
        else:
            m.kind, m.reflectance, m.glass = 1, 0.0, material.glass
        self.mats.append(m)
        return len(self.mats) - 1

    def add_sphere(self, center, radius, material):
        p = _lib.sc_primitive()
        p.center, p.radius, p.kind = _f3(center), float(radius), 0
        p.material = self._mat(material)
        self.prims.append(p)

    def add_solid(self, planes, material):
        """planes: iterable of (normal xyz, d); half-space n.x + d <= 0."""
        p = _lib.sc_primitive()
        p.kind, p.plane_start = 1, len(self.planes)
        for n, d in planes:
            pl = _lib.sc_plane()
            pl.normal, pl.d = _f3(n), float(d)
            self.planes.append(pl)
        p.plane_count = len(self.planes) - p.plane_start
        p.material = self._mat(material)
        self.prims.append(p)

    def arrays(self):
        prims = (_lib.sc_primitive * max(1, len(self.prims)))(*self.prims)
        planes = (_lib.sc_plane * max(1, len(self.planes)))(*self.planes)
        mats = (_lib.sc_material * max(1, len(self.mats)))(*self.mats)
        return prims, len(self.prims), planes, len(self.planes), mats, len(self.mats)


class Camera:
    """Pinhole camera (spectral-core/src/camera.rs:5-69) as its view basis."""

    def __init__(self, c):
        self.c = c

    @classmethod
    def look_at(cls, origin, target, up, vfov_deg, aspect):
        c = _lib.sc_camera()
        check(lib.sc_camera_look_at(_f3(origin), _f3(target), _f3(up), float(vfov_deg), float(aspect), C.byref(c)))
        return cls(c)

    def view_basis(self):
        c = self.c
        return tuple(tuple(getattr(c, k)) for k in ("origin", "lower_left", "horizontal", "vertical"))

    def origin(self):
        return tuple(self.c.origin)


class Beam:
    """Collimated source (spectral-core/src/lighttrace.rs:116-121)."""

    def __init__(self, corner, u, v, dir):
        self.c = _lib.sc_beam(_f3(corner), _f3(u), _f3(v), _f3(dir))

    @classmethod
    def from_c(cls, c):
        b = cls.__new__(cls)
        b.c = c
        return b


class VolWeights:
    """Single-scatter weights (spectral-gpu/src/vol_photons.rs:256-267); DSOTM defaults."""

    def __init__(self, sigma_s=0.5, sigma_t=0.06, g=0.5):
        self.sigma_s, self.sigma_t, self.g = float(sigma_s), float(sigma_t), float(g)

    def c(self):
        return _lib.sc_vol_weights(self.sigma_s, self.sigma_t, self.g)


def camera_proj_params(camera):
    """camera_proj_params (spectral-gpu/src/vol_photons.rs:100-115): 4x4 float32,
    rows (origin, 0), (u_hat, vw), (v_hat, vh), (w, 0)."""
    out = np.empty(16, np.float32)
    check(lib.sc_camera_proj_params(C.byref(camera.c), out.ctypes.data_as(C.POINTER(C.c_float))))
    return out.reshape(4, 4)


def glass_n(glass, lambda_nm):
    """Glass::n (spectral-core/src/sellmeier.rs:28-44) of one wavelength in nm,
    or, for an array, of every element (float32 array of the same shape)."""
    if np.ndim(lambda_nm) == 0:
        return lib.sc_glass_n(int(glass), float(lambda_nm))
    lam = np.ascontiguousarray(lambda_nm, dtype=np.float32)
    out = np.empty_like(lam)
    check(lib.sc_glass_n_many(int(glass), lam.ctypes.data_as(C.POINTER(C.c_float)), lam.size,
                              out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def dsotm_scene(aspect=1.0):
    """(Scene, Beam, Camera) of spectral-gpu/src/vol_photons.rs:188-222."""
    prim, mat = _lib.sc_primitive(), _lib.sc_material()
    planes = (_lib.sc_plane * 5)()
    beam, cam = _lib.sc_beam(), _lib.sc_camera()
    check(lib.sc_dsotm_scene(float(aspect), C.byref(prim), planes, C.byref(mat), C.byref(beam), C.byref(cam)))
    s = Scene(background=0.0)
    s.add_solid([(tuple(p.normal), p.d) for p in planes], Dielectric(SF11))
    return s, Beam.from_c(beam), Camera(cam)


def tir_beam():
    """The steep beam of spectral-gpu/src/vol_photons.rs:1259-1274 that makes
    violet photons totally internally reflect at the DSOTM prism's exit face."""
    bdir = f32_normalize((0.934, 0.358, 0.0))
    bperp = f32_scale(f32_normalize((-0.358, 0.934, 0.0)), 0.6)
    return Beam((-3.0, -1.1, -0.6), (0.0, 0.0, 1.2), bperp, bdir)


class GpuContext:
    """GpuContext (spectral-gpu/src/lib.rs:21-41): one CUDA device + the sensor tables."""

    def __init__(self, device=0, tables=None):
        self.tables = sample_tables() if tables is None else np.ascontiguousarray(tables, dtype=np.float32)
        self.h = C.c_void_p()
        check(lib.sc_ctx_create(int(device), self.tables.ctypes.data_as(C.POINTER(C.c_float)), C.byref(self.h)))

    @classmethod
    def new(cls, device=0, tables=None):
        """GpuContext::new (spectral-gpu/src/lib.rs:29-41): the context, or None
        when no usable sm_100 device is present (the reference's Option).  Any
        other failure (a bad device index or table, a CUDA error) raises."""
        try:
            return cls(device, tables)
        except _lib.SpectralError as e:
            if e.code == _lib.SC_E_NODEVICE:
                return None
            raise

    def synchronize(self):
        check(lib.sc_ctx_synchronize(self.h))

    def close(self):
        if self.h:
            lib.sc_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


POINT, ISOTROPIC, BEAM, FREE_FLIGHT = 0, 1, 2, 3


class GpuPhotonFilm:
    """GpuPhotonFilm (spectral-gpu/src/vol_photons.rs:228-851) on sm_100a.

    Extra keyword arguments select the film beyond the reference: ``bins`` (0 =
    XYZ film, N = spectral bins), the emission band, ``max_bounces``,
    ``scale_log2`` (default 2^32, 2^40 for the beam estimator) and
    ``estimator``: POINT (render_volumetric_scene_point, the GPU path of the
    reference), ISOTROPIC (render_volumetric), BEAM (render_volumetric_scene,
    spectral-core/src/volume.rs:170-329) or FREE_FLIGHT (the point estimator
    with free-flight distances and 1/pdf weights; no reference counterpart).
    ``haze_exact=True`` runs the haze samples in the CPU crate's operation
    order (films within a few fixed-point quanta of it, slower); by default
    they run in fast f32 arithmetic (the same photon paths and RNG stream)."""

    def __init__(self, ctx, scene, camera, beam, width, height, n_photons, seed, max_dist, weights=None,
                 zbuffer=None, bins=0, lambda_min=380.0, lambda_max=730.0, max_bounces=8, scale_log2=None,
                 estimator=0, haze_exact=False):
        if scale_log2 is None:
            scale_log2 = 40 if estimator == BEAM else 32
        self.ctx = ctx
        self.width, self.height = int(width), int(height)
        weights = weights or VolWeights()
        prims, np_, planes, npl, mats, nm = scene.arrays()
        opts = _lib.sc_film_options(int(bins), float(lambda_min), float(lambda_max), int(max_bounces),
                                    int(scale_log2), int(estimator), int(bool(haze_exact)))
        z = None
        if zbuffer is not None:
            z = np.ascontiguousarray(zbuffer, dtype=np.float32)
            if z.size != self.width * self.height:
                raise ValueError("zbuffer length %d != width*height %d" % (z.size, self.width * self.height))
        self.h = C.c_void_p()
        check(lib.sc_photon_film_create(ctx.h, prims, np_, planes, npl, mats, nm, scene.background,
                                        C.byref(camera.c), C.byref(beam.c), self.width, self.height,
                                        int(n_photons), int(seed), float(max_dist), C.byref(weights.c()),
                                        _fptr(z) if z is not None else None, C.byref(opts), C.byref(self.h)))
        w, h, ch = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib.sc_photon_film_dims(self.h, C.byref(w), C.byref(h), C.byref(ch)))
        self.channels = ch.value

    MAX_PER_DISPATCH = 4_000_000

    def trace_and_resolve(self, n_photons, seed):
        check(lib.sc_photon_film_trace_and_resolve(self.h, int(n_photons), int(seed)))

    def trace_chunked(self, total_photons, seed):
        check(lib.sc_photon_film_trace_chunked(self.h, int(total_photons), int(seed)))

    def dispatch_photons(self, photon_base, n_photons, seed):
        check(lib.sc_photon_film_dispatch(self.h, int(photon_base), int(n_photons), int(seed)))

    def trace_debug(self, n_photons, seed, debug_count):
        """Per-photon (origin, dir) records; a numpy structured view of DebugPhotonGpu."""
        recs = (_lib.sc_debug_photon * max(1, int(debug_count)))()
        check(lib.sc_photon_film_trace_debug(self.h, int(n_photons), int(seed), int(debug_count), recs))
        n = min(int(debug_count), int(n_photons))
        raw = np.frombuffer(recs, dtype=np.uint8, count=304 * max(1, int(debug_count)))
        num = raw.view(np.uint32)[0::76][:n].copy()
        lam = raw.view(np.float32)[1::76][:n].copy()
        states = raw.view(np.float32).reshape(-1, 76)[:n, 4:].reshape(n, 18, 4).copy()
        return num, lam, states

    def set_spectral(self, on):
        check(lib.sc_photon_film_set_spectral(self.h, 1 if on else 0))

    def spectral(self):
        v = C.c_int()
        check(lib.sc_photon_film_get_spectral(self.h, C.byref(v)))
        return bool(v.value)

    def set_camera(self, camera):
        check(lib.sc_photon_film_set_camera(self.h, C.byref(camera.c)))

    def recompute_surface(self, camera=None):
        check(lib.sc_photon_film_recompute_surface(self.h, C.byref(camera.c) if camera is not None else None))

    def surface(self):
        out = np.empty(3 * self.width * self.height, np.float32)
        check(lib.sc_photon_film_read_surface(self.h, _fptr(out)))
        return out

    def accum(self):
        out = np.empty(3 * self.width * self.height, np.float32)
        check(lib.sc_photon_film_read_accum(self.h, _fptr(out)))
        return out

    def read_raw(self):
        out = np.empty((self.height, self.width, self.channels), np.int64)
        check(lib.sc_photon_film_read_raw(self.h, out.ctypes.data_as(C.POINTER(C.c_int64))))
        return out

    def clear_film(self):
        check(lib.sc_photon_film_clear(self.h))

    def auto_expose(self, scale):
        v = C.c_float()
        check(lib.sc_photon_film_auto_expose(self.h, float(scale), C.byref(v)))
        return v.value

    def auto_expose_p997(self):
        v = C.c_float()
        check(lib.sc_photon_film_auto_expose_p997(self.h, C.byref(v)))
        return v.value

    def to_rgb8(self, exposure):
        out = np.empty(3 * self.width * self.height, np.uint8)
        check(lib.sc_photon_film_to_rgb8(self.h, float(exposure), out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    def gather_rgba8(self, total_photons, target_n=4_000_000.0, kradius=2.0, exposure=1.0):
        out = np.empty(4 * self.width * self.height, np.uint8)
        check(lib.sc_photon_film_gather_rgba8(self.h, int(total_photons), float(target_n), float(kradius),
                                              float(exposure), out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    def dims(self):
        return self.width, self.height

    def set_scene(self, scene, camera, beam):
        prims, np_, planes, npl, mats, nm = scene.arrays()
        check(lib.sc_photon_film_set_scene(self.h, prims, np_, planes, npl, mats, nm, C.byref(camera.c),
                                           C.byref(beam.c)))

    def trace_stats(self, photon_base, count, seed):
        """(photons, segments, in-frame haze samples, scatters) of a photon range."""
        out = (C.c_uint64 * 4)()
        check(lib.sc_photon_film_trace_stats(self.h, int(photon_base), int(count), int(seed), out))
        return tuple(out)

    def close(self):
        if self.h:
            lib.sc_photon_film_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuTracer:
    """GpuTracer (spectral-gpu/src/lib.rs:165-389): wavefront hero-wavelength
    camera tracer.  Keyword extensions (no reference counterpart): max_depth,
    rr_start, emitter=(center, radius, scale); scheduling only: wave_bounces
    (compacted wavefront bounces before the in-place tail), chains (waves in
    flight) and wave_paths_log2 (paths per wave)."""

    def __init__(self, ctx, scene, camera, width, height, illuminant=D65, seed=0, max_depth=8, rr_start=0,
                 emitter=None, wave_bounces=0, chains=0, wave_paths_log2=0):
        self.width, self.height = int(width), int(height)
        prims, np_, planes, npl, mats, nm = scene.arrays()
        opts = _lib.sc_tracer_options()
        opts.max_depth, opts.rr_start, opts.wave_bounces = int(max_depth), int(rr_start), int(wave_bounces)
        opts.chains, opts.wave_paths_log2 = int(chains), int(wave_paths_log2)
        if emitter is not None:
            c, r, s = emitter
            opts.emitter_center, opts.emitter_radius, opts.emitter_scale = _f3(c), float(r), float(s)
        self.h = C.c_void_p()
        check(lib.sc_tracer_create(ctx.h, prims, np_, planes, npl, mats, nm, scene.background,
                                   1 if scene.horizon is not None else 0,
                                   float(scene.horizon) if scene.horizon is not None else 0.0, C.byref(camera.c),
                                   self.width, self.height, int(illuminant), int(seed), C.byref(opts),
                                   C.byref(self.h)))

    def accumulate(self, spp):
        check(lib.sc_tracer_accumulate(self.h, int(spp)))

    def read_xyz(self):
        out = np.empty(3 * self.width * self.height, np.float32)
        check(lib.sc_tracer_read_xyz(self.h, _fptr(out)))
        return out

    def set_camera(self, camera):
        check(lib.sc_tracer_set_camera(self.h, C.byref(camera.c)))

    def set_spectral(self, on):
        """set_spectral (spectral-gpu/src/lib.rs:369-372): off = dielectrics at n(550 nm)."""
        check(lib.sc_tracer_set_spectral(self.h, 1 if on else 0))

    def set_rows(self, row_begin, row_end):
        """Trace only rows [row_begin, row_end) in later accumulate calls."""
        check(lib.sc_tracer_set_rows(self.h, int(row_begin), int(row_end)))

    def clear_accum(self):
        check(lib.sc_tracer_clear_accum(self.h))

    def dims(self):
        return self.width, self.height

    def stats(self):
        p, s = C.c_uint64(), C.c_uint64()
        check(lib.sc_tracer_last_stats(self.h, C.byref(p), C.byref(s)))
        return p.value, s.value

    def close(self):
        if self.h:
            lib.sc_tracer_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


N_SPLATS = 1_000_000


class AtomicFilm:
    """AtomicFilm (spectral-gpu/src/film.rs:40-277): u32 x4096 film + f32 accumulator."""

    def __init__(self, ctx, width, height):
        self.width, self.height = int(width), int(height)
        self.h = C.c_void_p()
        check(lib.sc_atomic_film_create(ctx.h, self.width, self.height, C.byref(self.h)))

    def splat(self, seed, n_splats=N_SPLATS):
        check(lib.sc_atomic_film_splat(self.h, int(seed), int(n_splats)))

    def read_film_raw(self):
        out = np.empty(3 * self.width * self.height, np.uint32)
        check(lib.sc_atomic_film_read_raw(self.h, out.ctypes.data_as(C.POINTER(C.c_uint32))))
        return out

    def resolve(self):
        check(lib.sc_atomic_film_resolve(self.h))

    def accum(self):
        out = np.empty(3 * self.width * self.height, np.float32)
        check(lib.sc_atomic_film_read_accum(self.h, _fptr(out)))
        return out

    def clear_film(self):
        check(lib.sc_atomic_film_clear_film(self.h))

    def clear_accum(self):
        check(lib.sc_atomic_film_clear_accum(self.h))

    def auto_expose_accum(self, scale=1.0):
        """auto_expose_accum (spectral-gpu/src/film.rs:262-270) on the device."""
        e = C.c_float()
        check(lib.sc_atomic_film_auto_expose_accum(self.h, float(scale), C.byref(e)))
        return e.value

    def to_rgb8(self, exposure):
        """to_rgb8 (spectral-gpu/src/film.rs:243-258): 3*w*h bytes."""
        out = np.empty(3 * self.width * self.height, np.uint8)
        check(lib.sc_atomic_film_to_rgb8(self.h, float(exposure), out.ctypes.data_as(C.POINTER(C.c_uint8))))
        return out

    def dims(self):
        return self.width, self.height

    def close(self):
        if self.h:
            lib.sc_atomic_film_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def check_determinism(ctx, width, height, seed, n_splats):
    """check_determinism (spectral-gpu/src/film.rs:282-305): None if identical,
    else the first differing index."""
    d = C.c_int64()
    check(lib.sc_atomic_film_check_determinism(ctx.h, int(width), int(height), int(seed), int(n_splats),
                                               C.byref(d)))
    return None if d.value < 0 else d.value


class Screen:
    """lighttrace::Screen (spectral-core/src/lighttrace.rs:14-112): a receiving
    rectangle corner + s*u + r*v of width x height texels whose ``sum`` holds
    the deposited XYZ (row 0 at r = 1), filled on the GPU by ``trace``."""

    def __init__(self, corner, u, v, width, height):
        self.corner, self.u, self.v = tuple(map(float, corner)), tuple(map(float, u)), tuple(map(float, v))
        self.width, self.height = int(width), int(height)
        self.sum = np.zeros((self.width * self.height, 3), np.float32)

    def c(self):
        return _lib.sc_screen(_f3(self.corner), _f3(self.u), _f3(self.v))

    def scaled(self, scale):
        return self.sum * np.float32(scale)


def trace(ctx, scene, screen, beam, n, seed, lambda_min=380.0, lambda_max=730.0, max_bounces=8, scale_log2=32):
    """lighttrace::trace (lighttrace.rs:157-166): photons 0..n from the beam,
    splatted bilinearly into ``screen.sum`` (accumulated, like the reference)."""
    prims, np_, planes, npl, mats, nm = scene.arrays()
    opts = _lib.sc_film_options(0, float(lambda_min), float(lambda_max), int(max_bounces), int(scale_log2), 0)
    out = np.zeros(3 * screen.width * screen.height, np.float32)
    check(lib.sc_lighttrace(ctx.h, prims, np_, planes, npl, mats, nm, C.byref(screen.c()), screen.width,
                            screen.height, C.byref(beam.c), int(n), int(seed), C.byref(opts), _fptr(out)))
    screen.sum += out.reshape(-1, 3)
    return screen


def scene_zbuffer(ctx, scene, camera, width, height, floor=None):
    """The z-buffer pass of spectral-core/examples/prism_on_plane.rs:125-160:
    per pixel the distance to the nearer of the scene and the ``floor`` Screen
    along the primary ray, +INF where nothing is hit (width*height floats)."""
    prims, np_, planes, npl, mats, nm = scene.arrays()
    out = np.zeros(int(width) * int(height), np.float32)
    check(lib.sc_scene_zbuffer(ctx.h, prims, np_, planes, npl, mats, nm,
                               C.byref(floor.c()) if floor is not None else None, C.byref(camera.c), int(width),
                               int(height), _fptr(out)))
    return out
