"""ctypes binding of the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference renderer's
CPU crate (spectral-core).  Only tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py load it; the product library never does.

Scenes are passed as the raw bytes of the flat records (same layout as the
reference's GPU upload PODs), so the oracle shares no code with the product.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
TABLES_CSV = os.path.join(os.path.dirname(HERE), "spectral_b200", "data", "sensor_tables.csv")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


if not os.path.exists(LIB_PATH):
    build()

F3 = C.c_float * 3


class or_prim(C.Structure):
    _fields_ = [("center", F3), ("radius", C.c_float), ("plane_start", C.c_uint32),
                ("plane_count", C.c_uint32), ("kind", C.c_uint32), ("material", C.c_uint32)]


class or_mat(C.Structure):
    _fields_ = [("reflectance", C.c_float), ("glass", C.c_uint32), ("kind", C.c_uint32), ("pad", C.c_uint32)]


class or_plane(C.Structure):
    _fields_ = [("normal", F3), ("d", C.c_float)]


class or_scene(C.Structure):
    _fields_ = [("prims", C.c_void_p), ("n_prims", C.c_uint32), ("planes", C.c_void_p), ("n_planes", C.c_uint32),
                ("mats", C.c_void_p), ("n_mats", C.c_uint32), ("background", C.c_float),
                ("has_horizon", C.c_int32), ("horizon", C.c_float)]


class or_beam(C.Structure):
    _fields_ = [("corner", F3), ("u", F3), ("v", F3), ("dir", F3)]


class or_camera(C.Structure):
    _fields_ = [("origin", F3), ("lower_left", F3), ("horizontal", F3), ("vertical", F3)]


class or_vol_params(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("seed", C.c_uint32), ("max_bounces", C.c_uint32),
                ("sigma_s", C.c_float), ("sigma_t", C.c_float), ("g", C.c_float), ("max_dist", C.c_float),
                ("lambda_min", C.c_float), ("lambda_range", C.c_float), ("spectral", C.c_uint32),
                ("bins", C.c_uint32), ("bin_min", C.c_float), ("bin_inv_width", C.c_float),
                ("scale", C.c_float), ("estimator", C.c_uint32)]


class or_tracer_ext(C.Structure):
    _fields_ = [("center", F3), ("radius", C.c_float), ("scale", C.c_float), ("rr_start", C.c_uint32)]


P = C.POINTER
_lib = C.CDLL(LIB_PATH)
_u32, _f32, _i32, _vp = C.c_uint32, C.c_float, C.c_int, C.c_void_p
for name, res, args in [
    ("or_pcg32", _u32, [_u32]),
    ("or_mix2", _u32, [_u32, _u32]),
    ("or_rng_draws_u32", None, [_u32, _u32, _u32, P(_u32)]),
    ("or_rng_draws_f32", None, [_u32, _u32, _u32, P(_f32)]),
    ("or_glass_n", _f32, [_u32, _f32]),
    ("or_glass_n_many", None, [_u32, P(_f32), C.c_size_t, P(_f32)]),
    ("or_tracer_set_spectral", None, [C.c_int]),
    ("or_set_fault", None, [C.c_int]),
    ("or_camera_proj_params", None, [C.c_void_p, P(_f32)]),
    ("or_load_tables_csv", _i32, [C.c_char_p]),
    ("or_get_tables", None, [P(_f32)]),
    ("or_cmf", None, [_f32, P(_f32)]),
    ("or_illuminant", _f32, [_u32, _f32]),
    ("or_integrate_illuminant", None, [_u32, P(_f32)]),
    ("or_xyz_to_linear_srgb", None, [P(_f32), P(_f32)]),
    ("or_tonemap_to_u8", None, [P(_f32), _f32, P(C.c_uint8)]),
    ("or_reflect", None, [P(_f32), P(_f32), P(_f32)]),
    ("or_refract", _i32, [P(_f32), P(_f32), _f32, _f32, P(_f32)]),
    ("or_fresnel", _f32, [_f32, _f32, _f32]),
    ("or_scene_intersect", _i32, [P(or_scene), P(_f32), P(_f32), P(_f32), P(_f32), P(_f32), P(_i32), P(_u32)]),
    ("or_camera_look_at", None, [P(_f32), P(_f32), P(_f32), _f32, _f32, P(or_camera)]),
    ("or_camera_primary_ray", None, [P(or_camera), _f32, _f32, P(_f32), P(_f32)]),
    ("or_camera_project", _i32, [P(or_camera), P(_f32), P(_f32)]),
    ("or_phase_hg", _f32, [_f32, _f32]),
    ("or_simulate_photon", _u32, [P(or_scene), P(or_beam), P(or_vol_params), _u32, _u32, P(_f32), P(_f32), P(_u32)]),
    ("or_render_point", None, [P(or_scene), P(or_camera), P(or_beam), P(or_vol_params), P(_f32), _u32, _u32,
                               P(_f32), P(C.c_int64), P(C.c_int64)]),
    ("or_render_point_mt", None, [P(or_scene), P(or_camera), P(or_beam), P(or_vol_params), P(_f32), _u32, _u32,
                                  P(C.c_int64), P(C.c_int64), _i32]),
    ("or_render_beam", None, [P(or_scene), P(or_camera), P(or_beam), P(or_vol_params), P(_f32), _u32, _u32, P(_f32)]),
    ("or_lighttrace", None, [P(or_scene), P(_f32), _u32, _u32, P(or_beam), P(or_vol_params), _u32, P(_f32)]),
    ("or_tracer_accumulate", None, [P(or_scene), P(or_camera), _u32, _u32, _u32, _u32, _u32, _u32, _u32, _u32, _u32,
                                    P(_f32)]),
    ("or_tracer_accumulate_mt", None, [P(or_scene), P(or_camera), _u32, _u32, _u32, _u32, _u32, _u32, _u32, P(_f32),
                                       _i32]),
    ("or_tracer_sample", None, [P(or_scene), P(or_camera), _u32, _u32, _u32, _u32, _u32, _u32, _u32, _u32, P(_f32)]),
    ("or_tracer_set_ext", None, [_vp]),
    ("or_scatter", _i32, [_u32, _f32, P(_f32), P(_f32), _i32, _f32, _u32, _u32, P(_f32), P(_f32)]),
    ("or_simulate_photon_fixed", _u32, [P(or_scene), P(or_beam), P(or_vol_params), _u32, _f32, _u32, P(_f32)]),
    ("or_mean_landing", _u32, [P(or_scene), P(_f32), P(or_beam), _f32, _u32, _u32, P(_f32)]),
    ("or_surface_rim", None, [P(or_scene), P(or_camera), _u32, _u32, P(_f32)]),
    ("or_scene_zbuffer", None, [P(or_scene), P(_f32), P(or_camera), _u32, _u32, P(_f32)]),
    ("or_synthetic_splat", None, [_u32, _u32, _u32, _u32, P(_u32)]),
    ("or_gather_tonemap", None, [P(_f32), P(_f32), _u32, _u32, _f32, _f32, _f32, P(C.c_uint8)]),
]:
    fn = getattr(_lib, name)
    fn.restype = res
    fn.argtypes = args

if _lib.or_load_tables_csv(TABLES_CSV.encode()) != 0:
    raise RuntimeError("oracle could not load sensor tables from %s" % TABLES_CSV)

lib = _lib


def fp(a):
    return a.ctypes.data_as(P(C.c_float))


def i64p(a):
    return a.ctypes.data_as(P(C.c_int64))


class OScene:
    """Oracle-side scene from raw record bytes (kept alive by this object)."""

    def __init__(self, prim_bytes, n_prims, plane_bytes, n_planes, mat_bytes, n_mats, background=0.0, horizon=None):
        self._p = (or_prim * max(1, n_prims)).from_buffer_copy(prim_bytes.ljust(32 * max(1, n_prims), b"\0"))
        self._pl = (or_plane * max(1, n_planes)).from_buffer_copy(plane_bytes.ljust(16 * max(1, n_planes), b"\0"))
        self._m = (or_mat * max(1, n_mats)).from_buffer_copy(mat_bytes.ljust(16 * max(1, n_mats), b"\0"))
        self.c = or_scene(C.cast(self._p, _vp), n_prims, C.cast(self._pl, _vp), n_planes, C.cast(self._m, _vp),
                          n_mats, float(background), 1 if horizon is not None else 0,
                          float(horizon) if horizon is not None else 0.0)


def camera_look_at(origin, target, up, vfov, aspect):
    c = or_camera()
    _lib.or_camera_look_at(F3(*origin), F3(*target), F3(*up), float(vfov), float(aspect), C.byref(c))
    return c


def vol_params(width, height, seed, sigma_s=0.5, sigma_t=0.06, g=0.5, max_dist=14.0, max_bounces=8,
               lambda_min=380.0, lambda_max=730.0, spectral=1, bins=0, scale_log2=32, estimator=0):
    lr = np.float32(lambda_max) - np.float32(lambda_min)
    inv_w = np.float32(bins) / lr if bins else np.float32(0.0)
    return or_vol_params(int(width), int(height), int(seed), int(max_bounces), float(sigma_s), float(sigma_t),
                         float(g), float(max_dist), float(lambda_min), float(lr), int(spectral), int(bins),
                         float(lambda_min), float(inv_w), float(2.0 ** scale_log2), int(estimator))


def render_point(scene, cam, beam, p, begin, end, zbuf=None, f32=True, xyz=True, spec=False, threads=1):
    npx = p.width * p.height
    img = np.zeros(3 * npx, np.float32) if f32 else None
    fx = np.zeros(3 * npx, np.int64) if xyz else None
    fs = np.zeros(npx * p.bins, np.int64) if spec else None
    z = fp(np.ascontiguousarray(zbuf, np.float32)) if zbuf is not None else None
    if threads > 1:
        _lib.or_render_point_mt(C.byref(scene.c), C.byref(cam), C.byref(beam), C.byref(p), z, begin, end,
                                i64p(fx) if xyz else None, i64p(fs) if spec else None, threads)
    else:
        _lib.or_render_point(C.byref(scene.c), C.byref(cam), C.byref(beam), C.byref(p), z, begin, end,
                             fp(img) if f32 else None, i64p(fx) if xyz else None, i64p(fs) if spec else None)
    return img, fx, fs


def render_beam(scene, cam, beam, p, begin, end, zbuf=None):
    """render_volumetric_scene (volume.rs:233-329), f32 XYZ image 3*w*h."""
    img = np.zeros(3 * p.width * p.height, np.float32)
    z = fp(np.ascontiguousarray(zbuf, np.float32)) if zbuf is not None else None
    _lib.or_render_beam(C.byref(scene.c), C.byref(cam), C.byref(beam), C.byref(p), z, begin, end, fp(img))
    return img


def simulate_photon(scene, beam, p, idx, max_pairs=9):
    st = np.zeros(8 * max_pairs, np.float32)
    lam = C.c_float()
    tir = C.c_uint32()
    n = _lib.or_simulate_photon(C.byref(scene.c), C.byref(beam), C.byref(p), idx, max_pairs, fp(st), C.byref(lam),
                                C.byref(tir))
    return n, lam.value, st.reshape(max_pairs, 2, 4), tir.value


def tracer_accumulate(scene, cam, w, h, illuminant, seed, spp, base=0, max_bounces=8, threads=8, ext=None,
                      out=None, spectral=True):
    """CpuTracer::accumulate into `out` (3*w*h f32 running sum); returns it.
    spectral=False: dielectrics at n(550 nm), as the GPU tracer's set_spectral(false)."""
    out = np.zeros(3 * w * h, np.float32) if out is None else out
    _lib.or_tracer_set_ext(C.byref(ext) if ext is not None else None)
    _lib.or_tracer_set_spectral(1 if spectral else 0)
    _lib.or_tracer_accumulate_mt(C.byref(scene.c), C.byref(cam), w, h, illuminant, seed, spp, base, max_bounces,
                                 fp(out), threads)
    _lib.or_tracer_set_spectral(1)
    _lib.or_tracer_set_ext(None)
    return out


def tables():
    out = np.zeros(5 * 71, np.float32)
    _lib.or_get_tables(fp(out))
    return out


def bin_weights(bins, lambda_min, lambda_max):
    """Bin-averaged CMF: mean of the clamped table lerp over 16 sub-bin
    midpoints per bin (f64 accumulation), as the sensor reduction uses."""
    out = np.zeros((3, bins), np.float32)
    width = (float(lambda_max) - float(lambda_min)) / bins
    c = np.zeros(3, np.float32)
    for b in range(bins):
        acc = [0.0, 0.0, 0.0]
        for j in range(16):
            nm = np.float32(float(lambda_min) + width * (b + (j + 0.5) / 16.0))
            _lib.or_cmf(float(nm), fp(c))
            for k in range(3):
                acc[k] += float(c[k])
        for k in range(3):
            out[k, b] = np.float32(acc[k] / 16.0)
    return out
