"""ctypes binding of ``include/spectral_cuda.h`` (the library's C ABI).

The shared library is loaded from the package directory.  There is no CPU
fallback: if the library is missing, importing this module raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspectral_cuda.so")
TABLES_CSV = os.path.join(HERE, "data", "sensor_tables.csv")

SC_OK = 0
SC_E_INVALID = -1
SC_E_CUDA = -2
SC_E_NOMEM = -3
SC_E_LIMIT = -4
SC_E_TIMEOUT = -5
SC_E_STATE = -6
SC_E_NODEVICE = -7
SC_MAX_PRIMS = 64
SC_MAX_PLANES = 256
SC_MAX_BINS = 256

F3 = C.c_float * 3


class sc_primitive(C.Structure):
    _fields_ = [("center", F3), ("radius", C.c_float), ("plane_start", C.c_uint32),
                ("plane_count", C.c_uint32), ("kind", C.c_uint32), ("material", C.c_uint32)]


class sc_material(C.Structure):
    _fields_ = [("reflectance", C.c_float), ("glass", C.c_uint32), ("kind", C.c_uint32), ("pad", C.c_uint32)]


class sc_plane(C.Structure):
    _fields_ = [("normal", F3), ("d", C.c_float)]


class sc_beam(C.Structure):
    _fields_ = [("corner", F3), ("u", F3), ("v", F3), ("dir", F3)]


class sc_camera(C.Structure):
    _fields_ = [("origin", F3), ("lower_left", F3), ("horizontal", F3), ("vertical", F3)]


class sc_screen(C.Structure):
    _fields_ = [("corner", F3), ("u", F3), ("v", F3)]


class sc_vol_weights(C.Structure):
    _fields_ = [("sigma_s", C.c_float), ("sigma_t", C.c_float), ("g", C.c_float)]


class sc_debug_photon(C.Structure):
    _fields_ = [("num_states", C.c_uint32), ("lambda_", C.c_float), ("pad0", C.c_uint32), ("pad1", C.c_uint32),
                ("states", (C.c_float * 4) * 18)]


class sc_film_options(C.Structure):
    _fields_ = [("bins", C.c_uint32), ("lambda_min", C.c_float), ("lambda_max", C.c_float),
                ("max_bounces", C.c_uint32), ("scale_log2", C.c_uint32), ("estimator", C.c_uint32),
                ("haze_exact", C.c_uint32)]


class sc_tracer_options(C.Structure):
    _fields_ = [("max_depth", C.c_uint32), ("rr_start", C.c_uint32), ("emitter_center", F3),
                ("emitter_radius", C.c_float), ("emitter_scale", C.c_float), ("wave_bounces", C.c_uint32),
                ("chains", C.c_uint32), ("wave_paths_log2", C.c_uint32)]


class sc_trace_desc(C.Structure):
    _fields_ = [("prims", C.c_void_p), ("n_prims", C.c_uint32), ("planes", C.c_void_p), ("n_planes", C.c_uint32),
                ("mats", C.c_void_p), ("n_mats", C.c_uint32), ("cam", sc_camera), ("beam", sc_beam),
                ("weights", sc_vol_weights), ("width", C.c_uint32), ("height", C.c_uint32), ("seed", C.c_uint32),
                ("spectral", C.c_uint32), ("max_dist", C.c_float), ("opts", sc_film_options),
                ("zbuffer", C.c_void_p)]


class sc_scene_job(C.Structure):
    _fields_ = [("n_prims", C.c_uint32), ("n_planes", C.c_uint32), ("n_mats", C.c_uint32), ("spectral", C.c_uint32),
                ("prims", sc_primitive * 4), ("planes", sc_plane * 16), ("mats", sc_material * 4),
                ("cam", sc_camera), ("beam", sc_beam), ("weights", sc_vol_weights), ("width", C.c_uint32),
                ("height", C.c_uint32), ("n_photons", C.c_uint32), ("seed", C.c_uint32), ("max_dist", C.c_float),
                ("opts", sc_film_options)]


class sc_batch_tuning(C.Structure):
    _fields_ = [("chunk_photons", C.c_uint32), ("minb", C.c_uint32), ("aggregate", C.c_uint32), ("grid", C.c_uint32),
                ("per_photon", C.c_uint32), ("block", C.c_uint32)]


class sc_server_config(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_slots", C.c_uint32), ("chunk_photons", C.c_uint32),
                ("warp_split", C.c_uint32)]


class sc_request(C.Structure):
    _fields_ = [("job", sc_scene_job), ("frames", C.c_uint32), ("orbit_deg", C.c_float), ("orbit_target", F3),
                ("orbit_up", F3), ("vfov_deg", C.c_float)]


assert C.sizeof(sc_primitive) == 32 and C.sizeof(sc_material) == 16 and C.sizeof(sc_plane) == 16
assert C.sizeof(sc_debug_photon) == 304

P = C.POINTER
_u32, _i32, _f32, _u64, _i64, _vp, _sz = C.c_uint32, C.c_int, C.c_float, C.c_uint64, C.c_int64, C.c_void_p, C.c_size_t

# name -> (restype, argtypes)
PROTOTYPES = {
    "sc_last_error": (C.c_char_p, []),
    "sc_version": (C.c_char_p, []),
    "sc_ctx_create": (_i32, [_i32, P(_f32), P(_vp)]),
    "sc_ctx_destroy": (_i32, [_vp]),
    "sc_ctx_synchronize": (_i32, [_vp]),
    "sc_load_sensor_tables": (_i32, [C.c_char_p, P(_f32)]),
    "sc_camera_look_at": (_i32, [P(_f32), P(_f32), P(_f32), _f32, _f32, P(sc_camera)]),
    "sc_glass_n": (_f32, [_u32, _f32]),
    "sc_camera_proj_params": (_i32, [_vp, P(_f32)]),
    "sc_tracer_set_spectral": (_i32, [_vp, _i32]),
    "sc_tracer_set_rows": (_i32, [_vp, _u32, _u32]),
    "sc_atomic_film_auto_expose_accum": (_i32, [_vp, _f32, P(_f32)]),
    "sc_atomic_film_to_rgb8": (_i32, [_vp, _f32, P(C.c_uint8)]),
    "sc_glass_n_many": (_i32, [_u32, P(_f32), C.c_size_t, P(_f32)]),
    "sc_glass_n_device": (_i32, [_vp, _u32, _vp, C.c_size_t, _vp, _vp]),
    "sc_rng_draws": (_i32, [_vp, _u32, _u32, _u32, P(_u32)]),
    "sc_dsotm_scene": (_i32, [_f32, P(sc_primitive), P(sc_plane), P(sc_material), P(sc_beam), P(sc_camera)]),
    "sc_photon_film_create": (_i32, [_vp, P(sc_primitive), _u32, P(sc_plane), _u32, P(sc_material), _u32, _f32,
                                     P(sc_camera), P(sc_beam), _u32, _u32, _u32, _u32, _f32, P(sc_vol_weights),
                                     P(_f32), P(sc_film_options), P(_vp)]),
    "sc_photon_film_destroy": (_i32, [_vp]),
    "sc_photon_film_trace_and_resolve": (_i32, [_vp, _u32, _u32]),
    "sc_photon_film_trace_chunked": (_i32, [_vp, _u32, _u32]),
    "sc_photon_film_dispatch": (_i32, [_vp, _u32, _u32, _u32]),
    "sc_photon_film_trace_debug": (_i32, [_vp, _u32, _u32, _u32, P(sc_debug_photon)]),
    "sc_photon_film_set_spectral": (_i32, [_vp, _i32]),
    "sc_photon_film_get_spectral": (_i32, [_vp, P(_i32)]),
    "sc_photon_film_set_camera": (_i32, [_vp, P(sc_camera)]),
    "sc_photon_film_recompute_surface": (_i32, [_vp, P(sc_camera)]),
    "sc_photon_film_read_surface": (_i32, [_vp, P(_f32)]),
    "sc_photon_film_read_accum": (_i32, [_vp, P(_f32)]),
    "sc_photon_film_read_raw": (_i32, [_vp, P(_i64)]),
    "sc_photon_film_clear": (_i32, [_vp]),
    "sc_photon_film_auto_expose": (_i32, [_vp, _f32, P(_f32)]),
    "sc_photon_film_auto_expose_p997": (_i32, [_vp, P(_f32)]),
    "sc_photon_film_to_rgb8": (_i32, [_vp, _f32, P(C.c_uint8)]),
    "sc_photon_film_gather_rgba8": (_i32, [_vp, _u64, _f32, _f32, _f32, P(C.c_uint8)]),
    "sc_photon_film_dims": (_i32, [_vp, P(_u32), P(_u32), P(_u32)]),
    "sc_photon_film_set_scene": (_i32, [_vp, P(sc_primitive), _u32, P(sc_plane), _u32, P(sc_material), _u32,
                                        P(sc_camera), P(sc_beam)]),
    "sc_photon_film_trace_stats": (_i32, [_vp, _u32, _u32, _u32, P(_u64)]),
    "sc_photon_film_device_buffers": (_i32, [_vp, P(_vp), P(_sz), P(_vp), P(_sz), P(_vp)]),
    "sc_photon_film_mark_all_dirty": (_i32, [_vp]),
    "sc_trace_stats_device": (_i32, [_vp, P(sc_trace_desc), _u32, _u32, _vp, _vp]),
    "sc_tracer_create": (_i32, [_vp, P(sc_primitive), _u32, P(sc_plane), _u32, P(sc_material), _u32, _f32, _i32,
                                _f32, P(sc_camera), _u32, _u32, _u32, _u32, P(sc_tracer_options), P(_vp)]),
    "sc_tracer_destroy": (_i32, [_vp]),
    "sc_tracer_accumulate": (_i32, [_vp, _u32]),
    "sc_tracer_read_xyz": (_i32, [_vp, P(_f32)]),
    "sc_tracer_set_camera": (_i32, [_vp, P(sc_camera)]),
    "sc_tracer_clear_accum": (_i32, [_vp]),
    "sc_tracer_dims": (_i32, [_vp, P(_u32), P(_u32)]),
    "sc_tracer_last_stats": (_i32, [_vp, P(_u64), P(_u64)]),
    "sc_tracer_stream": (_i32, [_vp, P(_vp)]),
    "sc_atomic_film_create": (_i32, [_vp, _u32, _u32, P(_vp)]),
    "sc_atomic_film_destroy": (_i32, [_vp]),
    "sc_atomic_film_splat": (_i32, [_vp, _u32, _u32]),
    "sc_atomic_film_read_raw": (_i32, [_vp, P(_u32)]),
    "sc_atomic_film_resolve": (_i32, [_vp]),
    "sc_atomic_film_read_accum": (_i32, [_vp, P(_f32)]),
    "sc_atomic_film_clear_film": (_i32, [_vp]),
    "sc_atomic_film_clear_accum": (_i32, [_vp]),
    "sc_atomic_film_check_determinism": (_i32, [_vp, _u32, _u32, _u32, _u32, P(_i64)]),
    "sc_atomic_film_stream": (_i32, [_vp, P(_vp)]),
    "sc_lighttrace": (_i32, [_vp, P(sc_primitive), _u32, P(sc_plane), _u32, P(sc_material), _u32, P(sc_screen),
                             _u32, _u32, P(sc_beam), _u32, _u32, P(sc_film_options), P(_f32)]),
    "sc_scene_zbuffer": (_i32, [_vp, P(sc_primitive), _u32, P(sc_plane), _u32, P(sc_material), _u32, P(sc_screen),
                                P(sc_camera), _u32, _u32, P(_f32)]),
    "sc_batch_create": (_i32, [_vp, P(sc_scene_job), _u32, P(sc_batch_tuning), P(_vp)]),
    "sc_batch_destroy": (_i32, [_vp]),
    "sc_batch_autotune": (_i32, [_vp, P(sc_batch_tuning)]),
    "sc_batch_set_tuning": (_i32, [_vp, P(sc_batch_tuning)]),
    "sc_batch_get_tuning": (_i32, [_vp, P(sc_batch_tuning)]),
    "sc_batch_update_jobs": (_i32, [_vp, P(sc_scene_job), _u32]),
    "sc_batch_run": (_i32, [_vp, _vp]),
    "sc_batch_run_plain": (_i32, [_vp, _vp]),
    "sc_batch_synchronize": (_i32, [_vp]),
    "sc_batch_read_xyz": (_i32, [_vp, _u32, P(_f32)]),
    "sc_batch_read_all_xyz": (_i32, [_vp, P(_f32), _sz, _vp]),
    "sc_batch_read_all_xyz_async": (_i32, [_vp, P(_f32), _sz, _vp]),
    "sc_batch_info": (_i32, [_vp, P(_u64), P(_u64), P(_u64), P(_u64)]),
    "sc_batch_device_xyz": (_i32, [_vp, _u32, P(P(_f32))]),
    "sc_batch_stats": (_i32, [_vp, P(_u64)]),
    "sc_server_create": (_i32, [_vp, P(sc_server_config), P(_vp)]),
    "sc_server_destroy": (_i32, [_vp]),
    "sc_server_submit": (_i32, [_vp, P(sc_request), P(_u64)]),
    "sc_server_step": (_i32, [_vp, P(_u32)]),
    "sc_server_poll": (_i32, [_vp, P(_u64), P(_f32), _sz, P(_u32), P(_u32), P(C.c_double)]),
    "sc_server_cancel": (_i32, [_vp, _u64]),
    "sc_server_peek": (_i32, [_vp, _u64, P(_f32), _sz, P(_u32)]),
    "sc_server_stats": (_i32, [_vp, P(_u64), P(_u64), P(_u32), P(_u32), P(_u32)]),
    "sc_trace_xyz_noalloc": (_i32, [P(_f32), P(sc_trace_desc), _u32, _u32, _vp, _vp]),
    "sc_film_bytes": (_sz, [_u32, _u32, _u32]),
    "sc_ipc_export": (_i32, [_vp, _vp, P(C.c_ubyte), P(_sz)]),
    "sc_ipc_import": (_i32, [_vp, P(C.c_ubyte), _sz, P(_vp)]),
    "sc_ipc_close": (_i32, [_vp, _vp, _sz]),
    "sc_sensor_reduce_peers": (_i32, [_vp, _u32, _u32, _u32, _f32, _f32, _u32, P(_vp), _u32, _u32, _u32, _vp, _vp]),
    "sc_film_flag_bytes": (_sz, [_u32, _u32]),
    "sc_trace_photons_device": (_i32, [_vp, P(sc_trace_desc), _u32, _u32, _vp, _vp, _vp]),
    "sc_sensor_reduce_device": (_i32, [_vp, _u32, _u32, _u32, _f32, _f32, _u32, _vp, _vp, _vp, _i32, _vp]),
}


class SpectralError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("spectral_cuda error %d: %s" % (code, msg))
        self.code = code


def load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("spectral_cuda library not built: %s (run python spectral_b200/build.py)" % LIB_PATH)
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()


def check(code):
    if code != SC_OK:
        raise SpectralError(code, lib.sc_last_error().decode(errors="replace"))
    return code
