"""C ABI checks that need no GPU: the library loads, exports every function
declared in include/*.h, its host helpers agree bit-for-bit with the oracle,
and calls fail with status codes (never a crash or a CPU fallback)."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

import oracle
import spectral_b200 as sb
from spectral_b200 import _lib

from helpers import ocam

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \t\*]*?\b(sc_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert len(names) > 40
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes binding covers them all
    assert not (names - set(_lib.PROTOTYPES)), sorted(names - set(_lib.PROTOTYPES))


def test_version_string():
    assert b"sm_100a" in _lib.lib.sc_version()


def test_camera_look_at_bitwise_equals_oracle():
    for args in [((0.5, -0.5, 12.0), (0.5, -0.5, 0.0), (0, 1, 0), 42.0, 1.0),
                 ((0, 1, 5), (0, 0, 0), (0, 1, 0), 50.0, 1.5),
                 ((3.0, 2.0, 9.0), (0.1, -0.3, 0.2), (0, 1, 0), 35.0, 16 / 9)]:
        a = sb.Camera.look_at(*args)
        b = oracle.camera_look_at(*args)
        assert bytes(a.c) == bytes(b)


def test_glass_index_bitwise_equals_oracle():
    for g in range(4):
        for nm in np.linspace(380, 780, 81, dtype=np.float32):
            x, y = np.float32(sb.glass_n(g, float(nm))), np.float32(oracle.lib.or_glass_n(g, float(nm)))
            assert x.tobytes() == y.tobytes(), (g, nm)


def _all_f32(lo, hi):
    return np.arange(np.float32(lo).view(np.uint32), np.float32(hi).view(np.uint32) + 1,
                     dtype=np.uint32).view(np.float32)


def test_glass_index_every_f32_wavelength_equals_oracle():
    # every f32 wavelength of 380-780 nm (8.7 M values): the single-division
    # Sellmeier sum with its midpoint check returns the reference-order f32
    lam = _all_f32(380.0, 780.0)
    for g in range(4):
        got, ref = sb.glass_n(g, lam), np.empty_like(lam)
        oracle.lib.or_glass_n_many(g, oracle.fp(lam), lam.size, oracle.fp(ref))
        assert got.tobytes() == ref.tobytes(), (g, int((got != ref).sum()))
    with pytest.raises(_lib.SpectralError):
        sb.glass_n(4, lam[:4])


def test_camera_proj_params_bitwise_equals_oracle():
    for args in [((0.5, -0.5, 12.0), (0.5, -0.5, 0.0), (0, 1, 0), 42.0, 1.0),
                 ((3.0, 2.0, 9.0), (0.1, -0.3, 0.2), (0, 1, 0), 35.0, 16 / 9)]:
        cam = sb.Camera.look_at(*args)
        got = sb.camera_proj_params(cam)
        ref = np.empty(16, np.float32)
        oc = oracle.camera_look_at(*args)
        oracle.lib.or_camera_proj_params(C.byref(oc), oracle.fp(ref))
        assert got.tobytes() == ref.tobytes()
        assert abs(np.linalg.norm(got[1, :3]) - 1.0) < 1e-6 and got[0, 3] == 0.0 and got[1, 3] > 0.0


def test_sensor_tables_equal_oracle():
    assert sb.sample_tables().tobytes() == oracle.tables().tobytes()


def test_dsotm_scene_matches_reference_constants():
    scene, beam, cam = sb.dsotm_scene(1.0)
    assert len(scene.prims) == 1 and len(scene.planes) == 5 and scene.mats[0].glass == sb.SF11
    assert tuple(scene.planes[0].normal) == tuple(np.float32([-0.8660254, 0.5, 0.0]))
    d = np.array(beam.c.dir, np.float32)
    assert abs(np.linalg.norm(d) - 1.0) < 1e-6
    assert bytes(cam.c) == bytes(oracle.camera_look_at((0.5, -0.5, 12.0), (0.5, -0.5, 0.0), (0, 1, 0), 42.0, 1.0))


def test_tir_beam_dir_is_normalized_f32():
    b = sb.tir_beam()
    d = np.array(b.c.dir, np.float32)
    assert abs(float(np.sqrt(np.dot(d, d))) - 1.0) < 1e-6


def test_film_sizes():
    assert _lib.lib.sc_film_bytes(640, 360, 64) == 80 * 45 * 64 * 64 * 8
    assert _lib.lib.sc_film_flag_bytes(641, 361) == (81 * 46 + 31) // 32 * 4


def test_null_arguments_fail_with_status():
    assert _lib.lib.sc_photon_film_trace_and_resolve(None, 10, 1) == _lib.SC_E_INVALID
    assert b"null" in _lib.lib.sc_last_error()
    assert _lib.lib.sc_ctx_create(0, None, None) == _lib.SC_E_INVALID
    assert _lib.lib.sc_load_sensor_tables(b"/nonexistent.csv", (C.c_float * 355)()) == _lib.SC_E_INVALID
    # entry points added beside the reference API refuse null handles the same way
    f16 = (C.c_float * 16)()
    assert _lib.lib.sc_camera_proj_params(None, f16) == _lib.SC_E_INVALID
    assert _lib.lib.sc_glass_n_device(None, 0, None, 4, None, None) == _lib.SC_E_INVALID
    assert _lib.lib.sc_tracer_set_rows(None, 0, 1) == _lib.SC_E_INVALID
    assert _lib.lib.sc_tracer_set_spectral(None, 0) == _lib.SC_E_INVALID
    e = C.c_float()
    assert _lib.lib.sc_atomic_film_auto_expose_accum(None, 1.0, C.byref(e)) == _lib.SC_E_INVALID
    assert _lib.lib.sc_atomic_film_to_rgb8(None, 1.0, None) == _lib.SC_E_INVALID
    n = C.c_float(500.0)
    assert _lib.lib.sc_glass_n_many(0, None, 1, None) == _lib.SC_E_INVALID
    assert _lib.lib.sc_glass_n_many(0, C.byref(n), 0, None) == _lib.SC_OK  # nothing to do


def test_context_new_is_none_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert sb.GpuContext.new() is None  # GpuContext::new() -> None, as the reference's Option
    # an argument error is not "no GPU": it raises
    with pytest.raises(_lib.SpectralError) as e:
        sb.GpuContext.new(-1)
    assert e.value.code == _lib.SC_E_INVALID


def test_no_gpu_means_error_not_fallback():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(_lib.SpectralError) as e:
        sb.GpuContext(0)
    assert e.value.code == _lib.SC_E_NODEVICE
