"""The allocation-free entry point (sc_trace_xyz_noalloc).

It exists for callers that cannot allocate device memory themselves, e.g. a
host whose framework owns every byte of device memory through its own pool,
or a render loop that must never stall on cudaMalloc / cudaFree.  Its scratch
film lives in a static device array shared by all calls, so this test makes
three calls in a row (different scenes, film kinds, sizes and estimators) and
checks each against the existing device-pointer path (sc_trace_photons_device
+ sc_sensor_reduce_device).  Both paths run the same kernels on the same
photons and the film sums are exact integers, so the images must be equal bit
for bit: any splat left over from an earlier call in the shared scratch would
show.  The second call's film (64 bins) spans every scratch cell the first
call (an XYZ film) lit, at pixels and bins of its own that its photons never
reach.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import spectral_b200 as sb
from spectral_b200 import _lib
from spectral_b200.scenes import prism_workload

pytestmark = pytest.mark.gpu

def _desc(scene, cam, beam, w, h, seed, bins, weights, torch, keep, estimator=0):
    prims, np_, planes, npl, mats, nm = scene.arrays()

    def dev(arr, n, size):
        t = torch.frombuffer(bytearray(bytes(arr)[: n * size] or b"\0"), dtype=torch.uint8).cuda()
        keep.append(t)
        return t.data_ptr()

    opts = _lib.sc_film_options(bins, 380.0, 780.0 if bins else 730.0, 8, 32, estimator)
    return _lib.sc_trace_desc(dev(prims, np_, 32), np_, dev(planes, npl, 16), npl, dev(mats, nm, 16), nm, cam.c,
                              beam.c, _lib.sc_vol_weights(*weights), w, h, seed, 1, 14.0, opts, None)


def _existing(ctx, desc, n, stream, torch):
    w, h = desc.width, desc.height
    ch = desc.opts.bins or 3
    film = torch.zeros(_lib.lib.sc_film_bytes(w, h, ch) // 8, dtype=torch.int64, device="cuda")
    flags = torch.zeros(_lib.lib.sc_film_flag_bytes(w, h) // 4, dtype=torch.int32, device="cuda")
    xyz = torch.empty(3 * w * h, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib.sc_trace_photons_device(ctx.h, C.byref(desc), 0, n, C.c_void_p(film.data_ptr()),
                                                C.c_void_p(flags.data_ptr()), stream))
    _lib.check(_lib.lib.sc_sensor_reduce_device(ctx.h, w, h, ch, desc.opts.lambda_min, desc.opts.lambda_max, 32,
                                                C.c_void_p(film.data_ptr()), C.c_void_p(flags.data_ptr()),
                                                C.c_void_p(xyz.data_ptr()), 0, stream))
    torch.cuda.synchronize()
    return xyz.cpu().numpy()


def _noalloc(tables, desc, n, stream, torch):
    xyz = torch.full((3 * desc.width * desc.height,), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib.sc_trace_xyz_noalloc(tables.ctypes.data_as(C.POINTER(C.c_float)), C.byref(desc), 0, n,
                                             C.c_void_p(xyz.data_ptr()), stream))
    torch.cuda.synchronize()
    return xyz.cpu().numpy()


def test_noalloc_matches_existing_entry_point_on_calls_in_a_row(ctx):
    import torch
    keep = []
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    tables = sb.sample_tables()
    dsotm, beam, cam = sb.dsotm_scene(1.0)
    prism, pbeam, pcam = prism_workload(640, 360)
    calls = [
        # an XYZ film of 691,200 cells, then a 64-bin film of 1,048,576 cells laid
        # over the same scratch, then a free-flight film: none may see another's splats
        (_desc(prism, pcam, pbeam, 640, 360, 11, 0, (0.05, 0.05, 0.0), torch, keep), 400_000),
        (_desc(dsotm, cam, beam, 128, 128, 7, 64, (0.5, 0.06, 0.5), torch, keep), 200_000),
        (_desc(dsotm, cam, beam, 200, 160, 5, 0, (0.5, 0.3, 0.5), torch, keep, estimator=3), 100_000),
    ]
    for desc, n in calls:
        ref = _existing(ctx, desc, n, stream, torch)
        got = _noalloc(tables, desc, n, stream, torch)
        assert np.isfinite(got).all() and ref.sum() > 0
        assert got.tobytes() == ref.tobytes(), int((got != ref).sum())


def test_noalloc_rejects_films_beyond_its_scratch(ctx):
    import torch
    keep = []
    scene, beam, cam = sb.dsotm_scene(1.0)
    desc = _desc(scene, cam, beam, 1024, 1024, 1, 64, (0.5, 0.06, 0.5), torch, keep)
    out = torch.empty(3, dtype=torch.float32, device="cuda")
    rc = _lib.lib.sc_trace_xyz_noalloc(sb.sample_tables().ctypes.data_as(C.POINTER(C.c_float)), C.byref(desc), 0,
                                       10, C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.SC_E_LIMIT and b"allocation-free path holds at most" in _lib.lib.sc_last_error()
    beam_est = _desc(scene, cam, beam, 64, 64, 1, 0, (0.5, 0.06, 0.5), torch, keep, estimator=2)
    rc = _lib.lib.sc_trace_xyz_noalloc(sb.sample_tables().ctypes.data_as(C.POINTER(C.c_float)),
                                       C.byref(beam_est), 0, 10, C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.SC_E_INVALID and b"estimator 2" in _lib.lib.sc_last_error()
