"""Device-pointer entry points (sc_trace_photons_device, sc_trace_stats_device,
sc_sensor_reduce_device) on caller-owned device memory: the same images as
the photon-film object for the point and beam estimators, work counters, and
the drain leaving film and dirty mask zeroed for the next pass."""
import ctypes as C

import numpy as np
import pytest

import spectral_b200 as sb
from spectral_b200 import _lib

pytestmark = pytest.mark.gpu


def _desc(scene, cam, beam, w, h, seed, bins, estimator, scale_log2, keep, torch):
    prims, np_, planes, npl, mats, nm = scene.arrays()

    def dev(arr, n, size):
        t = torch.frombuffer(bytearray(bytes(arr)[: n * size] or b"\0"), dtype=torch.uint8).cuda()
        keep.append(t)
        return t.data_ptr()

    opts = _lib.sc_film_options(bins, 380.0, 730.0, 8, scale_log2, estimator)
    w8 = sb.VolWeights()
    return _lib.sc_trace_desc(dev(prims, np_, 32), np_, dev(planes, npl, 16), npl, dev(mats, nm, 16), nm, cam.c,
                              beam.c, _lib.sc_vol_weights(w8.sigma_s, w8.sigma_t, w8.g), w, h, seed, 1, 14.0, opts,
                              None)


def _device_pass(ctx, desc, n, torch, drain=1):
    w, h = desc.width, desc.height
    ch = desc.opts.bins or 3
    film = torch.zeros(_lib.lib.sc_film_bytes(w, h, ch) // 8, dtype=torch.int64, device="cuda")
    flags = torch.zeros(_lib.lib.sc_film_flag_bytes(w, h) // 4, dtype=torch.int32, device="cuda")
    xyz = torch.empty(3 * w * h, dtype=torch.float32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(_lib.lib.sc_trace_photons_device(ctx.h, C.byref(desc), 0, n, C.c_void_p(film.data_ptr()),
                                                C.c_void_p(flags.data_ptr()), stream))
    dirty = int(np.unpackbits(flags.cpu().numpy().view(np.uint8)).sum())
    _lib.check(_lib.lib.sc_sensor_reduce_device(ctx.h, w, h, ch, desc.opts.lambda_min, desc.opts.lambda_max,
                                                desc.opts.scale_log2, C.c_void_p(film.data_ptr()),
                                                C.c_void_p(flags.data_ptr()), C.c_void_p(xyz.data_ptr()), drain,
                                                stream))
    torch.cuda.synchronize()
    return xyz.cpu().numpy(), film, flags, dirty


@pytest.mark.parametrize("estimator,bins,scale_log2", [(0, 0, 32), (0, 16, 32), (2, 0, 40), (2, 8, 40)])
def test_device_path_equals_film_object(ctx, estimator, bins, scale_log2):
    import torch
    keep = []
    scene, beam, cam = sb.dsotm_scene(96 / 72)
    n, seed = 3000, 17
    desc = _desc(scene, cam, beam, 96, 72, seed, bins, estimator, scale_log2, keep, torch)
    got, film, flags, dirty = _device_pass(ctx, desc, n, torch)
    f = sb.GpuPhotonFilm(ctx, scene, cam, beam, 96, 72, n, seed, 14.0, sb.VolWeights(), bins=bins,
                         scale_log2=scale_log2, estimator=estimator)
    f.trace_and_resolve(n, seed)
    ref = f.accum()
    assert ref.sum() > 0 and dirty > 0
    assert got.tobytes() == ref.tobytes()  # same kernels, same integers, same reduction
    # the drain left the film and its dirty mask ready for the next pass
    assert not film.any().item() and not flags.any().item()


def test_stats_counters(ctx):
    import torch
    keep = []
    scene, beam, cam = sb.dsotm_scene(1.0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for estimator, ncnt in ((0, 4), (2, 5)):
        desc = _desc(scene, cam, beam, 64, 64, 3, 0, estimator, 32 if estimator == 0 else 40, keep, torch)
        out = torch.zeros(5, dtype=torch.int64, device="cuda")
        _lib.check(_lib.lib.sc_trace_stats_device(ctx.h, C.byref(desc), 0, 1000, C.c_void_p(out.data_ptr()), stream))
        torch.cuda.synchronize()
        c = [int(x) for x in out.cpu()]
        assert c[0] == 1000 and c[1] >= 1000  # photons, segments (at least one each)
        assert all(v > 0 for v in c[2:ncnt]) and all(v == 0 for v in c[ncnt:])
        if estimator == 2:  # steps >= in-frame steps; footprints of several pixels each
            assert c[2] >= c[3] and c[4] > c[3]
