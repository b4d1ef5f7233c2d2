"""Batched uneven workload: many scenes in one persistent, graph-captured launch.

``Batch(ctx, jobs)`` wraps ``sc_batch_*`` (include/spectral_cuda.h); ``jobs`` are
``sc_scene_job`` records, e.g. from ``prism_jobs`` below.
"""
import ctypes as C

import numpy as np

from . import _lib, Camera
from ._lib import check, lib
from .scenes import prism_beam, prism_planes
from .specs import PRISM_CAMERA


def prism_job(glass, apex_deg, incidence_deg, n_photons, width, height, sigma_s, sigma_t, g, seed, bins,
              lambda_min, lambda_max, beam_width=0.02, max_dist=6.0, max_bounces=8, spectral=1):
    """One sc_scene_job: an isosceles prism (side 1) in haze, a square beam on
    its left face, a camera framing prism and fan, a spectral film."""
    j = _lib.sc_scene_job()
    planes = prism_planes(apex_deg, 1.0, 1.0)
    j.n_prims, j.n_planes, j.n_mats, j.spectral = 1, len(planes), 1, int(spectral)
    for k, (nrm, d) in enumerate(planes):
        j.planes[k].normal = _lib.F3(*nrm)
        j.planes[k].d = d
    j.prims[0].plane_start, j.prims[0].plane_count, j.prims[0].kind, j.prims[0].material = 0, len(planes), 1, 0
    j.mats[0].kind, j.mats[0].glass = 1, int(glass)
    o, t, up, vfov = PRISM_CAMERA
    j.cam = Camera.look_at(o, t, up, vfov, width / height).c
    j.beam = prism_beam(apex_deg, 1.0, incidence_deg, beam_width).c
    j.weights = _lib.sc_vol_weights(sigma_s, sigma_t, g)
    j.width, j.height, j.n_photons, j.seed, j.max_dist = int(width), int(height), int(n_photons), int(seed), max_dist
    j.opts = _lib.sc_film_options(int(bins), float(lambda_min), float(lambda_max), int(max_bounces), 32, 0)
    return j


def job_from_spec(s):
    """sc_scene_job of one prism job dict (spectral_b200.specs)."""
    return prism_job(s["glass"], s["apex_deg"], s["incidence_deg"], s["n_photons"], s["width"], s["height"],
                     s["sigma_s"], s["sigma_t"], s["g"], s["seed"], s["bins"], s["lambda_min"], s["lambda_max"])


def prism_jobs(specs):
    """sc_scene_job array from dicts of spectral_b200.specs.random_prism_jobs."""
    arr = (_lib.sc_scene_job * len(specs))()
    for i, s in enumerate(specs):
        arr[i] = job_from_spec(s)
    return arr


class Batch:
    def __init__(self, ctx, jobs, chunk_photons=0, minb=0, aggregate=0, per_photon=0, block=0):
        self.jobs = jobs
        self.h = C.c_void_p()
        t = _lib.sc_batch_tuning(chunk_photons, minb, aggregate, 0, per_photon, block)
        check(lib.sc_batch_create(ctx.h, jobs, len(jobs), C.byref(t), C.byref(self.h)))
        tp, fb, xf, jb = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(lib.sc_batch_info(self.h, C.byref(tp), C.byref(fb), C.byref(xf), C.byref(jb)))
        self.total_photons, self.film_bytes, self.xyz_floats = tp.value, fb.value, xf.value
        self.job_table_bytes = jb.value

    def autotune(self):
        t = _lib.sc_batch_tuning()
        check(lib.sc_batch_autotune(self.h, C.byref(t)))
        return dict(chunk_photons=t.chunk_photons, minb=t.minb, aggregate=t.aggregate, grid=t.grid,
                    per_photon=t.per_photon, block=t.block)

    def tuning(self):
        t = _lib.sc_batch_tuning()
        check(lib.sc_batch_get_tuning(self.h, C.byref(t)))
        return dict(chunk_photons=t.chunk_photons, minb=t.minb, aggregate=t.aggregate, grid=t.grid,
                    per_photon=t.per_photon, block=t.block)

    def set_tuning(self, chunk_photons=0, minb=0, aggregate=0, grid=0, per_photon=0, block=0):
        t = _lib.sc_batch_tuning(chunk_photons, minb, aggregate, grid, per_photon, block)
        check(lib.sc_batch_set_tuning(self.h, C.byref(t)))

    def update_jobs(self, jobs):
        self.jobs = jobs
        check(lib.sc_batch_update_jobs(self.h, jobs, len(jobs)))

    def run(self, stream=None):
        check(lib.sc_batch_run(self.h, C.c_void_p(stream) if stream else None))

    def run_plain(self, stream=None):
        check(lib.sc_batch_run_plain(self.h, C.c_void_p(stream) if stream else None))

    def synchronize(self):
        check(lib.sc_batch_synchronize(self.h))

    def read_xyz(self, job):
        j = self.jobs[job]
        out = np.empty(3 * j.width * j.height, np.float32)
        check(lib.sc_batch_read_xyz(self.h, int(job), out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def read_all_xyz(self, out=None, stream=None):
        if out is None:
            out = np.empty(self.xyz_floats, np.float32)
        check(lib.sc_batch_read_all_xyz(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size,
                                        C.c_void_p(stream) if stream else None))
        return out

    def read_all_xyz_async(self, out, stream=None):
        """Start copying every image into `out` (pinned, kept alive by the
        caller) without waiting; the next pass overlaps the copy."""
        check(lib.sc_batch_read_all_xyz_async(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size,
                                              C.c_void_p(stream) if stream else None))
        return out

    def stats(self):
        out = (C.c_uint64 * 6)()
        check(lib.sc_batch_stats(self.h, out))
        keys = ("photons", "segments", "in_frame_samples", "scatters", "dirty_tiles", "dirty_tile_bytes")
        return dict(zip(keys, [int(x) for x in out]))

    def close(self):
        if self.h:
            lib.sc_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
