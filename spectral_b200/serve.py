"""Serving loop: continuous batching of render requests (sc_server_* ABI).

``Server`` wraps the C object; ``poisson_requests`` draws a seeded request
stream (Poisson arrivals; prism scenes; photons per frame log-uniform; a share
of progressive orbit sessions); ``run_stream`` replays a stream in real time
and returns latency percentiles and throughput.
"""
import ctypes as C
import math
import time

import numpy as np

from . import _lib
from ._lib import check, lib
from . import specs
from .batch import job_from_spec

ORBIT_TARGET = (0.6, -0.4, 0.0)


class Server:
    def __init__(self, ctx, budget_bytes=40 << 30, max_slots=256, chunk_photons=2048, warp_split=0):
        self.h = C.c_void_p()
        cfg = _lib.sc_server_config(int(budget_bytes), int(max_slots), int(chunk_photons), int(warp_split))
        check(lib.sc_server_create(ctx.h, C.byref(cfg), C.byref(self.h)))
        self._dims = {}
        self._buf = None

    def submit(self, job, frames=1, orbit_deg=0.0, target=ORBIT_TARGET, up=(0.0, 1.0, 0.0), vfov=42.0):
        """Queue a render of `frames` frames of job.n_photons photons each:
        with orbit_deg == 0 the frames accumulate (a progressive session), else
        the camera orbits by orbit_deg per frame and the last frame is kept."""
        r = _lib.sc_request()
        r.job, r.frames, r.orbit_deg = job, int(frames), float(orbit_deg)
        r.orbit_target, r.orbit_up, r.vfov_deg = _lib.F3(*target), _lib.F3(*up), float(vfov)
        rid = C.c_uint64()
        check(lib.sc_server_submit(self.h, C.byref(r), C.byref(rid)))
        self._dims[rid.value] = 3 * job.width * job.height
        return rid.value

    def step(self):
        a = C.c_uint32()
        check(lib.sc_server_step(self.h, C.byref(a)))
        return a.value

    def poll(self, want_image=True, copy=True):
        """(id, xyz or None, (t_submit, t_admit, t_first_frame, t_done)) or None.
        With copy=False the image is a view of a buffer that the next poll
        overwrites (the library has already copied it into host memory)."""
        rid, w, h = C.c_uint64(), C.c_uint32(), C.c_uint32()
        times = (C.c_double * 4)()
        # room for the largest image of any request still outstanding (buffer kept between polls)
        cap = max(self._dims.values()) if (want_image and self._dims) else 0
        if cap and (self._buf is None or self._buf.size < cap):
            self._buf = np.empty(cap, np.float32)
        buf = self._buf
        rc = lib.sc_server_poll(self.h, C.byref(rid), buf.ctypes.data_as(C.POINTER(C.c_float)) if cap else None,
                                cap, C.byref(w), C.byref(h), times)
        if rc == _lib.SC_E_STATE:
            return None
        check(rc)
        n = self._dims.pop(rid.value, 0)
        img = (buf[:n].copy() if copy else buf[:n]) if cap else None
        return rid.value, img, tuple(times)

    def peek(self, rid):
        """(frames done, current XYZ image) of an active request, or None when
        it has no frame on the device: a progressive session's accumulated
        image so far, an orbit session's latest frame."""
        n = self._dims.get(rid)
        if n is None:
            return None
        out = np.empty(n, np.float32)
        fr = C.c_uint32()
        rc = lib.sc_server_peek(self.h, int(rid), out.ctypes.data_as(C.POINTER(C.c_float)), n, C.byref(fr))
        if rc == _lib.SC_E_STATE:
            return None
        check(rc)
        return fr.value, out

    def cancel(self, rid):
        check(lib.sc_server_cancel(self.h, int(rid)))
        self._dims.pop(rid, None)

    def stats(self):
        p, b = C.c_uint64(), C.c_uint64()
        q, a, f = C.c_uint32(), C.c_uint32(), C.c_uint32()
        check(lib.sc_server_stats(self.h, C.byref(p), C.byref(b), C.byref(q), C.byref(a), C.byref(f)))
        return dict(photons=p.value, bytes_in_use=b.value, queued=q.value, active=a.value, finished=f.value)

    def close(self):
        if self.h:
            lib.sc_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def poisson_requests(rate=200.0, seconds=60.0, seed=0x5E7E, **kw):
    """Seeded request stream: list of (arrival_s, job, frames, orbit_deg), the
    request dicts of specs.poisson_request_specs as sc_scene_job records."""
    return [(t, job_from_spec(spec), nf, orbit) for t, spec, nf, orbit in
            specs.poisson_request_specs(rate, seconds, seed, **kw)]


def orbit_camera(job, frame, deg, target=ORBIT_TARGET, up=(0.0, 1.0, 0.0), vfov=42.0):
    """Camera of frame `frame` of an orbit session, as the server builds it: the
    job camera's origin rotated about the vertical axis through `target` by
    deg * frame (f32 offsets, rotation in double, rounded to f32), then
    Camera::look_at."""
    from . import Camera
    if deg == 0.0 or frame == 0:
        return job.cam
    a = deg * frame * math.pi / 180.0
    ox, oy, oz = job.cam.origin
    tx, _, tz = target
    dx, dz = float(np.float32(ox) - np.float32(tx)), float(np.float32(oz) - np.float32(tz))
    o = (float(np.float32(float(np.float32(tx)) + dx * math.cos(a) + dz * math.sin(a))), float(oy),
         float(np.float32(float(np.float32(tz)) - dx * math.sin(a) + dz * math.cos(a))))
    return Camera.look_at(o, target, up, vfov, float(np.float32(job.width) / np.float32(job.height))).c


def run_plain_stream(ctx, stream, time_scale=1.0):
    """The same stream served the plain way, one request at a time in arrival
    order, each through its own GpuPhotonFilm-shaped object: create the film,
    per frame set the camera, trace the frame's photon range, read the XYZ image
    back to the host and clear; destroy.  Returns the metrics of run_stream."""
    t0 = time.perf_counter()
    lat, ttff, photons = [], [], 0
    # one host image buffer, as large as the largest image (reused, as the server's is)
    host_all = np.empty(max(3 * r[1].width * r[1].height for r in stream) if stream else 0, np.float32)
    for arrival, job, nf, orbit in stream:
        now = time.perf_counter() - t0
        if now < arrival * time_scale:
            time.sleep(arrival * time_scale - now)
        f = C.c_void_p()
        host = host_all[:3 * job.width * job.height]
        check(lib.sc_photon_film_create(ctx.h, job.prims, job.n_prims, job.planes, job.n_planes, job.mats,
                                        job.n_mats, 0.0, C.byref(job.cam), C.byref(job.beam), job.width, job.height,
                                        job.n_photons, job.seed, job.max_dist, C.byref(job.weights), None,
                                        C.byref(job.opts), C.byref(f)))
        try:
            check(lib.sc_photon_film_set_spectral(f, int(job.spectral)))
            n = job.n_photons
            for fr in range(nf):
                if orbit:
                    cam = orbit_camera(job, fr, orbit)
                    check(lib.sc_photon_film_set_camera(f, C.byref(cam)))
                check(lib.sc_photon_film_dispatch(f, fr * n, (fr + 1) * n, job.seed))
                check(lib.sc_photon_film_read_accum(f, host.ctypes.data_as(C.POINTER(C.c_float))))
                check(lib.sc_photon_film_clear(f))
                if fr == 0:
                    ttff.append(time.perf_counter() - t0 - arrival * time_scale)
                photons += n
        finally:
            lib.sc_photon_film_destroy(f)
        lat.append(time.perf_counter() - t0 - arrival * time_scale)
    wall = time.perf_counter() - t0
    lat, ttff = np.array(lat), np.array(ttff)
    return dict(requests=len(stream), wall_s=wall, steps=len(stream), photons=photons, photons_per_s=photons / wall,
                p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3),
                p50_first_frame_ms=float(np.percentile(ttff, 50) * 1e3),
                p99_first_frame_ms=float(np.percentile(ttff, 99) * 1e3))


def run_stream(server, stream, time_scale=1.0, idle_sleep=2e-4, want_image=False):
    """Replay `stream` in real time against `server`; returns a metrics dict.
    Latencies come from the server's own timestamps (submit to last frame
    done), or with `want_image` from the host clock (arrival to the XYZ image
    in host memory)."""
    t0 = time.perf_counter()
    k, done, lat, ttff = 0, 0, [], []
    pending = {}
    steps, photons0 = 0, server.stats()["photons"]
    while done < len(stream):
        now = time.perf_counter() - t0
        while k < len(stream) and stream[k][0] * time_scale <= now:
            arrival, job, nf, orbit = stream[k]
            rid = server.submit(job, nf, orbit)
            pending[rid] = arrival * time_scale
            k += 1
        st = server.stats()
        if st["queued"] or st["active"]:
            server.step()
            steps += 1
        elif k < len(stream):
            time.sleep(min(idle_sleep, max(0.0, stream[k][0] * time_scale - now)))
        while True:
            r = server.poll(want_image=want_image, copy=False)
            if r is None:
                break
            rid, _, (ts, ta, tf, td) = r
            arrived = pending.pop(rid, None)
            lat.append(time.perf_counter() - t0 - arrived if want_image else td - ts)
            ttff.append(tf - ts)
            done += 1
    wall = time.perf_counter() - t0
    photons = server.stats()["photons"] - photons0
    lat, ttff = np.array(lat), np.array(ttff)
    return dict(requests=len(stream), wall_s=wall, steps=steps, photons=photons, photons_per_s=photons / wall,
                p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3),
                p50_first_frame_ms=float(np.percentile(ttff, 50) * 1e3),
                p99_first_frame_ms=float(np.percentile(ttff, 99) * 1e3))


def main():
    """Replay the seeded request stream (Poisson arrivals) with continuous
    batching and with one request at a time; print one JSON line."""
    import argparse
    import json
    from . import GpuContext
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--seconds", type=float, default=60.0)
    ap.add_argument("--budget-gb", type=float, default=40.0)
    ap.add_argument("--seed", type=int, default=0x5E7E)
    ap.add_argument("--skip-serial", action="store_true")
    a = ap.parse_args()
    ctx = GpuContext(0)
    stream = poisson_requests(a.rate, a.seconds, a.seed)
    out = {"requests": len(stream), "rate_per_s": a.rate, "seconds": a.seconds, "budget_gb": a.budget_gb,
           "sessions": sum(1 for s in stream if s[2] > 1), "frames": sum(s[2] for s in stream)}
    srv = Server(ctx, budget_bytes=int(a.budget_gb * (1 << 30)))
    out["continuous_batching"] = run_stream(srv, stream)
    srv.close()
    if not a.skip_serial:
        srv = Server(ctx, budget_bytes=int(a.budget_gb * (1 << 30)), max_slots=1)
        out["one_request_at_a_time"] = run_stream(srv, stream)
        srv.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
