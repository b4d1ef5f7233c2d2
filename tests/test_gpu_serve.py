"""Serving loop (continuous batching): a request's image is the same alone and
in any mix of concurrent requests (bit-identical: its photons are keyed by its
own index), single renders, orbit frames and progressive sessions match the
CPU oracle, admission respects the device-memory budget, and a real-time
Poisson stream completes."""
import math

import numpy as np
import pytest

import oracle
import spectral_b200 as sb
from spectral_b200 import _lib
from spectral_b200.batch import prism_job
from spectral_b200.serve import ORBIT_TARGET, Server, orbit_camera, poisson_requests, run_plain_stream, run_stream

from helpers import rel_l1

pytestmark = pytest.mark.gpu

FAST_TOL = 2e-3  # relative L1 against the oracle: batched films run the fast haze samples


def job(i, n=20_000, side=48, bins=16):
    return prism_job((0, 1, 3)[i % 3], 40.0 + 7 * i, 35.0 + 3 * i, n + 1000 * i, side + 8 * (i % 3),
                     side + 8 * (i % 3), 0.03 + 0.01 * i, 0.03 + 0.01 * i, 0.0, 1000 + i, bins, 380.0, 780.0)


def drain(server):
    out = {}
    for _ in range(10_000):
        st = server.stats()
        if not (st["queued"] or st["active"]):
            break
        server.step()
    while True:
        r = server.poll()
        if r is None:
            return out
        out[r[0]] = r[1]


def oracle_image(j, photon_begin, photon_end, cam=None):
    sc = oracle.OScene(bytes(j.prims)[:32 * j.n_prims], j.n_prims, bytes(j.planes)[:16 * j.n_planes], j.n_planes,
                       bytes(j.mats)[:16 * j.n_mats], j.n_mats, 0.0)
    oc = oracle.or_camera.from_buffer_copy(bytes(cam if cam is not None else j.cam))
    ob = oracle.or_beam.from_buffer_copy(bytes(j.beam))
    o = j.opts
    p = oracle.vol_params(j.width, j.height, j.seed, j.weights.sigma_s, j.weights.sigma_t, j.weights.g, j.max_dist,
                          o.max_bounces, o.lambda_min, o.lambda_max, bins=o.bins)
    _, _, fs = oracle.render_point(sc, oc, ob, p, photon_begin, photon_end, f32=False, xyz=False, spec=True)
    w = oracle.bin_weights(o.bins, o.lambda_min, o.lambda_max).astype(np.float64)
    return (fs.reshape(-1, o.bins).astype(np.float64) @ w.T).reshape(-1) * 2.0 ** -32


def test_same_alone_and_in_the_mix(ctx):
    jobs = [job(i) for i in range(6)]
    alone = {}
    for i, j in enumerate(jobs):
        s = Server(ctx, budget_bytes=1 << 30)
        rid = s.submit(j, frames=3 if i % 2 else 1, orbit_deg=2.0 if i % 2 else 0.0)
        alone[i] = drain(s)[rid]
        s.close()
    s = Server(ctx, budget_bytes=1 << 30)
    ids = {}
    for i, j in enumerate(jobs):
        ids[s.submit(j, frames=3 if i % 2 else 1, orbit_deg=2.0 if i % 2 else 0.0)] = i
        if i == 2:
            s.step()  # later arrivals join while earlier ones are on the device
    mixed = drain(s)
    assert len(mixed) == len(jobs)
    for rid, img in mixed.items():
        assert img.tobytes() == alone[ids[rid]].tobytes(), ids[rid]
    # single renders match the CPU oracle; orbit sessions return their last frame
    for i, j in enumerate(jobs):
        if i % 2 == 0:
            exp = oracle_image(j, 0, j.n_photons)
        else:
            exp = oracle_image(j, 2 * j.n_photons, 3 * j.n_photons, orbit_camera(j, 2, 2.0))
        assert exp.sum() > 0 and rel_l1(alone[i], exp) < FAST_TOL, i


def test_budget_admission_and_cancel(ctx):
    small = job(0, side=64, bins=32)
    per = 64 // 8 * (64 // 8) * 64 * 32 * 8  # film bytes of one request
    s = Server(ctx, budget_bytes=int(per * 2.5), max_slots=8)
    big = job(1, side=512, bins=64)
    with pytest.raises(_lib.SpectralError) as e:
        s.submit(big)
    assert e.value.code == _lib.SC_E_NOMEM
    ids = [s.submit(small, frames=2) for _ in range(4)]
    s.step()
    st = s.stats()
    assert st["active"] == 2 and st["queued"] == 2 and st["bytes_in_use"] <= int(per * 2.5)
    s.cancel(ids[3])
    s.cancel(ids[0])
    got = drain(s)
    assert sorted(got) == sorted(ids[1:3]) and s.stats()["bytes_in_use"] == 0
    with pytest.raises(_lib.SpectralError):
        s.cancel(12345)


def test_queued_steps_overflowing_image_ring_and_cancel(ctx):
    """Steps queue ahead of the host (two deep while requests wait): 24 requests
    of 1024x1024 images (303 MB) finish before any poll, past the 256 MB pinned
    ring, and each still equals its render alone; cancelling a session whose
    frames are queued leaves the other request's result and frees the budget."""
    big = [job(i, n=4096, side=1024, bins=1) for i in range(24)]
    s = Server(ctx, budget_bytes=2 << 30, max_slots=8)
    ids = [s.submit(j) for j in big]
    while s.stats()["queued"] or s.stats()["active"]:
        s.step()
    got = {}
    while (r := s.poll()) is not None:
        got[r[0]] = r[1]
    assert sorted(got) == sorted(ids) and s.stats()["bytes_in_use"] == 0
    s.close()
    # a slow poller (one result per step): finished images wait on the device
    # for ring room instead of taking pinned buffers of their own
    s = Server(ctx, budget_bytes=2 << 30, max_slots=8)
    ids2 = [s.submit(j) for j in big]
    got2 = {}
    while s.stats()["queued"] or s.stats()["active"]:
        s.step()
        if (r := s.poll()) is not None:
            got2[r[0]] = r[1]
    while (r := s.poll()) is not None:
        got2[r[0]] = r[1]
    assert sorted(got2) == sorted(ids2) and s.stats()["bytes_in_use"] == 0
    s.close()
    for a, b in zip(ids, ids2):
        assert got2[b].tobytes() == got[a].tobytes()
    for i in (0, 11, 23):
        a = Server(ctx, budget_bytes=1 << 30)
        rid = a.submit(big[i])
        alone = drain(a)[rid]
        a.close()
        assert alone.sum() > 0 and got[ids[i]].tobytes() == alone.tobytes(), i
    s = Server(ctx, budget_bytes=1 << 30)
    session = s.submit(job(0), frames=6, orbit_deg=2.0)
    single = s.submit(job(1))
    s.step()
    s.step()  # the session's frames are queued on the device
    s.cancel(session)
    res = drain(s)
    assert list(res) == [single] and s.stats()["bytes_in_use"] == 0
    a = Server(ctx, budget_bytes=1 << 30)
    rid = a.submit(job(1))
    assert drain(a)[rid].tobytes() == res[single].tobytes()
    a.close()
    s.close()


def test_realtime_stream_completes(ctx):
    stream = poisson_requests(rate=60.0, seconds=1.0, seed=7, frames=(2, 6), photons=(2 ** 12, 2 ** 15),
                              side=(32, 128), bins=16)
    s = Server(ctx, budget_bytes=2 << 30)
    m = run_stream(s, stream)
    assert m["requests"] == len(stream) > 10
    assert 0 < m["p50_ms"] <= m["p99_ms"] and m["photons"] > 0
    assert s.stats()["bytes_in_use"] == 0
    # the plain per-request path renders the same frames (same photon total)
    plain = run_plain_stream(ctx, stream)
    assert plain["requests"] == len(stream) and plain["photons"] == m["photons"]
    assert 0 < plain["p50_ms"] <= plain["p99_ms"]


def plain_image(ctx, j, begin, end):
    """XYZ image of photons [begin, end) of a job through the plain film object."""
    import ctypes as C
    f = C.c_void_p()
    _lib.check(_lib.lib.sc_photon_film_create(ctx.h, j.prims, j.n_prims, j.planes, j.n_planes, j.mats, j.n_mats,
                                              0.0, C.byref(j.cam), C.byref(j.beam), j.width, j.height, j.n_photons,
                                              j.seed, j.max_dist, C.byref(j.weights), None, C.byref(j.opts),
                                              C.byref(f)))
    try:
        _lib.check(_lib.lib.sc_photon_film_set_spectral(f, int(j.spectral)))
        _lib.check(_lib.lib.sc_photon_film_dispatch(f, begin, end, j.seed))
        out = np.empty(3 * j.width * j.height, np.float32)
        _lib.check(_lib.lib.sc_photon_film_read_accum(f, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out
    finally:
        _lib.lib.sc_photon_film_destroy(f)


def test_progressive_session_accumulates(ctx):
    """A session of 4 frames on a fixed camera adds photons [0, 4N) into one
    film on the device: its image is the film of those photons times 1/4 (the
    same bits as the plain film object's image of [0, 4N), scaled by 2^-2),
    within FAST_TOL of the oracle, and the same alone and in a mix.  Midway,
    peek shows the image of the frames done so far."""
    j = job(2, n=15_000)
    n = j.n_photons
    s = Server(ctx, budget_bytes=1 << 30)
    rid = s.submit(j, frames=4)
    s.step()
    s.step()
    fr, mid = s.peek(rid)
    assert fr == 2
    assert mid.tobytes() == (plain_image(ctx, j, 0, 2 * n) * np.float32(0.5)).tobytes()
    alone = drain(s)[rid]
    out = np.empty(3 * j.width * j.height, np.float32)
    import ctypes as C
    assert _lib.lib.sc_server_peek(s.h, rid, out.ctypes.data_as(C.POINTER(C.c_float)), out.size,
                                   None) == _lib.SC_E_STATE  # finished: polled, not peeked
    s.close()
    plain = plain_image(ctx, j, 0, 4 * n)
    assert alone.tobytes() == (plain * np.float32(0.25)).tobytes()
    exp = oracle_image(j, 0, 4 * n) * 0.25
    assert exp.sum() > 0 and rel_l1(alone, exp) < FAST_TOL
    # in a mix with single renders, an orbit session and another progressive session
    m = Server(ctx, budget_bytes=1 << 30)
    others = [m.submit(job(0)), m.submit(job(1), frames=3, orbit_deg=2.0)]
    m.step()
    mine = m.submit(j, frames=4)
    others.append(m.submit(job(3), frames=2))
    got = drain(m)
    m.close()
    assert sorted(got) == sorted(others + [mine])
    assert got[mine].tobytes() == alone.tobytes()
    exp3 = oracle_image(job(3), 0, 2 * job(3).n_photons) * 0.5
    assert rel_l1(got[others[2]], exp3) < FAST_TOL


def test_mixed_free_flight_and_uniform_requests(ctx):
    """A server step that holds a free-flight request and uniform ones runs
    the kernel built with free-flight sampling: every image is the same as
    the request's image alone (run by the kernel without it)."""
    reqs = [job(0), job(1), job(4)]
    reqs[1].opts.estimator = 3
    reqs[1].weights.sigma_t = 0.3
    alone = {}
    for i, r in enumerate(reqs):
        a = Server(ctx, budget_bytes=1 << 30)
        rid = a.submit(r)
        alone[i] = drain(a)[rid]
        a.close()
    m = Server(ctx, budget_bytes=1 << 30)
    ids = {m.submit(r): i for i, r in enumerate(reqs)}
    got = drain(m)
    m.close()
    for rid, img in got.items():
        assert img.tobytes() == alone[ids[rid]].tobytes(), ids[rid]
    assert alone[1].tobytes() != plain_image(ctx, job(1), 0, job(1).n_photons).tobytes()
