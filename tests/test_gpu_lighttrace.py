"""Screen-caustic light tracer (spectral-core/src/lighttrace.rs:125-166) and the
z-buffer pass of spectral-core/examples/prism_on_plane.rs:125-160, against the
oracle on the same scenes."""
import ctypes as C

import numpy as np
import pytest

import oracle
import spectral_b200 as sb
from spectral_b200 import _lib
from spectral_b200.scenes import prism_on_plane, wedge_planes

from helpers import obeam, ocam, oscene, rel_l1

pytestmark = pytest.mark.gpu

# The screen of the lighttrace.rs tests (lighttrace.rs:439-476).
SCREEN = ((4.0, -3.0, -2.0), (0.0, 0.0, 4.0), (0.0, 8.0, 0.0))
TEST_BEAM = sb.Beam((-3.0, -0.05, -0.05), (0.0, 0.0, 0.1), (0.0, 0.1, 0.0), (1.0, 0.0, 0.0))


def oracle_trace(scene, screen, beam, n, seed, max_bounces=8):
    p = oracle.vol_params(screen.width, screen.height, seed, max_bounces=max_bounces)
    out = np.zeros(3 * screen.width * screen.height, np.float32)
    scr = np.array(screen.corner + screen.u + screen.v, np.float32)
    oracle.lib.or_lighttrace(C.byref(oscene(scene).c), oracle.fp(scr), screen.width, screen.height,
                             C.byref(obeam(beam)), C.byref(p), n, oracle.fp(out))
    return out


def wedge_scene(glass=sb.SF11):
    sc = sb.Scene(background=0.0)
    sc.add_solid(wedge_planes(30.0, 1.0, 2.0), sb.Dielectric(glass))
    return sc


@pytest.mark.parametrize("w,h,n,seed", [(64, 64, 100_000, 1), (37, 91, 50_000, 0xBEEF)])
def test_lighttrace_matches_oracle(ctx, w, h, n, seed):
    sc = wedge_scene()
    scr = sb.Screen(*SCREEN, w, h)
    sb.trace(ctx, sc, scr, TEST_BEAM, n, seed)
    exp = oracle_trace(sc, scr, TEST_BEAM, n, seed)
    got = scr.sum.reshape(-1)
    assert exp.sum() > 0
    # per-photon paths are bit-identical; the film is int64 at 2^-32 vs the
    # oracle's f32 running sums, so only accumulation rounding differs
    assert rel_l1(got, exp) < 1e-5
    assert np.abs(got - exp).max() <= 1e-4 * max(1.0, float(exp.max()))


def test_lighttrace_accumulates_and_disperses(ctx):
    sc = wedge_scene()
    a = sb.Screen(*SCREEN, 48, 48)
    sb.trace(ctx, sc, a, TEST_BEAM, 20_000, 3)
    once = a.sum.copy()
    sb.trace(ctx, sc, a, TEST_BEAM, 20_000, 3)
    assert np.array_equal(a.sum, 2 * once)  # Screen::sum accumulates across calls
    # without the prism the collimated beam lands on a compact spot; the prism
    # spreads it over many more texels
    empty = sb.Screen(*SCREEN, 48, 48)
    sb.trace(ctx, sb.Scene(background=0.0), empty, TEST_BEAM, 20_000, 3)
    lit = lambda s: int((s.sum[:, 1] > 0).sum())
    assert lit(empty) > 0 and lit(a) > 2 * lit(empty)
    # the empty scene loses nothing: every photon lands with power 1
    y = sb.sample_tables()[71:142].astype(np.float64)
    band_mean = (y.sum() - 0.5 * (y[0] + y[-1])) / 70.0  # mean of the linear interpolant
    assert abs(empty.sum[:, 1].sum() / 20_000 - band_mean) < 0.04 * band_mean


def test_lighttrace_band_and_bounces_match_oracle(ctx):
    sc = wedge_scene(sb.BK7)
    scr = sb.Screen(*SCREEN, 32, 40)
    sb.trace(ctx, sc, scr, TEST_BEAM, 30_000, 9, max_bounces=2)
    assert rel_l1(scr.sum.reshape(-1), oracle_trace(sc, scr, TEST_BEAM, 30_000, 9, max_bounces=2)) < 1e-5


def test_lighttrace_errors(ctx):
    sc = wedge_scene()
    scr = sb.Screen(*SCREEN, 8, 8)
    prims, np_, planes, npl, mats, nm = sc.arrays()
    out = np.zeros(3 * 64, np.float32)
    with pytest.raises(_lib.SpectralError):
        sb.check(sb.lib.sc_lighttrace(ctx.h, prims, np_, planes, npl, mats, nm, None, 8, 8, C.byref(TEST_BEAM.c), 10,
                                      1, None, out.ctypes.data_as(C.POINTER(C.c_float))))
    with pytest.raises(_lib.SpectralError):
        sb.check(sb.lib.sc_lighttrace(ctx.h, prims, np_, planes, npl, mats, nm, C.byref(scr.c()), 0, 8,
                                      C.byref(TEST_BEAM.c), 10, 1, None, out.ctypes.data_as(C.POINTER(C.c_float))))
    bad = sb.Scene(background=0.0)
    bad.add_solid(wedge_planes(30.0, 1.0, 2.0), sb.Dielectric(sb.SF11))
    bad.prims[0].plane_count = 9  # past the plane array
    with pytest.raises(_lib.SpectralError):
        sb.trace(ctx, bad, scr, TEST_BEAM, 10, 1)
    # zero photons is a valid empty trace
    sb.trace(ctx, sc, scr, TEST_BEAM, 0, 1)
    assert not scr.sum.any()


@pytest.mark.parametrize("with_floor", [True, False])
def test_zbuffer_matches_oracle(ctx, with_floor):
    w, h = 160, 120
    scene, floor, _, cam = prism_on_plane(w, h)
    z = sb.scene_zbuffer(ctx, scene, cam, w, h, floor if with_floor else None)
    exp = np.zeros(w * h, np.float32)
    f9 = np.array(floor.corner + floor.u + floor.v, np.float32)
    oracle.lib.or_scene_zbuffer(C.byref(oscene(scene).c), oracle.fp(f9) if with_floor else None,
                                C.byref(ocam(cam)), w, h, oracle.fp(exp))
    assert np.isfinite(exp).sum() > 100 and np.isinf(exp).sum() > 0
    assert z.tobytes() == exp.tobytes()


def test_zbuffered_film_matches_oracle(ctx):
    """The prism_on_plane pipeline on the GPU: z-buffer, then the haze film
    occluded by it, against the oracle's point estimator with the same z."""
    w, h = 96, 72
    scene, floor, beam, cam = prism_on_plane(w, h)
    z = sb.scene_zbuffer(ctx, scene, cam, w, h, floor)
    wts = sb.VolWeights(0.4, 0.12, 0.6)
    film = sb.GpuPhotonFilm(ctx, scene, cam, beam, w, h, 20_000, 0xBEE5, 22.0, wts, zbuffer=z, haze_exact=True)
    film.trace_and_resolve(20_000, 0xBEE5)
    got = film.read_raw().reshape(-1)
    p = oracle.vol_params(w, h, 0xBEE5, 0.4, 0.12, 0.6, 22.0)
    _, fx, _ = oracle.render_point(oscene(scene), ocam(cam), obeam(beam), p, 0, 20_000, zbuf=z, f32=False)
    assert fx.sum() > 0 and rel_l1(got, fx) < 1e-6
    fast = sb.GpuPhotonFilm(ctx, scene, cam, beam, w, h, 20_000, 0xBEE5, 22.0, wts, zbuffer=z)
    fast.trace_and_resolve(20_000, 0xBEE5)
    assert rel_l1(fast.read_raw().reshape(-1), fx) < 2e-3  # fast haze samples
    # occlusion removes energy: the same film without the z-buffer is brighter
    free = sb.GpuPhotonFilm(ctx, scene, cam, beam, w, h, 20_000, 0xBEE5, 22.0, wts)
    free.trace_and_resolve(20_000, 0xBEE5)
    assert free.read_raw().reshape(-1)[1::3].sum() > got[1::3].sum()
