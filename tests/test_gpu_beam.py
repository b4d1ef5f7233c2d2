"""Photon-beam estimator (render_volumetric_scene + splat_transverse,
spectral-core/src/volume.rs:170-329) on the GPU against the oracle."""
import os

import numpy as np
import pytest

import oracle
import spectral_b200 as sb
from spectral_b200 import _lib

from helpers import obeam, ocam, oscene, rel_l1

pytestmark = pytest.mark.gpu

# Per-step weights use expf / powf (a few ulp apart between CUDA and glibc) and
# the oracle sums in f32; the film is int64 at 2^-40.  Everything else (march
# counts, footprints, tent weights) is bit-identical.
BEAM_TOL = 1e-4


def beam_film(ctx, scene, cam, beam, w, h, n, seed, max_dist=14.0, weights=None, **kw):
    f = sb.GpuPhotonFilm(ctx, scene, cam, beam, w, h, n, seed, max_dist, weights or sb.VolWeights(),
                         estimator=sb.BEAM, **kw)
    f.trace_and_resolve(n, seed)
    return f


@pytest.mark.parametrize("w,h,n,seed", [(64, 64, 2000, 7), (120, 90, 3000, 0xDED)])
def test_beam_dsotm_matches_oracle(ctx, w, h, n, seed):
    scene, beam, cam = sb.dsotm_scene(w / h)
    f = beam_film(ctx, scene, cam, beam, w, h, n, seed)
    p = oracle.vol_params(w, h, seed, 0.5, 0.06, 0.5, 14.0)
    exp = oracle.render_beam(oscene(scene), ocam(cam), obeam(beam), p, 0, n)
    got = f.accum()
    assert exp.sum() > 0
    assert rel_l1(got, exp) < BEAM_TOL


def test_beam_film_against_golden_fixture(ctx):
    """The committed beam-estimator fixture (tests/golden/make_golden.py:
    600 DSOTM photons, seed 3, 48x40)."""
    scene, beam, cam = sb.dsotm_scene(48 / 40)
    f = beam_film(ctx, scene, cam, beam, 48, 40, 600, 3)
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "beam_film_48x40.npz"))["img_f32"]
    assert g.sum() > 0 and rel_l1(f.accum(), g) < BEAM_TOL


def test_beam_empty_scene_energy_matches_point_estimator(ctx):
    """volume.rs:361-395 on the GPU: beam and point estimators integrate the
    same in-scatter (Y sums within 8 %)."""
    w, h = 128, 96
    scene = sb.Scene(background=0.0)
    beam = sb.Beam((-2.0, 0.0, 0.0), (0.0, 0.0, 0.6), (0.0, 0.4, 0.0), (1.0, 0.0, 0.0))
    cam = sb.Camera.look_at((0.0, 0.5, 6.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 45.0, w / h)
    wts = sb.VolWeights(0.5, 0.06, 0.4)
    bm = beam_film(ctx, scene, cam, beam, w, h, 20_000, 7, 12.0, wts).accum()
    pt = sb.GpuPhotonFilm(ctx, scene, cam, beam, w, h, 20_000, 7, 12.0, wts)
    pt.trace_and_resolve(20_000, 7)
    yp, yb = pt.accum()[1::3].sum(dtype=np.float64), bm[1::3].sum(dtype=np.float64)
    assert yp > 0 and yb > 0 and 0.92 <= yb / yp <= 1.08
    p = oracle.vol_params(w, h, 7, 0.5, 0.06, 0.4, 12.0)
    assert rel_l1(bm, oracle.render_beam(oscene(scene), ocam(cam), obeam(beam), p, 0, 20_000)) < BEAM_TOL


def test_beam_zbuffer(ctx):
    w, h, n, seed = 96, 64, 1500, 11
    scene, beam, cam = sb.dsotm_scene(w / h)
    zb = np.full(w * h, np.inf, np.float32)
    zb[: w * h // 3] = 11.0
    f = beam_film(ctx, scene, cam, beam, w, h, n, seed, zbuffer=zb)
    p = oracle.vol_params(w, h, seed, 0.5, 0.06, 0.5, 14.0)
    exp = oracle.render_beam(oscene(scene), ocam(cam), obeam(beam), p, 0, n, zbuf=zb)
    free = oracle.render_beam(oscene(scene), ocam(cam), obeam(beam), p, 0, n)
    assert 0 < exp.sum() < free.sum() and rel_l1(f.accum(), exp) < BEAM_TOL


def test_beam_wide_footprints_near_camera(ctx):
    """A thin beam passing ~0.1 from the camera: projected radii up to the
    24 px clamp, footprints clipped by the frame edge, the 4096-step clamp."""
    w, h, n, seed = 64, 48, 300, 13
    scene = sb.Scene(background=0.0)
    beam = sb.Beam((-2.0, -0.01, -0.01), (0.0, 0.0, 0.02), (0.0, 0.02, 0.0), (1.0, 0.0, 0.0))
    cam = sb.Camera.look_at((0.5, 0.06, 0.06), (3.0, 0.0, 0.0), (0.0, 1.0, 0.0), 70.0, w / h)
    f = beam_film(ctx, scene, cam, beam, w, h, n, seed, 8.0)
    p = oracle.vol_params(w, h, seed, 0.5, 0.06, 0.5, 8.0)
    exp = oracle.render_beam(oscene(scene), ocam(cam), obeam(beam), p, 0, n)
    assert exp.sum() > 0 and rel_l1(f.accum(), exp) < BEAM_TOL


def test_beam_launch_variants_identical(ctx, monkeypatch):
    scene, beam, cam = sb.dsotm_scene(1.0)
    films = []
    for agg in ("0", "1"):
        monkeypatch.setenv("SPECTRAL_CUDA_AGGREGATE", agg)
        films.append(beam_film(ctx, scene, cam, beam, 80, 80, 2500, 5).read_raw())
    assert films[0].tobytes() == films[1].tobytes() and films[0].any()
    # photon ranges add exactly: [0, 1000) + [1000, 2500) == [0, 2500)
    f = sb.GpuPhotonFilm(ctx, scene, cam, beam, 80, 80, 2500, 5, 14.0, sb.VolWeights(), estimator=sb.BEAM)
    f.dispatch_photons(0, 1000, 5)  # dispatch_photons(base, end): photons [base, end)
    f.dispatch_photons(1000, 2500, 5)
    assert f.read_raw().tobytes() == films[0].tobytes()


def test_beam_spectral_film_reduces_to_xyz(ctx):
    w, h, n, seed = 64, 48, 2000, 3
    scene, beam, cam = sb.dsotm_scene(w / h)
    xyz = beam_film(ctx, scene, cam, beam, w, h, n, seed).accum()
    spec = beam_film(ctx, scene, cam, beam, w, h, n, seed, bins=128).accum()
    # the spectral film bins radiance and applies bin-averaged CMF weights:
    # equal to the XYZ film up to the CMF variation inside a 2.7 nm bin
    assert rel_l1(spec, xyz) < 0.02


def test_beam_rejects_point_only_calls(ctx):
    scene, beam, cam = sb.dsotm_scene(1.0)
    f = sb.GpuPhotonFilm(ctx, scene, cam, beam, 16, 16, 100, 1, 14.0, sb.VolWeights(), estimator=sb.BEAM)
    with pytest.raises(_lib.SpectralError) as e:
        f.trace_debug(10, 1, 4)
    assert e.value.code == _lib.SC_E_STATE
    with pytest.raises(_lib.SpectralError):  # estimators are 0-3
        sb.GpuPhotonFilm(ctx, scene, cam, beam, 16, 16, 100, 1, 14.0, sb.VolWeights(), estimator=4)
