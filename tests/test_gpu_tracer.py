"""GPU parity of the wavefront hero-wavelength camera tracer against the CPU
oracle (spectral-gpu/tests/diff_gate.rs, lambertian_gate.rs, lib.rs tests;
spectral-core/src/tracer.rs tests).

Scenes without Lambertian surfaces use only + - * / sqrt on the path and are
required to be bit-identical.  Lambertian sampling calls cosf/sinf, whose last
bits differ between CUDA and glibc, so those scenes use the reference's
statistical gates (frac of pixels above 10x the mean difference, p99, energy).
"""
import math
import os

import numpy as np
import pytest

import oracle
import spectral_b200 as sb
from spectral_b200 import _lib

from helpers import axis_box, ocam, oscene, triangular_prism

pytestmark = pytest.mark.gpu

ENERGY_TOL = 0.01   # diff_gate.rs:220
P99_TOL = 0.05      # diff_gate.rs:216
FRAC_TOL = 0.005    # diff_gate.rs:212


def fixed_scene(lambertian_front=False):
    s = sb.Scene(background=1.0)
    s.add_sphere((0, 0, -3), 1.0, sb.Lambertian(0.5) if lambertian_front else sb.Dielectric(sb.SF11))
    s.add_sphere((0, 0, -6), 2.0, sb.Lambertian(0.7))
    return s


def cam64():
    return sb.Camera.look_at((0, 0, 0), (0, 0, -1), (0, 1, 0), 50.0, 1.0)


def gate_stats(cpu_mean, gpu_mean):
    c = cpu_mean.reshape(-1, 3).astype(np.float64)
    g = gpu_mean.reshape(-1, 3).astype(np.float64)
    pp = np.abs(c - g).sum(1)
    mean_pp = pp.mean()
    frac = (pp > 10 * mean_pp).mean() if mean_pp > 0 else 0.0
    p99 = np.sort(pp)[min(int(len(pp) * 0.99), len(pp) - 1)]
    energy = abs(c.sum() - g.sum()) / max(c.sum(), 1e-6)
    return frac, p99, energy


def run_both(ctx, scene, cam, w, h, spp, seed, illuminant=sb.D65, **kw):
    t = sb.GpuTracer(ctx, scene, cam, w, h, illuminant, seed, **kw)
    t.accumulate(spp)
    gpu = t.read_xyz()
    ext = None
    if kw.get("emitter") or kw.get("rr_start"):
        c, r, sc = kw.get("emitter") or ((0, 0, 0), 0.0, 0.0)
        ext = oracle.or_tracer_ext(oracle.F3(*c), r, sc, kw.get("rr_start", 0))
    cpu = oracle.tracer_accumulate(oscene(scene), ocam(cam), w, h, illuminant, seed, spp,
                                   max_bounces=kw.get("max_depth", 8), ext=ext) / np.float32(spp)
    return gpu, cpu, t


def test_gpu_renders_nonzero_for_lit_scene(ctx):
    t = sb.GpuTracer(ctx, sb.Scene(background=1.0), sb.Camera.look_at((0, 0, 0), (0, 0, -1), (0, 1, 0), 60, 1),
                     16, 16, sb.D65, 42)
    t.accumulate(4)
    xyz = t.read_xyz()
    assert xyz.size == 3 * 256 and xyz[1::3].sum() > 0


@pytest.mark.parametrize("seed", [0xD1FF, 0xD200])
def test_diff_gate(ctx, seed):
    gpu, cpu, _ = run_both(ctx, fixed_scene(), cam64(), 64, 64, 64, seed)
    frac, p99, energy = gate_stats(cpu, gpu)
    print("diff gate seed %#x: frac %.4f p99 %.4f energy %.2e, identical pixels %.3f" % (
        seed, frac, p99, energy, (gpu.reshape(-1, 3) == cpu.reshape(-1, 3)).all(1).mean()))
    assert frac < FRAC_TOL and p99 < P99_TOL and energy < ENERGY_TOL


def test_lambertian_gate(ctx):
    gpu, cpu, _ = run_both(ctx, fixed_scene(lambertian_front=True), cam64(), 64, 64, 64, 0xD1FF)
    frac, p99, energy = gate_stats(cpu, gpu)
    assert frac < 0.002 and p99 < 0.02 and energy < ENERGY_TOL


def test_dielectric_scene_bit_identical(ctx):
    s = sb.Scene(background=1.0, horizon=2.0)
    s.add_sphere((0, 0, -3), 1.0, sb.Dielectric(sb.SF11))
    s.add_solid(axis_box((-3, -2, -6), (-1.5, 2, -4)), sb.Dielectric(sb.BK7))
    s.add_sphere((1.8, 0.5, -4), 0.7, sb.Dielectric(sb.WATER))
    cam = sb.Camera.look_at((0, 0.3, 0.5), (0, 0, -3), (0, 1, 0), 55.0, 1.5)
    gpu, cpu, t = run_both(ctx, s, cam, 96, 64, 16, 77)
    assert gpu.tobytes() == cpu.tobytes()
    # progressive: sample indices continue across accumulate calls
    t.accumulate(8)
    t.accumulate(8)
    acc = oracle.tracer_accumulate(oscene(s), ocam(cam), 96, 64, 0, 77, 16)
    acc = oracle.tracer_accumulate(oscene(s), ocam(cam), 96, 64, 0, 77, 8, base=16, out=acc)
    acc = oracle.tracer_accumulate(oscene(s), ocam(cam), 96, 64, 0, 77, 8, base=24, out=acc)
    assert t.read_xyz().tobytes() == (acc / np.float32(32)).tobytes()
    paths, segs = t.stats()
    assert paths == 96 * 64 * 8 and segs > paths


def test_set_spectral_off_uses_n550_bit_identical(ctx):
    """set_spectral(false) (lib.rs:369-372, trace.wgsl:477-480): every dielectric
    hit refracts with n(550 nm); the image equals the oracle's with the same
    switch, and differs from the dispersive image."""
    s = sb.Scene(background=1.0, horizon=2.0)
    s.add_sphere((0, 0, -3), 1.0, sb.Dielectric(sb.SF11))
    s.add_solid(axis_box((-3, -2, -6), (-1.5, 2, -4)), sb.Dielectric(sb.BK7))
    cam = sb.Camera.look_at((0, 0.3, 0.5), (0, 0, -3), (0, 1, 0), 55.0, 1.5)
    t = sb.GpuTracer(ctx, s, cam, 80, 56, sb.D65, 21)
    t.set_spectral(False)
    t.accumulate(8)
    off = t.read_xyz()
    cpu = oracle.tracer_accumulate(oscene(s), ocam(cam), 80, 56, 0, 21, 8, spectral=False) / np.float32(8)
    assert off.tobytes() == cpu.tobytes()
    t.clear_accum()
    t.set_spectral(True)
    t.accumulate(8)
    on = t.read_xyz()
    assert on.tobytes() != off.tobytes()
    cpu_on = oracle.tracer_accumulate(oscene(s), ocam(cam), 80, 56, 0, 21, 8) / np.float32(8)  # cleared: from 0
    assert on.tobytes() == cpu_on.tobytes()


def test_row_bands_render_like_the_full_image(ctx):
    """set_rows (the camera tracer's pixel-row ownership for multi-GPU): a band
    traced alone equals the same rows of the full render bit for bit, rows
    outside it stay empty, and an empty band traces nothing."""
    s = sb.Scene(background=1.0, horizon=2.0)
    s.add_sphere((0, 0, -3), 1.0, sb.Dielectric(sb.SF11))
    cam = sb.Camera.look_at((0, 0.3, 0.5), (0, 0, -3), (0, 1, 0), 55.0, 1.5)
    w, h = 64, 41
    full = sb.GpuTracer(ctx, s, cam, w, h, sb.D65, 9)
    full.accumulate(8)
    full.accumulate(4)
    ref = full.read_xyz().reshape(h, w, 3)
    for b, e in ((0, 13), (13, 41), (20, 20)):
        t = sb.GpuTracer(ctx, s, cam, w, h, sb.D65, 9)
        t.set_rows(b, e)
        t.accumulate(8)
        t.accumulate(4)
        img = t.read_xyz().reshape(h, w, 3)
        assert img[b:e].tobytes() == ref[b:e].tobytes(), (b, e)
        assert not img[:b].any() and not img[e:].any()
        t.close()
    with pytest.raises(_lib.SpectralError):
        full.set_rows(5, h + 1)


def _chroma_spread(img):
    """Largest chromaticity distance from the D65 white point over the pixels
    (core/tests/scene_a_prism.rs:51-65)."""
    px = img.reshape(-1, 3).astype(np.float32)
    s = px.sum(1)
    m = s > 1e-5
    x, y = px[m, 0] / s[m], px[m, 1] / s[m]
    return float(np.sqrt((x - 0.3127) ** 2 + (y - 0.3290) ** 2).max()) if m.any() else 0.0


def test_dispersive_prism_colors_horizon_more_than_diffuse(ctx):
    """core/tests/scene_a_prism.rs:67-90 on the GPU tracer: an SF11 prism in
    front of a bright horizon colours the image far more than a Lambertian prism
    of the same shape (128x128, 256 spp, seed 11)."""
    def render(mat):
        s = sb.Scene(background=0.3, horizon=4.0)
        s.add_solid(triangular_prism(1.0, 2.0), mat)
        cam = sb.Camera.look_at((0.0, 0.0, 4.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 50.0, 1.0)
        t = sb.GpuTracer(ctx, s, cam, 128, 128, sb.D65, 11)
        t.accumulate(256)
        return t.read_xyz()
    cg = _chroma_spread(render(sb.Dielectric(sb.SF11)))
    cd = _chroma_spread(render(sb.Lambertian(0.8)))
    assert cg > 0.05 and cg > 2.0 * cd, (cg, cd)


def test_tracer_against_golden_fixture(ctx):
    """The committed camera-tracer fixture (tests/golden/make_golden.py: SF11 and
    water spheres under a horizon, 32x24, 8 spp, seed 77): bit-identical."""
    s = sb.Scene(background=1.0, horizon=2.0)
    s.add_sphere((0.0, 0.0, -3.0), 1.0, sb.Dielectric(sb.SF11))
    s.add_sphere((1.8, 0.5, -4.0), 0.7, sb.Dielectric(sb.WATER))
    cam = sb.Camera.look_at((0.0, 0.3, 0.5), (0.0, 0.0, -3.0), (0.0, 1.0, 0.0), 55.0, 32.0 / 24.0)
    t = sb.GpuTracer(ctx, s, cam, 32, 24, sb.D65, 77)
    t.accumulate(8)
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "tracer_glass_32x24.npz"))["mean_xyz"]
    assert t.read_xyz().tobytes() == g.tobytes()


def test_background_integrates_to_d65_and_illuminant_a(ctx):
    cam = sb.Camera.look_at((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, 1.0)
    t = sb.GpuTracer(ctx, sb.Scene(background=1.0), cam, 32, 32, sb.D65, 7)
    t.accumulate(256)
    m = t.read_xyz().reshape(-1, 3).sum(0).astype(np.float64)
    assert abs(m[0] / m.sum() - 0.3127) < 6e-3 and abs(m[1] / m.sum() - 0.3290) < 6e-3
    gpu, cpu, _ = run_both(ctx, sb.Scene(background=1.0), cam, 32, 32, 16, 3, illuminant=sb.ILLUMINANT_A)
    assert gpu.tobytes() == cpu.tobytes()
    # the render-level illuminant gate (core/tests/scene_b_metamerism.rs:69-100):
    # the chromaticity moves by more than 0.05 from D65 to illuminant A
    a = gpu.reshape(-1, 3).sum(0).astype(np.float64)
    dist = math.hypot(m[0] / m.sum() - a[0] / a.sum(), m[1] / m.sum() - a[1] / a.sum())
    assert dist > 0.05, dist


def test_dispersion_collapse_preserves_brightness(ctx):
    cam = sb.Camera.look_at((0, 0, 3), (0, 0, 0), (0, 1, 0), 18.0, 1.0)
    t0 = sb.GpuTracer(ctx, sb.Scene(background=1.0), cam, 8, 8, sb.D65, 3)
    t0.accumulate(256)
    slab = sb.Scene(background=1.0)
    slab.add_solid(axis_box((-5, -5, -0.1), (5, 5, 0.1)), sb.Dielectric(sb.BK7))
    t1 = sb.GpuTracer(ctx, slab, cam, 8, 8, sb.D65, 3)
    t1.accumulate(256)
    y0, y1 = t0.read_xyz()[1::3].mean(), t1.read_xyz()[1::3].mean()
    assert y0 > 0 and 0.7 * y0 < y1 < 1.05 * y0


def test_emitter_roulette_ground_plane(ctx):
    """The camera-tracer extensions of the benchmark scene (prism on a diffuse
    plane, spherical D65 emitter, Russian roulette after 3 scatters)."""
    from spectral_b200.scenes import prism_planes
    s = sb.Scene(background=0.0)
    s.add_solid(prism_planes(60.0, 1.0, 1.0), sb.Dielectric(sb.SF11))
    s.add_solid([((0, 1, 0), 0.6)], sb.Lambertian(0.8))  # ground y >= -0.6 is outside
    cam = sb.Camera.look_at((0.5, 1.5, 5.0), (0, -0.3, 0), (0, 1, 0), 45.0, 16 / 9)
    kw = dict(emitter=((2.0, 3.0, 1.0), 0.2, 40.0), rr_start=3)
    gpu, cpu, _ = run_both(ctx, s, cam, 96, 54, 32, 11, **kw)
    frac, p99, energy = gate_stats(cpu, gpu)
    assert cpu[1::3].sum() > 0
    assert energy < 0.03 and frac < 0.02
    # without Lambertian surfaces the extensions are bit-exact too
    s2 = sb.Scene(background=0.0)
    s2.add_solid(prism_planes(60.0, 1.0, 1.0), sb.Dielectric(sb.SF11))
    gpu2, cpu2, _ = run_both(ctx, s2, cam, 64, 36, 16, 12, emitter=((0.0, 0.0, -2.0), 1.5, 3.0), rr_start=1)
    assert gpu2.tobytes() == cpu2.tobytes() and cpu2.sum() > 0


def test_set_camera_and_clear(ctx):
    s = fixed_scene()
    t = sb.GpuTracer(ctx, s, cam64(), 32, 32, sb.D65, 5)
    t.accumulate(4)
    t.clear_accum()
    assert not t.read_xyz().any()
    cam2 = sb.Camera.look_at((0.2, 0.1, 0), (0, 0, -3), (0, 1, 0), 40.0, 1.0)
    t.set_camera(cam2)
    t.accumulate(8)
    cpu = oracle.tracer_accumulate(oscene(s), ocam(cam2), 32, 32, 0, 5, 8, base=0) / np.float32(8)
    frac, p99, energy = gate_stats(cpu, t.read_xyz())
    assert energy < ENERGY_TOL and p99 < P99_TOL


def test_many_waves_on_both_chains_bit_identical(ctx):
    """An image of several 2^19-path waves: consecutive waves run on the two
    overlapping chains, and the image still equals the CPU tracer's bit for bit
    (a ragged last wave included)."""
    s = sb.Scene(background=1.0, horizon=2.0)
    s.add_sphere((0, 0, -3), 1.0, sb.Dielectric(sb.SF11))
    s.add_solid(axis_box((-3, -2, -6), (-1.5, 2, -4)), sb.Dielectric(sb.BK7))
    cam = sb.Camera.look_at((0, 0.3, 0.5), (0, 0, -3), (0, 1, 0), 55.0, 1.5)
    w, h, spp = 150, 101, 96  # 15150 pixels x 96 = 1.45 M paths: 3 waves, the last one partial
    gpu, cpu, t = run_both(ctx, s, cam, w, h, spp, 0x51)
    assert cpu.sum() > 0 and gpu.tobytes() == cpu.tobytes()
    paths, segs = t.stats()
    assert paths == w * h * spp and segs >= paths


@pytest.mark.parametrize("sched", [dict(wave_bounces=1), dict(wave_bounces=3), dict(wave_bounces=8),
                                   dict(chains=1), dict(chains=4, wave_paths_log2=12),
                                   dict(chains=3, wave_paths_log2=13, wave_bounces=3)])
def test_wave_schedule_is_scheduling_only(ctx, sched):
    """How many bounces run as compacted wavefront stages before the in-place
    tail, how many waves are in flight and how many paths a wave holds change
    only the schedule: the image is bit-identical."""
    from spectral_b200.scenes import tracer_workload
    scene, cam, kw = tracer_workload(96, 64)
    ref = sb.GpuTracer(ctx, scene, cam, 96, 64, sb.D65, 0x51, **kw)
    ref.accumulate(8)
    t = sb.GpuTracer(ctx, scene, cam, 96, 64, sb.D65, 0x51, **sched, **kw)
    t.accumulate(8)
    a, b = ref.read_xyz(), t.read_xyz()
    assert a.sum() > 0 and a.tobytes() == b.tobytes()


def _shifted(planes, offset):
    """The same convex solid moved by `offset` (n . (x - c) + d <= 0)."""
    return [(n, d - (n[0] * offset[0] + n[1] * offset[1] + n[2] * offset[2])) for n, d in planes]


@pytest.mark.parametrize("eye", [(0.0, 0.3, 0.0), (0.0, 0.2, -6.0)])
def test_bounding_spheres_keep_every_hit(ctx, eye):
    """The tracer skips the plane tests of a convex solid when a ray misses a
    sphere around it; the nearest hit must not change.  A dielectric scene of
    21 small boxes (one behind the camera, some that rays graze), a wedge, an
    unbounded three-plane prism (no caps: never skipped) and a ground
    half-space renders bit-identically to the oracle, with the eye outside
    every solid's sphere and with the eye inside a box."""
    s = sb.Scene(background=1.0, horizon=3.0)
    s.add_solid([((0.0, 1.0, 0.0), 1.5)], sb.Dielectric(sb.BK7))  # ground half-space y <= -1.5
    for i in range(-3, 4):
        for j in range(3):
            c = (i * 1.2, -0.6 + j * 0.8, -5.0 - j)
            s.add_solid(axis_box((c[0] - 0.3, c[1] - 0.3, c[2] - 0.3), (c[0] + 0.3, c[1] + 0.3, c[2] + 0.3)),
                        sb.Dielectric(sb.SF11 if (i + j) % 2 else sb.BK7))
    s.add_solid(axis_box((-0.4, -0.4, 2.6), (0.4, 0.4, 3.4)), sb.Dielectric(sb.BK7))  # behind the camera
    s.add_solid(_shifted(triangular_prism(0.4, 0.0)[:3], (2.5, 1.2, 0.0)), sb.Dielectric(sb.SF11))  # no caps
    from helpers import wedge
    s.add_solid(_shifted(wedge(40.0, 0.3, 0.5), (-2.2, 1.1, -3.0)), sb.Dielectric(sb.BK7))
    cam = sb.Camera.look_at(eye, (0.0, 0.0, -10.0), (0.0, 1.0, 0.0), 70.0, 4.0 / 3.0)
    gpu, cpu, _ = run_both(ctx, s, cam, 96, 72, 4, 0xB0B)
    assert cpu.sum() > 0 and gpu.tobytes() == cpu.tobytes()
