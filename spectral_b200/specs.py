"""Seeded synthetic workloads as plain numbers (no library load).

The benchmark scenes, the uneven batch of prism scenes and the serving request
stream, described by plain Python values: half-spaces as (normal, d), beams
as (corner, u, v, dir), cameras as look_at arguments, jobs and requests as
dicts.  ``scenes.py``, ``batch.py`` and ``serve.py`` turn these into the
library's records; the CPU baseline turns them into the oracle's.  This module
imports nothing from the package (only math and numpy), so it can be loaded on
its own by file path where the CUDA library must not be loaded.

Scene parameters are drawn from the PCG hash stream of spectral-core/src/rng.rs
(``Pcg``), so a seed fixes a whole batch or request stream.
"""
import math

import numpy as np

BK7, SF11, WATER, FUSED_SILICA = 0, 1, 2, 3

# Camera of the prism scenes: in front of the prism on +z, framing prism and fan.
PRISM_CAMERA = ((0.6, -0.4, 6.0), (0.6, -0.4, 0.0), (0.0, 1.0, 0.0), 42.0)


class Pcg:
    """Scene-parameter generator: the PCG hash stream of spectral-core/src/rng.rs."""

    def __init__(self, key, seed):
        self.state = self._pcg(key ^ self._pcg(seed))

    @staticmethod
    def _pcg(x):
        s = (x * 747796405 + 2891336453) & 0xFFFFFFFF
        w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & 0xFFFFFFFF
        return (w >> 22) ^ w

    def u32(self):
        self.state = (self.state + 1) & 0xFFFFFFFF
        return self._pcg(self.state)

    def f(self):
        return (self.u32() >> 8) * (1.0 / 16777216.0)

    def uniform(self, lo, hi):
        return lo + (hi - lo) * self.f()

    def log_uniform(self, lo, hi):
        return math.exp(self.uniform(math.log(lo), math.log(hi)))


def prism_planes(apex_deg, side, depth):
    """Outward half-spaces n.x + d <= 0 of a prism with its apex up, the two
    faces of length `side` meeting at the apex, centroid at the origin."""
    a = math.radians(apex_deg) / 2.0
    y_top = (2.0 / 3.0) * side * math.cos(a)
    y_base = y_top - side * math.cos(a)
    left = (-math.cos(a), math.sin(a), 0.0)
    right = (math.cos(a), math.sin(a), 0.0)
    return [(left, -(math.sin(a) * y_top)), (right, -(math.sin(a) * y_top)), ((0.0, -1.0, 0.0), y_base),
            ((0.0, 0.0, 1.0), -depth / 2.0), ((0.0, 0.0, -1.0), -depth / 2.0)]


def prism_beam(apex_deg, side, incidence_deg, width, back=2.0):
    """(corner, u, v, dir) of a square beam of side `width` aimed at the middle
    of the left face with the given angle of incidence (from the face normal)."""
    a = math.radians(apex_deg) / 2.0
    y_top = (2.0 / 3.0) * side * math.cos(a)
    mid = np.array([-math.sin(a) * side / 2.0, y_top - math.cos(a) * side / 2.0, 0.0])
    inward = np.array([math.cos(a), -math.sin(a), 0.0])  # -normal of the left face
    t = math.radians(incidence_deg)
    d = np.array([inward[0] * math.cos(t) - inward[1] * math.sin(t),
                  inward[0] * math.sin(t) + inward[1] * math.cos(t), 0.0])
    d = d / np.linalg.norm(d)
    perp = np.array([-d[1], d[0], 0.0])
    origin = mid - d * back
    corner = origin - perp * (width / 2.0) - np.array([0.0, 0.0, width / 2.0])
    return (tuple(float(x) for x in corner), (0.0, 0.0, float(width)), tuple(float(x) for x in perp * width),
            tuple(float(x) for x in np.float32(d)))


def prism_scene(apex_deg=60.0, side=1.0, incidence_deg=45.0, beam_width=0.02, depth=1.0, glass=SF11):
    """The single-prism benchmark scene: dict with the solid's half-spaces, its
    glass, the beam and the camera's look_at arguments (aspect set by the film)."""
    return dict(solids=[(prism_planes(apex_deg, side, depth), ("glass", glass))], spheres=[],
                beam=prism_beam(apex_deg, side, incidence_deg, beam_width), camera=PRISM_CAMERA)


def rainbow_scene(beam_width=2.2):
    """Water sphere r=1 at the origin; photons travel +x; camera on the sun
    side, off axis, so the backward primary/secondary bows cross the frame."""
    h = beam_width / 2.0
    return dict(solids=[], spheres=[((0.0, 0.0, 0.0), 1.0, ("glass", WATER))],
                beam=((-3.0, -h, -h), (0.0, 0.0, beam_width), (0.0, beam_width, 0.0), (1.0, 0.0, 0.0)),
                camera=((-7.0, 1.0, 2.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 60.0))


def tracer_scene():
    """Camera-tracer scene: SF11 prism (apex 60, side 1) on a diffuse ground
    half-space (albedo 0.8, y = -0.6), a spherical D65 emitter of radius 0.2 at
    (2, 3, 1), Russian roulette after 3 scatters."""
    return dict(solids=[(prism_planes(60.0, 1.0, 1.0), ("glass", SF11)), ([((0.0, 1.0, 0.0), 0.6)],
                                                                          ("lambertian", 0.8))],
                spheres=[], camera=((0.5, 1.5, 5.0), (0.0, -0.3, 0.0), (0.0, 1.0, 0.0), 45.0),
                tracer=dict(emitter=((2.0, 3.0, 1.0), 0.2, 40.0), rr_start=3, max_depth=8))


def f32_normalize(v):
    """glam Vec3::normalize in f32: v * (1 / sqrt((x*x + y*y) + z*z))."""
    x, y, z = (np.float32(c) for c in v)
    ln = np.sqrt(x * x + y * y + z * z, dtype=np.float32)
    r = np.float32(1.0) / ln
    return (float(x * r), float(y * r), float(z * r))


def dsotm_scene():
    """dsotm_scene (spectral-gpu/src/vol_photons.rs:188-222): the SF11 prism of
    planes k = 0.9, base y = -1, its beam and its camera (aspect set by the film)."""
    k = 0.9
    planes = [((-0.8660254, 0.5, 0.0), -k), ((0.8660254, 0.5, 0.0), -k), ((0.0, -1.0, 0.0), -1.0),
              ((0.0, 0.0, 1.0), -1.0), ((0.0, 0.0, -1.0), -1.0)]
    bdir = f32_normalize((0.84, 0.54, 0.0))
    bperp = tuple(float(np.float32(c) * np.float32(0.05)) for c in f32_normalize((-0.54, 0.84, 0.0)))
    return dict(solids=[(planes, ("glass", SF11))], spheres=[],
                beam=((-2.6, -0.95, -0.6), (0.0, 0.0, 1.2), bperp, bdir),
                camera=((0.5, -0.5, 12.0), (0.5, -0.5, 0.0), (0.0, 1.0, 0.0), 42.0))


def _prism_spec(g, seed, index, bins, photons, side, lambda_min, lambda_max, glasses=(BK7, SF11, FUSED_SILICA)):
    glass = glasses[g.u32() % 3]
    apex = g.uniform(30.0, 75.0)
    inc = g.uniform(30.0, 60.0)
    n = int(round(g.log_uniform(*photons)))
    s = int(round(g.log_uniform(*side)))
    sigma_s = g.uniform(0.01, 0.1)
    return dict(glass=glass, apex_deg=apex, incidence_deg=inc, n_photons=n, width=s, height=s, sigma_s=sigma_s,
                sigma_t=sigma_s, g=0.0, seed=(seed * 2654435761 + index) & 0xFFFFFFFF, bins=bins,
                lambda_min=lambda_min, lambda_max=lambda_max)


def random_prism_jobs(n_jobs=256, seed=0xB200, bins=32, photons=(2 ** 14, 2 ** 22), side=(128, 1024),
                      lambda_min=380.0, lambda_max=780.0):
    """The uneven batch, one dict per scene: glass from {BK7, SF11, fused
    silica}, apex U(30, 75) deg, incidence U(30, 60) deg, photons
    log-U(2^14, 2^22), square film side log-U(128, 1024), sigma_s U(0.01, 0.1)."""
    return [_prism_spec(Pcg(j, seed), seed, j, bins, photons, side, lambda_min, lambda_max) for j in range(n_jobs)]


def poisson_request_specs(rate=200.0, seconds=60.0, seed=0x5E7E, session_share=0.3, frames=(16, 128),
                          photons=(2 ** 16, 2 ** 20), side=(128, 1024), bins=32, orbit_deg=2.0):
    """Seeded request stream: list of (arrival_s, job dict, frames, orbit_deg).
    Arrivals are Poisson at `rate`; each request is a prism scene of the batch
    distribution with 2^16-2^20 photons per frame; a `session_share` of them are
    orbit sessions of 16-128 frames stepping the camera azimuth `orbit_deg`."""
    g = Pcg(0, seed)
    out, t, i = [], 0.0, 0
    while True:
        t += -math.log(1.0 - g.f()) / rate
        if t >= seconds:
            break
        r = Pcg(i, seed ^ 0x9E3779B9)
        spec = _prism_spec(r, seed, i, bins, photons, side, 380.0, 780.0)
        sess = r.f() < session_share
        nf = (frames[0] + r.u32() % (frames[1] - frames[0] + 1)) if sess else 1
        out.append((t, spec, nf, orbit_deg if sess else 0.0))
        i += 1
    return out
