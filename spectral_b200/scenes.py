"""Scene builders for the benchmark workloads (seeded, synthetic).

* ``prism_workload``: an isosceles glass prism (apex angle, side length) built
  from five half-spaces, lit by a square collimated beam hitting the middle of
  the left face at a given incidence; camera in front on +z.
* ``rainbow_workload``: a water sphere of radius 1 in a wide collimated beam,
  camera on the sun side looking at the sphere.
* ``random_prism_jobs``: the uneven batch of prism scenes (glass from
  {BK7, SF11, fused silica}, apex U(30, 75) deg, incidence U(30, 60) deg,
  photons log-U(2^14, 2^22), square film side log-U(128, 1024)), drawn from a
  PCG-seeded generator so a seed fixes the whole batch.
"""
import math

import numpy as np

from . import BK7, FUSED_SILICA, SF11, WATER, Beam, Camera, Dielectric, Lambertian, Scene, Screen


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
    """Square beam of side `width` aimed at the middle of the left face with
    the given angle of incidence (measured from the face normal)."""
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
    return Beam(tuple(corner), (0.0, 0.0, width), tuple(perp * width), tuple(np.float32(d)))


def prism_workload(width=640, height=360, glass=SF11, apex_deg=60.0, side=1.0, incidence_deg=45.0,
                   beam_width=0.02, depth=1.0):
    scene = Scene(background=0.0)
    scene.add_solid(prism_planes(apex_deg, side, depth), Dielectric(glass))
    beam = prism_beam(apex_deg, side, incidence_deg, beam_width)
    cam = Camera.look_at((0.6, -0.4, 6.0), (0.6, -0.4, 0.0), (0.0, 1.0, 0.0), 42.0, width / height)
    return scene, beam, cam


def wedge_planes(apex_deg, size, depth):
    """ConvexSolid::wedge (spectral-core/src/geom.rs:110-121) in f32 trig."""
    a = np.float32(apex_deg) * np.float32(np.float32(math.pi) / np.float32(180.0))
    return [((-1.0, 0.0, 0.0), -size), ((float(np.cos(a)), float(np.sin(a)), 0.0), -size), ((0.0, -1.0, 0.0), -size),
            ((0.0, 0.0, 1.0), -depth / 2.0), ((0.0, 0.0, -1.0), -depth / 2.0)]


def prism_on_plane(width=800, height=600, floor_texels=512):
    """The floor, SF11 wedge, beam and oblique camera of
    spectral-core/examples/prism_on_plane.rs:77-119: returns
    (scene, floor Screen, beam, camera)."""
    floor = Screen((-5.0, -1.0, -5.0), (0.0, 0.0, 10.0), (14.0, 0.0, 0.0), floor_texels, floor_texels)
    scene = Scene(background=0.0)
    scene.add_solid(wedge_planes(30.0, 1.0, 2.0), Dielectric(SF11))
    beam = Beam((-3.0, 0.55, -0.75), (0.0, 0.0, 1.5), (0.0, 0.12, 0.0), (1.0, 0.0, 0.0))
    cam = Camera.look_at((0.0, 4.5, 9.0), (4.0, -1.2, 0.0), (0.0, 1.0, 0.0), 50.0, width / height)
    return scene, floor, beam, cam


def tracer_workload(width=1280, height=720):
    """Camera-tracer scene: SF11 prism (apex 60, side 1) on a diffuse ground
    half-space (albedo 0.8, y = -0.6), lit by a spherical D65 emitter of radius
    0.2 at (2, 3, 1); Russian roulette after 3 scatters.  Returns (scene,
    camera, tracer keyword arguments)."""
    scene = Scene(background=0.0)
    scene.add_solid(prism_planes(60.0, 1.0, 1.0), Dielectric(SF11))
    scene.add_solid([((0.0, 1.0, 0.0), 0.6)], Lambertian(0.8))
    cam = Camera.look_at((0.5, 1.5, 5.0), (0.0, -0.3, 0.0), (0.0, 1.0, 0.0), 45.0, width / height)
    return scene, cam, dict(emitter=((2.0, 3.0, 1.0), 0.2, 40.0), rr_start=3, max_depth=8)


def rainbow_workload(width=1920, height=1080, beam_width=2.2):
    """Water sphere r=1 at the origin; photons travel +x; camera on the sun
    side, off axis, so the backward primary/secondary bows cross the frame."""
    scene = Scene(background=0.0)
    scene.add_sphere((0.0, 0.0, 0.0), 1.0, Dielectric(WATER))
    h = beam_width / 2.0
    beam = Beam((-3.0, -h, -h), (0.0, 0.0, beam_width), (0.0, beam_width, 0.0), (1.0, 0.0, 0.0))
    cam = Camera.look_at((-7.0, 1.0, 2.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 60.0, width / height)
    return scene, beam, cam


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


def random_prism_jobs(n_jobs=256, seed=0xB200, bins=32, photons=(2 ** 14, 2 ** 22), side=(128, 1024),
                      lambda_min=380.0, lambda_max=780.0):
    """List of dicts describing the uneven batch (one per scene)."""
    jobs = []
    for j in range(n_jobs):
        g = Pcg(j, seed)
        glass = (BK7, SF11, FUSED_SILICA)[g.u32() % 3]
        apex = g.uniform(30.0, 75.0)
        inc = g.uniform(30.0, 60.0)
        n = int(round(g.log_uniform(*photons)))
        s = int(round(g.log_uniform(*side)))
        sigma_s = g.uniform(0.01, 0.1)
        jobs.append(dict(glass=glass, apex_deg=apex, incidence_deg=inc, n_photons=n, width=s, height=s,
                         sigma_s=sigma_s, sigma_t=sigma_s, g=0.0, seed=(seed * 2654435761 + j) & 0xFFFFFFFF,
                         bins=bins, lambda_min=lambda_min, lambda_max=lambda_max))
    return jobs
