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

from . import BK7, FUSED_SILICA, SF11, WATER, Beam, Camera, Dielectric, Lambertian, Scene, Screen  # noqa: F401
from . import specs
from .specs import Pcg, prism_planes, random_prism_jobs  # noqa: F401  (re-exported)


def prism_beam(apex_deg, side, incidence_deg, width, back=2.0):
    """Square beam of side `width` aimed at the middle of the left face with
    the given angle of incidence (measured from the face normal)."""
    return Beam(*specs.prism_beam(apex_deg, side, incidence_deg, width, back))


def scene_from_spec(d):
    """Scene of a specs.py scene dict (solids and spheres with their materials)."""
    scene = Scene(background=0.0)

    def mat(m):
        return Dielectric(m[1]) if m[0] == "glass" else Lambertian(m[1])
    for planes, m in d["solids"]:
        scene.add_solid(planes, mat(m))
    for center, radius, m in d["spheres"]:
        scene.add_sphere(center, radius, mat(m))
    return scene


def prism_workload(width=640, height=360, glass=SF11, apex_deg=60.0, side=1.0, incidence_deg=45.0,
                   beam_width=0.02, depth=1.0):
    d = specs.prism_scene(apex_deg, side, incidence_deg, beam_width, depth, glass)
    o, t, up, vfov = d["camera"]
    return scene_from_spec(d), Beam(*d["beam"]), Camera.look_at(o, t, up, vfov, width / height)


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
    d = specs.tracer_scene()
    o, t, up, vfov = d["camera"]
    return scene_from_spec(d), Camera.look_at(o, t, up, vfov, width / height), dict(d["tracer"])


def rainbow_workload(width=1920, height=1080, beam_width=2.2):
    """Water sphere r=1 at the origin; photons travel +x; camera on the sun
    side, off axis, so the backward primary/secondary bows cross the frame."""
    d = specs.rainbow_scene(beam_width)
    o, t, up, vfov = d["camera"]
    return scene_from_spec(d), Beam(*d["beam"]), Camera.look_at(o, t, up, vfov, width / height)
