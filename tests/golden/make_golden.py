"""Regenerate the committed golden fixtures in this directory from the CPU oracle.

    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py --extra    # the beam and tracer fixtures only

* rng_draws.json: 16 draws of PathRng(0xABCD, 0x1234) (the stream of
  spectral-gpu/tests/rng_parity.rs; its first four are the reference's frozen
  values, spectral-core/src/rng.rs:82) plus f32 draws for a few keys.
* dsotm_photons.npz: per-photon (origin, dir) states, wavelength and bounce
  count for photons 0..63 of the DSOTM beam and of the TIR beam, seed 42
  (spectral-gpu/src/vol_photons.rs:1280-1414).
* dsotm_film_64.npz: the 64x64 XYZ fixed-point film (scale 2^32) of 4096 DSOTM
  photons, seed 7, DSOTM weights (spectral-gpu/src/vol_photons.rs:1425-1458).
* beam_film_48x40.npz: the photon-beam estimator image (render_volumetric_scene,
  spectral-core/src/volume.rs:233-329) of 600 DSOTM photons, seed 3, 48x40.
* tracer_glass_32x24.npz: the camera tracer's mean XYZ image (CpuTracer,
  spectral-core/src/tracer.rs:44-141) of two dielectric spheres under a
  horizon, 32x24, 8 spp, seed 77, D65.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
import ctypes as C  # noqa: E402


def dsotm():
    from oracle import F3
    bdir = np.array([0.84, 0.54, 0.0], np.float32)
    ln = np.sqrt(bdir[0] * bdir[0] + bdir[1] * bdir[1] + bdir[2] * bdir[2], dtype=np.float32)
    bdir = bdir * (np.float32(1.0) / ln)
    bp = np.array([-0.54, 0.84, 0.0], np.float32)
    ln = np.sqrt(bp[0] * bp[0] + bp[1] * bp[1] + bp[2] * bp[2], dtype=np.float32)
    bp = bp * (np.float32(1.0) / ln) * np.float32(0.05)
    beam = oracle.or_beam(F3(-2.6, -0.95, -0.6), F3(0, 0, 1.2), F3(*bp), F3(*bdir))
    td = np.array([0.934, 0.358, 0.0], np.float32)
    ln = np.sqrt(td[0] * td[0] + td[1] * td[1] + td[2] * td[2], dtype=np.float32)
    td = td * (np.float32(1.0) / ln)
    tp = np.array([-0.358, 0.934, 0.0], np.float32)
    ln = np.sqrt(tp[0] * tp[0] + tp[1] * tp[1] + tp[2] * tp[2], dtype=np.float32)
    tp = tp * (np.float32(1.0) / ln) * np.float32(0.6)
    tir = oracle.or_beam(F3(-3.0, -1.1, -0.6), F3(0, 0, 1.2), F3(*tp), F3(*td))
    planes = [(-0.8660254, 0.5, 0.0, -0.9), (0.8660254, 0.5, 0.0, -0.9), (0, -1, 0, -1.0), (0, 0, 1, -1.0),
              (0, 0, -1, -1.0)]
    pb = b"".join(bytes(oracle.or_plane(F3(a, b, c), d)) for a, b, c, d in planes)
    prim = bytes(oracle.or_prim(F3(0, 0, 0), 0.0, 0, 5, 1, 0))
    mat = bytes(oracle.or_mat(0.0, 1, 1, 0))
    scene = oracle.OScene(prim, 1, pb, 5, mat, 1, 0.0)
    return scene, beam, tir


def glass_spheres():
    """SF11 sphere r=1 at (0, 0, -3) and water sphere r=0.7 at (1.8, 0.5, -4),
    background 1, horizon 2; camera at (0, 0.3, 0.5) looking at (0, 0, -3)."""
    from oracle import F3
    prims = bytes(oracle.or_prim(F3(0, 0, -3), 1.0, 0, 0, 0, 0)) + bytes(oracle.or_prim(F3(1.8, 0.5, -4), 0.7, 0, 0, 0, 1))
    mats = bytes(oracle.or_mat(0.0, 1, 1, 0)) + bytes(oracle.or_mat(0.0, 2, 1, 0))
    scene = oracle.OScene(prims, 2, b"", 0, mats, 2, 1.0, 2.0)
    cam = oracle.camera_look_at((0.0, 0.3, 0.5), (0.0, 0.0, -3.0), (0, 1, 0), 55.0, 32.0 / 24.0)
    return scene, cam


def extra_fixtures():
    """The beam-estimator and camera-tracer fixtures (written by themselves so
    that the older fixtures are not rewritten)."""
    scene, beam, _ = dsotm()
    cam = oracle.camera_look_at((0.5, -0.5, 12.0), (0.5, -0.5, 0.0), (0, 1, 0), 42.0, 48.0 / 40.0)
    p = oracle.vol_params(48, 40, 3, 0.5, 0.06, 0.5, 14.0)
    img = oracle.render_beam(scene, cam, beam, p, 0, 600)
    np.savez_compressed(os.path.join(HERE, "beam_film_48x40.npz"), img_f32=img)
    gs, gcam = glass_spheres()
    acc = oracle.tracer_accumulate(gs, gcam, 32, 24, 0, 77, 8)
    np.savez_compressed(os.path.join(HERE, "tracer_glass_32x24.npz"), mean_xyz=acc / np.float32(8))


def main():
    out = {}
    d = (C.c_uint32 * 16)()
    oracle.lib.or_rng_draws_u32(0xABCD, 0x1234, 16, d)
    out["key_0xABCD_seed_0x1234"] = list(d)
    for key, seed in [(0, 0), (7, 12345), (4294967295, 42)]:
        f = np.zeros(8, np.float32)
        oracle.lib.or_rng_draws_f32(key, seed, 8, oracle.fp(f))
        out["f32_key_%d_seed_%d" % (key, seed)] = [float(x) for x in f]
    json.dump(out, open(os.path.join(HERE, "rng_draws.json"), "w"), indent=1)

    scene, beam, tir = dsotm()
    p = oracle.vol_params(256, 256, 42, max_dist=14.0)
    arrays = {}
    for name, b in [("dsotm", beam), ("tir", tir)]:
        n = np.zeros(64, np.uint32)
        lam = np.zeros(64, np.float32)
        st = np.zeros((64, 9, 2, 4), np.float32)
        for i in range(64):
            k, l, s, _ = oracle.simulate_photon(scene, b, p, i)
            n[i], lam[i], st[i] = k, l, s
        arrays[name + "_num_states"] = n
        arrays[name + "_lambda"] = lam
        arrays[name + "_states"] = st
    np.savez_compressed(os.path.join(HERE, "dsotm_photons.npz"), **arrays)

    cam = oracle.camera_look_at((0.5, -0.5, 12.0), (0.5, -0.5, 0.0), (0, 1, 0), 42.0, 1.0)
    p = oracle.vol_params(64, 64, 7, 0.5, 0.06, 0.5, 14.0)
    img, fx, _ = oracle.render_point(scene, cam, beam, p, 0, 4096)
    np.savez_compressed(os.path.join(HERE, "dsotm_film_64.npz"), film_xyz=fx, img_f32=img)
    extra_fixtures()
    print("wrote golden fixtures to", HERE)


if __name__ == "__main__":
    if sys.argv[1:] == ["--extra"]:
        extra_fixtures()
    else:
        main()
