"""GPU films against the CPU oracle at the sizes the benchmarks run.

The other parity tests use small films; these run the benchmarked shapes:
  * the single-prism pass at full size: 2^20 photons into a 640x360x64-bin film;
  * the rainbow's 1920x1080x64-bin film (1.06 GB, larger than L2, so the launch
    takes the wavelength-ordered dispatch) on a 2^22-photon prefix;
  * the whole 256-scene uneven batch (17.3 GB film arena: cell offsets beyond
    2^31), every scene on the prefix of its first 2^16 photons;
  * a batch film with more tiles than a warp's shared-memory mask holds, whose
    tiles are marked straight in the global mask.
Films must be within FILM_TOL relative L1 of the oracle (the 0.5 % bar);
spectral films are compared cell by cell, batch images through the sensor
reduction (the oracle's spectral film times the bin-averaged CMF).
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

import oracle
import spectral_b200 as sb
from spectral_b200.batch import Batch, prism_jobs
from spectral_b200.scenes import prism_workload, rainbow_workload

from helpers import obeam, ocam, oracle_job_xyz, oscene

pytestmark = pytest.mark.gpu

FILM_TOL = 5e-3
THREADS = max(1, min(16, os.cpu_count() or 1))


def int_rel_l1(a, b):
    """Relative L1 of two int64 films without float copies of the whole film."""
    a = a.reshape(-1)
    b = b.reshape(-1)
    num = den = 0
    for i in range(0, a.size, 1 << 24):
        x, y = a[i:i + (1 << 24)], b[i:i + (1 << 24)]
        num += int(np.abs(x - y).sum())
        den += int(np.abs(y).sum())
    return num / den if den else 0.0


def _spectral_case(ctx, scene, beam, cam, w, h, bins, n, seed, sig, max_dist, max_bounces, threads):
    film = sb.GpuPhotonFilm(ctx, scene, cam, beam, w, h, n, seed, max_dist, sb.VolWeights(sig, sig, 0.0), bins=bins,
                            lambda_min=380.0, lambda_max=780.0, max_bounces=max_bounces)
    film.dispatch_photons(0, n, seed)
    raw = film.read_raw()
    film.close()
    p = oracle.vol_params(w, h, seed, sig, sig, 0.0, max_dist, max_bounces, 380.0, 780.0, bins=bins)
    _, _, fs = oracle.render_point(oscene(scene), ocam(cam), obeam(beam), p, 0, n, f32=False, xyz=False, spec=True,
                                   threads=threads)
    return raw, fs.reshape(h, w, bins)


def test_prism_pass_full_size(ctx):
    """Config 1 as benchmarked: SF11 prism, 2^20 photons, 640x360x64 bins."""
    w, h, n = 640, 360, 1 << 20
    scene, beam, cam = prism_workload(w, h)
    raw, ref = _spectral_case(ctx, scene, beam, cam, w, h, 64, n, 0xDED, 0.05, 6.0, 8, THREADS)
    l1 = int_rel_l1(raw, ref)
    print("prism 640x360x64, 2^20 photons: film rel L1 %.3e" % l1)
    assert ref.sum() > 0 and l1 < FILM_TOL


def test_rainbow_film_ordered_dispatch_prefix(ctx):
    """Config 3's 1920x1080x64 film (1.06 GB) on photons [0, 2^22): the
    launch sorts its photons by film bin first, as at full size."""
    w, h, n = 1920, 1080, 1 << 22
    scene, beam, cam = rainbow_workload(w, h)
    raw, ref = _spectral_case(ctx, scene, beam, cam, w, h, 64, n, 0x8A1B, 0.02, 8.0, 6, min(THREADS, 4))
    l1 = int_rel_l1(raw, ref)
    print("rainbow 1920x1080x64, 2^22 photons: film rel L1 %.3e" % l1)
    assert ref.sum() > 0 and l1 < FILM_TOL


def _batch_vs_oracle(ctx, jobs):
    b = Batch(ctx, jobs)
    b.run()
    got = [b.read_xyz(i) for i in range(len(jobs))]
    b.close()
    with cf.ThreadPoolExecutor(THREADS) as ex:  # the oracle releases the GIL
        refs = list(ex.map(oracle_job_xyz, list(jobs)))
    out = []
    for g, r in zip(got, refs):
        den = float(np.abs(r).sum())
        out.append((float(np.abs(g.astype(np.float64) - r).sum() / den) if den > 0 else 0.0, den))
    return out


def test_full_uneven_batch_every_scene_on_a_prefix(ctx):
    """All 256 scenes of the benchmarked batch with their film sizes (the same
    17.3 GB arena), each traced on photons [0, 2^16) of its own stream."""
    from spectral_b200.specs import random_prism_jobs
    specs = random_prism_jobs(256, seed=0xB200, bins=32, lambda_min=380.0, lambda_max=780.0)
    for s in specs:
        s["n_photons"] = min(s["n_photons"], 1 << 16)
    jobs = prism_jobs(specs)
    cells = sum(((j.width + 7) // 8) * ((j.height + 7) // 8) * 64 * j.opts.bins for j in jobs)
    assert cells > 2 ** 31  # film offsets past 2^31 cells
    res = _batch_vs_oracle(ctx, jobs)
    worst = max(r[0] for r in res)
    total = sum(r[0] * r[1] for r in res) / sum(r[1] for r in res)
    print("256-scene batch, 2^16-photon prefixes: worst scene rel L1 %.3e, all scenes %.3e" % (worst, total))
    assert all(r[1] > 0 for r in res) and worst < FILM_TOL


def test_batch_film_beyond_the_shared_mask(ctx):
    """A film of 1100x1100 pixels has 19,044 tiles (596 mask words, more than
    the 512 a warp keeps in shared memory): its tiles are marked straight in
    the global mask, and the drain must still read every lit tile."""
    from spectral_b200.specs import random_prism_jobs
    specs = random_prism_jobs(3, seed=0xB17, bins=16, photons=(2 ** 15, 2 ** 16), side=(200, 300))
    specs[1]["width"] = specs[1]["height"] = 1100
    res = _batch_vs_oracle(ctx, prism_jobs(specs))
    print("batch with a 1100x1100 film: rel L1 %s" % [round(r[0], 9) for r in res])
    assert all(r[1] > 0 and r[0] < FILM_TOL for r in res)
