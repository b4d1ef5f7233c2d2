"""Batched uneven workload: one persistent graph-captured launch over many
scenes must give, per scene, exactly the image of a plain per-scene launch,
and match the CPU oracle's spectral film through the sensor reduction."""
import numpy as np
import pytest

import oracle
import spectral_b200 as sb
from spectral_b200 import _lib
from spectral_b200.batch import Batch, prism_job, prism_jobs
from spectral_b200.scenes import random_prism_jobs

from helpers import oracle_job_xyz, rel_l1

pytestmark = pytest.mark.gpu

FAST_TOL = 2e-3  # relative L1 against the oracle: batched films run the fast haze samples


def small_specs(n=12, seed=0x5EED):
    specs = random_prism_jobs(n, seed=seed, photons=(2 ** 10, 2 ** 14), side=(24, 96), bins=16)
    for i, s in enumerate(specs):  # vary the films beyond the defaults
        s["bins"] = (8, 16, 32, 5)[i % 4]
        s["height"] = max(8, s["width"] - 7 * (i % 3))
    return specs


def oracle_xyz(job):
    return oracle_job_xyz(job)


def test_batched_equals_plain_and_oracle(ctx):
    jobs = prism_jobs(small_specs())
    b = Batch(ctx, jobs, chunk_photons=256)
    b.run()
    batched = [b.read_xyz(i) for i in range(len(jobs))]
    b.run_plain()
    plain = [b.read_xyz(i) for i in range(len(jobs))]
    for i in range(len(jobs)):
        assert batched[i].tobytes() == plain[i].tobytes(), i
        exp = oracle_xyz(jobs[i])
        assert exp.sum() > 0 and rel_l1(batched[i], exp) < FAST_TOL, i
    # films were drained: a second pass gives the same images again
    b.run()
    for i in range(len(jobs)):
        assert b.read_xyz(i).tobytes() == batched[i].tobytes()
    assert b.total_photons == sum(j.n_photons for j in jobs)


def test_autotune_and_tunings_agree(ctx):
    jobs = prism_jobs(small_specs(9, seed=77))
    b = Batch(ctx, jobs)
    b.run()
    ref = b.read_all_xyz().copy()
    chosen = b.autotune()
    assert chosen["chunk_photons"] in (512, 2048, 8192) and chosen["minb"] in (4, 5)
    assert chosen["block"] in (128, 256)
    for t in [(64, 4, 0, 0, 0), (1024, 5, 1, 0, 0), (32, 4, 1, 0, 1), (96, 5, 0, 0, 1), (4096, 4, 0, 7, 0),
              (512, 4, 0, 0, 0, 128), (2048, 5, 1, 0, 1, 128), (96, 4, 0, 13, 0, 128)]:
        b.set_tuning(*t)
        b.run()
        assert b.read_all_xyz().tobytes() == ref.tobytes(), t
    st = b.stats()
    assert st["photons"] == b.total_photons and st["in_frame_samples"] > 0 and st["dirty_tiles"] > 0


def test_update_jobs_and_errors(ctx):
    specs = small_specs(4, seed=3)
    jobs = prism_jobs(specs)
    b = Batch(ctx, jobs)
    b.run()
    first = b.read_xyz(0).copy()
    for s in specs:
        s["seed"] ^= 0xABCDEF
    jobs2 = prism_jobs(specs)
    b.update_jobs(jobs2)
    b.run()
    assert b.read_xyz(0).tobytes() != first.tobytes()
    assert rel_l1(b.read_xyz(0), oracle_xyz(jobs2[0])) < FAST_TOL
    specs[1]["width"] += 1
    with pytest.raises(_lib.SpectralError) as e:
        b.update_jobs(prism_jobs(specs))
    assert e.value.code == _lib.SC_E_STATE
    bad = prism_jobs(small_specs(2))
    bad[1].opts.bins = 0
    with pytest.raises(_lib.SpectralError):
        Batch(ctx, bad)
    bad = prism_jobs(small_specs(2))
    bad[0].n_prims = 5
    with pytest.raises(_lib.SpectralError) as e:
        Batch(ctx, bad)
    assert e.value.code == _lib.SC_E_LIMIT


def test_async_readback_overlaps_next_pass(ctx):
    """The asynchronous image copy of pass k runs while pass k+1 traces; the
    next job upload waits for pass k and the next drain for the copy, so each
    buffer holds exactly its own pass's images."""
    import torch
    specs = small_specs(6, seed=21)
    jobs1 = prism_jobs(specs)
    for s in specs:
        s["seed"] ^= 0x5A5A5A
    jobs2 = prism_jobs(specs)
    b = Batch(ctx, jobs1)
    b.run()
    ref1 = b.read_all_xyz().copy()
    b.update_jobs(jobs2)
    b.run()
    ref2 = b.read_all_xyz().copy()
    assert ref1.tobytes() != ref2.tobytes()
    bufs = [torch.empty(b.xyz_floats, dtype=torch.float32, pin_memory=True).numpy() for _ in range(4)]
    for k in range(4):  # back to back, no host wait between passes
        b.update_jobs(jobs1 if k % 2 == 0 else jobs2)
        b.run()
        b.read_all_xyz_async(bufs[k])
    b.synchronize()
    for k in range(4):
        assert bufs[k].tobytes() == (ref1 if k % 2 == 0 else ref2).tobytes(), k


def test_mixed_free_flight_batch_and_variant_switch(ctx):
    """A batch holding a free-flight job (estimator 3) and uniform ones runs the
    kernel built with free-flight sampling; each image equals its plain
    per-scene launch and the oracle.  Switching that job to the uniform
    estimator with update_jobs swaps the kernel (and the captured graph): the
    replayed pass gives the images of a fresh batch of the updated jobs."""
    specs = small_specs(4, seed=0xFF)
    jobs = prism_jobs(specs)
    jobs[1].opts.estimator = 3
    jobs[1].weights.sigma_t = 0.3
    b = Batch(ctx, jobs)
    b.run()
    batched = [b.read_xyz(i) for i in range(len(jobs))]
    b.run_plain()
    for i in range(len(jobs)):
        assert batched[i].tobytes() == b.read_xyz(i).tobytes(), i
        exp = oracle_xyz(jobs[i])
        assert exp.sum() > 0 and rel_l1(batched[i], exp) < FAST_TOL, i
    jobs2 = prism_jobs(specs)
    jobs2[1].weights.sigma_t = 0.3  # the same weights, now the uniform estimator
    b.update_jobs(jobs2)
    b.run()
    switched = [b.read_xyz(i) for i in range(len(jobs2))]
    fresh = Batch(ctx, jobs2)
    fresh.run()
    for i in range(len(jobs2)):
        assert switched[i].tobytes() == fresh.read_xyz(i).tobytes(), i
    assert switched[1].tobytes() != batched[1].tobytes()  # another estimator of the same scene
    assert rel_l1(switched[1], oracle_xyz(jobs2[1])) < FAST_TOL
    fresh.close()
    b.close()
