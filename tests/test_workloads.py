"""The seeded synthetic workloads have the shapes the benchmark configurations
name (checked on CPU): the uneven batch's scene distribution, the serving
stream's arrivals, sessions and budgets, and the single-scene workloads."""
import math

import numpy as np

import bench
from spectral_b200.scenes import random_prism_jobs
from spectral_b200.serve import poisson_requests


def test_uneven_batch_distribution():
    jobs = random_prism_jobs()
    assert len(jobs) == 256
    assert {j["glass"] for j in jobs} == {0, 1, 3}  # BK7, SF11, fused silica
    ap = np.array([j["apex_deg"] for j in jobs])
    inc = np.array([j["incidence_deg"] for j in jobs])
    assert 30.0 <= ap.min() and ap.max() <= 75.0 and 30.0 <= inc.min() and inc.max() <= 60.0
    n = np.array([j["n_photons"] for j in jobs], np.float64)
    side = np.array([j["width"] for j in jobs], np.float64)
    assert 2 ** 14 <= n.min() and n.max() <= 2 ** 22 and 128 <= side.min() and side.max() <= 1024
    # log-uniform: the logs spread evenly (mean near the middle of the log range)
    assert abs(np.log2(n).mean() - 18.0) < 0.5 and abs(np.log2(side).mean() - 8.5) < 0.3
    assert all(j["width"] == j["height"] and j["bins"] == 32 for j in jobs)
    s = np.array([j["sigma_s"] for j in jobs])
    assert 0.01 <= s.min() and s.max() <= 0.1
    assert random_prism_jobs() == jobs  # seeded


def test_serving_stream_shape():
    reqs = poisson_requests(200.0, 60.0)
    arrivals = np.array([r[0] for r in reqs])
    assert abs(len(reqs) / 60.0 - 200.0) < 10.0 and np.all(np.diff(arrivals) > 0)
    gaps = np.diff(arrivals)
    assert abs(gaps.mean() - 1 / 200.0) < 1e-4 and abs(gaps.std() / gaps.mean() - 1.0) < 0.05  # exponential
    sess = [r for r in reqs if r[2] > 1]
    assert abs(len(sess) / len(reqs) - 0.3) < 0.03
    assert all(16 <= r[2] <= 128 and r[3] == 2.0 for r in sess)
    n = np.array([r[1].n_photons for r in reqs], np.float64)
    assert 2 ** 16 <= n.min() and n.max() <= 2 ** 20
    assert bench.SERVE["rate"] == 200.0 and bench.SERVE["budget_gb"] == 40.0


def test_single_scene_workloads():
    p, r = bench.WORKLOADS["prism"], bench.WORKLOADS["rainbow"]
    assert (p["width"], p["height"], p["bins"], p["photons"]) == (640, 360, 64, 2 ** 20)
    assert p["sigma_s"] == 0.05 and p["sigma_t"] == 0.05 and p["g"] == 0.0  # sigma_a 0, isotropic
    assert (p["lambda_min"], p["lambda_max"]) == (380.0, 780.0)
    assert (r["width"], r["height"], r["bins"], r["photons"]) == (1920, 1080, 64, 2 ** 26)
    assert r["sigma_s"] == 0.02 and r["max_bounces"] == 6  # up to 4 internal bounces
    t = bench.TRACER
    assert (t["width"], t["height"], t["spp"]) == (1280, 720, 64)
    assert math.isclose(bench.BATCH["lambda_max"], 780.0) and bench.BATCH["bins"] == 32
