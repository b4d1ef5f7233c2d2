"""Sensitivity of the parity gates (the reference's README claims its gates
were mutation-tested by hand).  Each fault below is planted in the CPU oracle,
never in the product, and at least one gate that the GPU tests apply must
reject the faulty oracle's output against the committed fixtures: the golden
RNG draws (bit-identical), the per-photon states of the DSOTM and TIR beams
(exact bounce count and wavelength, origin / direction within 1e-6) or the
point-estimator image (0.5 % relative L1).  The fault-free oracle passes all."""
import importlib.util
import json
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
PATH_TOL, FILM_TOL = 1e-6, 5e-3
FAULTS = {1: "PCG multiplier", 2: "Sellmeier index + 2e-4", 3: "Fresnel without its p term",
          4: "haze weight without the 1/4", 5: "HG phase with g negated"}


def _make_golden():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _gates():
    """(rng, paths, film) gate results of the oracle as it stands."""
    import ctypes as C
    draws = (C.c_uint32 * 16)()
    oracle.lib.or_rng_draws_u32(0xABCD, 0x1234, 16, draws)
    rng_ok = list(draws) == json.load(open(os.path.join(GOLDEN, "rng_draws.json")))["key_0xABCD_seed_0x1234"]
    scene, beam, tir = _make_golden().dsotm()
    g = np.load(os.path.join(GOLDEN, "dsotm_photons.npz"))
    p = oracle.vol_params(256, 256, 42, max_dist=14.0)
    paths_ok = True
    for name, b in (("dsotm", beam), ("tir", tir)):
        for i in range(64):
            k, lam, st, _ = oracle.simulate_photon(scene, b, p, i)
            kk = int(g[name + "_num_states"][i])
            if k != kk or np.float32(lam) != g[name + "_lambda"][i]:
                paths_ok = False
                break
            m = min(k, 9)
            if np.abs(st[:m] - g[name + "_states"][i][:m]).max() > PATH_TOL:
                paths_ok = False
                break
    cam = oracle.camera_look_at((0.5, -0.5, 12.0), (0.5, -0.5, 0.0), (0, 1, 0), 42.0, 1.0)
    img, _, _ = oracle.render_point(scene, cam, beam, oracle.vol_params(64, 64, 7, 0.5, 0.06, 0.5, 14.0), 0, 4096)
    ref = np.load(os.path.join(GOLDEN, "dsotm_film_64.npz"))["img_f32"].astype(np.float64)
    film_ok = np.abs(img.astype(np.float64) - ref).sum() / np.abs(ref).sum() < FILM_TOL
    return rng_ok, paths_ok, film_ok


def test_fault_free_oracle_passes_every_gate():
    assert _gates() == (True, True, True)


@pytest.mark.parametrize("fault", sorted(FAULTS))
def test_each_planted_fault_is_caught(fault):
    oracle.lib.or_set_fault(fault)
    try:
        gates = _gates()
    finally:
        oracle.lib.or_set_fault(0)
    assert not all(gates), "%s passed every gate %s" % (FAULTS[fault], gates)
