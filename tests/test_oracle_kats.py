"""Pins the CPU oracle to the reference renderer's own unit tests and
known-answer values (spectral-core/src/*.rs #[cfg(test)], spectral-core/tests/,
spectral-gpu/tests/, spectral-gpu/src/*.rs tests).  CPU only."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle
from oracle import F3, fp, lib as O

from helpers import axis_box, triangular_prism, wedge

FROZEN_DRAWS = [0xA1DD5847, 0x13248A2D, 0x37278DEF, 0xDE1D5B62]  # spectral-core/src/rng.rs:82


def draws_u32(key, seed, n):
    out = (C.c_uint32 * n)()
    O.or_rng_draws_u32(key, seed, n, out)
    return list(out)


def draws_f32(key, seed, n):
    out = np.zeros(n, np.float32)
    O.or_rng_draws_f32(key, seed, n, fp(out))
    return out


# ---- rng.rs:46-82, spectral-gpu/tests/rng_parity.rs ------------------------
def test_rng_frozen_draws():
    assert draws_u32(0xABCD, 0x1234, 4) == FROZEN_DRAWS


def test_rng_same_key_same_sequence():
    a, b = draws_f32(7, 12345, 16), draws_f32(7, 12345, 16)
    assert a.tobytes() == b.tobytes()


def test_rng_different_key_different_sequence():
    assert draws_f32(7, 12345, 4).tobytes() != draws_f32(8, 12345, 4).tobytes()


def test_rng_floats_in_unit_interval():
    x = draws_f32(1, 2, 1000)
    assert (x >= 0).all() and (x < 1).all()


def test_rng_golden_sixteen(tmp_path):
    import json, os
    golden = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "rng_draws.json")))
    assert draws_u32(0xABCD, 0x1234, 16) == golden["key_0xABCD_seed_0x1234"]
    assert golden["key_0xABCD_seed_0x1234"][:4] == FROZEN_DRAWS


def test_mix2():
    assert O.or_mix2(5, 9) == O.or_pcg32(5 ^ O.or_pcg32(9))


# ---- sellmeier.rs:136-161, spectral-gpu/tests/f32_budget.rs ------------------
def n(glass, nm):
    return O.or_glass_n(glass, nm)


def test_bk7_matches_published_lines():
    assert abs(n(0, 486.1) - 1.52238) <= 5e-4
    assert abs(n(0, 587.6) - 1.51680) <= 5e-4
    assert abs(n(0, 656.3) - 1.51432) <= 5e-4


def test_dispersion_is_normal_and_sf11_disperses_more():
    assert n(0, 450) > n(0, 650) and n(1, 450) > n(1, 650)
    assert n(1, 450) - n(1, 650) > n(0, 450) - n(0, 650)


def test_water_index():
    assert abs(n(2, 589.0) - 1.333) <= 2e-3
    assert n(2, 450) > n(2, 650)


def test_fused_silica_d_line():
    # Malitson (1965): n_d = 1.4585 at 587.6 nm; n_F - n_C = 0.00676.
    assert abs(n(3, 587.6) - 1.4585) < 2e-4
    assert abs((n(3, 486.1) - n(3, 656.3)) - 0.00676) < 2e-4


def test_f32_sellmeier_budget():
    coeffs = {0: ([1.039_612_2, 0.231_792_35, 1.010_469_4], [0.006_000_698_5, 0.020_017_914, 103.560_65]),
              1: ([1.737_597, 0.313_747_35, 1.898_781_1], [0.013188707, 0.062_306_814, 155.236_3])}
    worst = 0.0
    for g in (0, 1, 2):
        for nm in np.arange(380.0, 730.0 + 1e-3, 5.0, dtype=np.float32):
            l_um = np.float32(nm) / np.float32(1000.0)
            l2 = l_um * l_um
            if g == 2:
                f = np.float32(1.3238) + np.float32(0.00314) / l2
            else:
                b, c = coeffs[g]
                n2 = np.float32(1.0)
                for k in range(3):
                    n2 = n2 + np.float32(b[k]) * l2 / (l2 - np.float32(c[k]))
                f = np.sqrt(n2)
            worst = max(worst, abs(float(f) - n(g, float(nm))))
    assert worst < 1e-4


# ---- cie.rs:151-174, spectral-gpu/src/data.rs:27-35 -------------------------
def test_d65_white_point():
    out = np.zeros(3, np.float32)
    O.or_integrate_illuminant(0, fp(out))
    s = out.sum()
    assert abs(out[0] / s - 0.3127) <= 2e-3 and abs(out[1] / s - 0.3290) <= 2e-3


# ---- core/tests/rayleigh.rs: 1/lambda^4 through the shipped sensor tables ---
def _integrate_d65(weight):
    """sum over 380..730 nm in 5 nm steps of D65 * weight * cmf * 5 (f32, as rayleigh.rs:10-23)."""
    x = y = z = np.float32(0.0)
    c = np.zeros(3, np.float32)
    nm = np.float32(380.0)
    while nm <= np.float32(730.0):
        sv = np.float32(O.or_illuminant(0, float(nm))) * np.float32(weight(nm))
        O.or_cmf(float(nm), fp(c))
        x += sv * c[0] * np.float32(5.0)
        y += sv * c[1] * np.float32(5.0)
        z += sv * c[2] * np.float32(5.0)
        nm += np.float32(5.0)
    xyz = np.array([x, y, z], np.float32)
    rgb = np.zeros(3, np.float32)
    O.or_xyz_to_linear_srgb(fp(xyz), fp(rgb))
    return xyz / xyz.sum(), rgb


def test_scattered_sky_is_blue():
    ch, rgb = _integrate_d65(lambda nm: np.float32(550.0 / nm) ** 4)
    assert ch[0] < 0.28 and ch[1] < 0.33 and rgb[2] > rgb[0]


def test_sunset_transmitted_is_red():
    ch, rgb = _integrate_d65(lambda nm: np.exp(np.float32(-1.5) * np.float32(550.0 / nm) ** 4))
    assert ch[0] > 0.40 and rgb[0] > rgb[2]


# ---- core/tests/scene_b_metamerism.rs:16-66: illuminant-dependent colour ------
def _chroma_under(refl, ill):
    x = y = z = np.float32(0.0)
    c = np.zeros(3, np.float32)
    nm = np.float32(380.0)
    while nm <= np.float32(730.0):
        sv = np.float32(O.or_illuminant(ill, float(nm))) * np.float32(refl(nm))
        O.or_cmf(float(nm), fp(c))
        x += sv * c[0] * np.float32(5.0)
        y += sv * c[1] * np.float32(5.0)
        z += sv * c[2] * np.float32(5.0)
        nm += np.float32(5.0)
    s = x + y + z
    return x / s, y / s


def test_illuminant_swap_changes_color_relationship():
    smooth = lambda nm: 0.5 + 0.3 * math.cos((nm - 555.0) / 120.0)  # noqa: E731
    g = lambda nm, c, w: math.exp(-(((nm - c) / w) ** 2))  # noqa: E731
    bumpy = lambda nm: min(max(0.55 * g(nm, 450, 25) + 0.75 * g(nm, 540, 25) + 0.65 * g(nm, 610, 25), 0.0), 1.0)  # noqa: E731
    assert sum(abs(smooth(n) - bumpy(n)) for n in range(400, 700, 20)) > 0.5

    def gap(ill):
        a, b = _chroma_under(smooth, ill), _chroma_under(bumpy, ill)
        return math.hypot(a[0] - b[0], a[1] - b[1])
    assert abs(gap(1) - gap(0)) > 1e-3  # illuminant A vs D65


def test_cmf_in_band_and_tables():
    c = np.zeros(3, np.float32)
    O.or_cmf(555.0, fp(c))
    assert c[0] >= 0 and c[1] > 0 and c[2] >= 0
    assert O.or_illuminant(0, 555.0) > 0
    t = oracle.tables()
    assert t.size == 355 and np.isfinite(t).all()
    assert abs(t[71 + 35] - 1.0) < 0.05  # ybar(555) ~ 1


def test_cmf_clamps_beyond_table():
    a, b = np.zeros(3, np.float32), np.zeros(3, np.float32)
    O.or_cmf(730.0, fp(a))
    O.or_cmf(780.0, fp(b))
    assert a.tobytes() == b.tobytes()
    O.or_cmf(300.0, fp(b))
    O.or_cmf(380.0, fp(a))
    assert a.tobytes() == b.tobytes()


def test_xyz_to_srgb_white():
    out = np.zeros(3, np.float32)
    O.or_xyz_to_linear_srgb(fp(np.array([0.9505, 1.0, 1.089], np.float32)), fp(out))
    assert np.all(np.abs(out - 1.0) < 1e-2)


# ---- optics.rs:58-190 --------------------------------------------------------
def refract(d, nrm, n1, n2):
    out = np.zeros(3, np.float32)
    ok = O.or_refract(fp(np.array(d, np.float32)), fp(np.array(nrm, np.float32)), n1, n2, fp(out))
    return out if ok else None


def reflect(d, nrm):
    out = np.zeros(3, np.float32)
    O.or_reflect(fp(np.array(d, np.float32)), fp(np.array(nrm, np.float32)), fp(out))
    return out


def unit(v):
    v = np.array(v, np.float64)
    return (v / np.linalg.norm(v)).astype(np.float32)


def test_refract_matches_snell_angle():
    for deg in [5.0, 15.0, 30.0, 45.0, 60.0]:
        th = math.radians(deg)
        t = refract(unit([math.sin(th), -math.cos(th), 0]), [0, 1, 0], 1.0, 1.5)
        got = math.acos(max(-1.0, min(1.0, float(-t[1]))))
        assert abs(got - math.asin(math.sin(th) / 1.5)) < 1e-5 and abs(t[2]) < 1e-6


# ---- core/tests/scene_a_prism.rs:18-47 (analytic gate) ------------------------
def _bk7_deviation(d, lam):
    t = refract(d, [0, 1, 0], 1.0, O.or_glass_n(0, lam))
    c = float(np.clip(np.dot(d.astype(np.float64), t.astype(np.float64)), -1.0, 1.0))
    return math.acos(c)


def test_prism_interface_blue_deviates_more_than_red():
    d = unit([0.5, -0.8660254, 0.0])  # 30 deg incidence
    assert _bk7_deviation(d, 450.0) > _bk7_deviation(d, 650.0)


def test_prism_interface_spread_matches_analytic():
    th = math.radians(30.0)
    d = unit([math.sin(th), -math.cos(th), 0.0])
    for lam in (440.0, 520.0, 600.0, 680.0):
        analytic = th - math.asin(math.sin(th) / O.or_glass_n(0, lam))
        assert abs(_bk7_deviation(d, lam) - analytic) / analytic < 0.03, lam


def test_transmitted_ray_forward_and_tangential_sense():
    th = math.radians(50.0)
    d = unit([math.sin(th), -math.cos(th), 0])
    t = refract(d, [0, 1, 0], 1.0, 1.5)
    assert float(np.dot(t, d)) > 0 and t[1] < 0
    dt = d - np.dot(d, [0, 1, 0]) * np.array([0, 1, 0])
    tt = t - np.dot(t, [0, 1, 0]) * np.array([0, 1, 0])
    assert np.dot(dt, tt) > 0 and abs(1.0 * np.linalg.norm(dt) - 1.5 * np.linalg.norm(tt)) < 1e-5


def test_refraction_is_reversible():
    th = math.radians(35.0)
    d = unit([math.sin(th), -math.cos(th), 0])
    back = refract(refract(d, [0, 1, 0], 1.0, 1.5), [0, 1, 0], 1.5, 1.0)
    assert np.allclose(back, d, atol=1e-5)


def test_tir_past_critical_and_predicates_agree():
    tc = math.asin(1 / 1.5)
    for th, tir in [(tc + 0.05, True), (tc - 0.05, False)]:
        assert (refract(unit([math.sin(th), -math.cos(th), 0]), [0, 1, 0], 1.5, 1.0) is None) == tir
    for deg in [10.0, 30.0, 41.0, 42.0, 50.0, 70.0]:
        th = math.radians(deg)
        d = unit([math.sin(th), -math.cos(th), 0])
        r = O.or_fresnel(abs(float(-d[1])), 1.5, 1.0)
        assert (refract(d, [0, 1, 0], 1.5, 1.0) is not None) == (r < 1.0)


def test_fresnel_normal_grazing_monotonic():
    assert abs(O.or_fresnel(1.0, 1.0, 1.5) - ((1.0 - 1.5) / 2.5) ** 2) < 1e-6
    assert O.or_fresnel(1e-5, 1.0, 1.5) > 0.999
    prev = O.or_fresnel(1.0, 1.0, 1.5)
    for step in range(1, 21):
        r = O.or_fresnel(1.0 - step / 20.0 * 0.999, 1.0, 1.5)
        assert 0.0 <= r <= 1.0 and r >= prev - 1e-6
        prev = r


def test_reflect_is_mirror():
    d = unit([1, -1, 0])
    r = reflect(d, [0, 1, 0])
    assert np.allclose(r, unit([d[0], -d[1], 0]), atol=1e-6)
    d3 = unit([0.4, -0.7, 0.3])
    assert np.allclose(reflect(d3, [0, 1, 0]), [d3[0], -d3[1], d3[2]], atol=1e-6)


# ---- geom.rs:183-286, scene.rs:245-280 ----------------------------------------
def mk_scene(solids=(), spheres=()):
    prims, planes, mats = [], [], []
    for center, radius in spheres:
        prims.append(oracle.or_prim(F3(*center), radius, 0, 0, 0, len(mats)))
        mats.append(oracle.or_mat(0.5, 0, 0, 0))
    for pl in solids:
        start = len(planes)
        for nrm, d in pl:
            planes.append(oracle.or_plane(F3(*nrm), d))
        prims.append(oracle.or_prim(F3(0, 0, 0), 0.0, start, len(pl), 1, len(mats)))
        mats.append(oracle.or_mat(0.0, 1, 1, 0))
    pb = b"".join(bytes(p) for p in prims)
    plb = b"".join(bytes(p) for p in planes)
    mb = b"".join(bytes(m) for m in mats)
    return oracle.OScene(pb, len(prims), plb, len(planes), mb, len(mats), 1.0)


def hit(scene, o, d):
    t, pt, nrm, ff, m = C.c_float(), np.zeros(3, np.float32), np.zeros(3, np.float32), C.c_int(), C.c_uint32()
    ok = O.or_scene_intersect(C.byref(scene.c), F3(*o), F3(*d), C.byref(t), fp(pt), fp(nrm), C.byref(ff), C.byref(m))
    return (t.value, pt, nrm, bool(ff.value)) if ok else None


def test_sphere_hit_and_miss():
    h = hit(mk_scene(spheres=[((0, 0, -5), 1.0)]), (0, 0, 0), (0, 0, -1))
    assert abs(h[0] - 4.0) < 1e-4 and np.allclose(h[2], [0, 0, 1], atol=1e-4)
    assert hit(mk_scene(spheres=[((5, 0, -5), 1.0)]), (0, 0, 0), (0, 0, -1)) is None


def test_convex_box_cases():
    cube = mk_scene(solids=[axis_box((-1, -1, -1), (1, 1, 1))])
    h = hit(cube, (0, 0, 5), (0, 0, -1))
    assert abs(h[0] - 4.0) < 1e-4 and np.allclose(h[2], [0, 0, 1], atol=1e-4) and h[3]
    assert hit(cube, (2, 0, -5), (0, 0, 1)) is None
    assert hit(cube, (-5, 2, 0), (1, 0, 0)) is None
    h = hit(cube, (5, 0, 0), (-1, 0, 0))
    assert abs(h[0] - 4.0) < 1e-4 and np.allclose(h[2], [1, 0, 0], atol=1e-4)
    h = hit(cube, (0, 0, 0), (0, 0, 1))
    assert abs(h[0] - 1.0) < 1e-4 and np.allclose(h[2], [0, 0, -1], atol=1e-4) and not h[3]


def test_prism_axial_and_miss():
    assert len(triangular_prism(2.0, 2.0)) == 5 and len(wedge(30.0, 1.0, 2.0)) == 5
    prism = mk_scene(solids=[triangular_prism(1.0, 2.0)])
    h = hit(prism, (0, 5, 0), (0, -1, 0))
    assert abs(h[0] - 4.0) < 1e-3 and np.allclose(h[2], [0, 1, 0], atol=1e-3)
    assert hit(prism, (5, 5, 0), (0, -1, 0)) is None


def test_scene_picks_nearest_and_empty():
    s = mk_scene(spheres=[((0, 0, -3), 1.0), ((0, 0, -6), 1.0)])
    assert abs(hit(s, (0, 0, 0), (0, 0, -1))[0] - 2.0) < 1e-3
    assert hit(s, (0, 0, 0), (0, 0, 1)) is None
    assert hit(mk_scene(), (0, 0, 0), (0, 0, -1)) is None


# ---- material.rs:94-159 -------------------------------------------------------
def scatter(kind, refl, wo, nrm, ff, nh, key, seed):
    d, w = np.zeros(3, np.float32), C.c_float()
    O.or_scatter(kind, refl, fp(np.array(wo, np.float32)), fp(np.array(nrm, np.float32)), int(ff), nh, key, seed,
                 fp(d), C.byref(w))
    return d, w.value


def test_lambertian_hemisphere():
    for s in range(200):
        d, w = scatter(0, 0.8, [0, -1, 0], [0, 1, 0], True, 1.5, s, 7)
        assert d[1] > 0 and abs(np.linalg.norm(d) - 1) < 1e-5 and 0 <= w <= 1


def test_dielectric_front_face_and_tir():
    th = math.radians(30.0)
    wo = unit([math.sin(th), -math.cos(th), 0])
    nh = n(0, 550.0)
    ent = [scatter(1, 0, wo, [0, 1, 0], True, nh, s, 99)[0].tobytes() for s in range(32)]
    ext = [scatter(1, 0, wo, [0, 1, 0], False, nh, s, 99)[0].tobytes() for s in range(32)]
    assert ent != ext
    th = math.radians(60.0)
    wo = unit([math.sin(th), -math.cos(th), 0])
    for s in range(8):
        d, _ = scatter(1, 0, wo, [0, 1, 0], False, nh, s, 5)
        assert np.allclose(d, reflect(wo, [0, 1, 0]), atol=1e-5)


def test_dielectric_disperses():
    d = unit([0.6, -0.8, 0])
    assert np.linalg.norm(refract(d, [0, 1, 0], 1.0, n(1, 450)) - refract(d, [0, 1, 0], 1.0, n(1, 650))) > 1e-3


# ---- camera.rs:72-111 ----------------------------------------------------------
def ray(cam, s, t):
    o, d = np.zeros(3, np.float32), np.zeros(3, np.float32)
    O.or_camera_primary_ray(C.byref(cam), s, t, fp(o), fp(d))
    return o, d


def test_camera_rays():
    cam = oracle.camera_look_at((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, 1.0)
    assert np.dot(ray(cam, 0.5, 0.5)[1], [0, 0, -1]) > 0.99
    assert np.linalg.norm(ray(cam, 0.5, 0.5)[1] - ray(cam, 0, 0)[1]) > 1e-2
    cam2 = oracle.camera_look_at((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, 1.5)
    for s, t in [(0, 0), (1, 1), (0.3, 0.7)]:
        assert abs(np.linalg.norm(ray(cam2, s, t)[1]) - 1) < 1e-5


def test_project_inverts_primary_ray():
    cam = oracle.camera_look_at((0, 1, 5), (0, 0, 0), (0, 1, 0), 50.0, 1.5)
    for s, t in [(0.5, 0.5), (0.2, 0.7), (0.8, 0.35)]:
        o, d = ray(cam, s, t)
        out = np.zeros(3, np.float32)
        assert O.or_camera_project(C.byref(cam), fp((o + d * np.float32(4.0)).astype(np.float32)), fp(out))
        assert abs(out[0] - s) < 1e-3 and abs(out[1] - t) < 1e-3 and out[2] > 0


# ---- volume.rs:334-395, vol_photons.rs:876-904 --------------------------------
def test_phase_hg():
    assert O.or_phase_hg(0.6, 1.0) > O.or_phase_hg(0.6, -1.0)
    assert abs(O.or_phase_hg(0.0, 0.5) - O.or_phase_hg(0.0, -0.5)) < 1e-6
    for g, c in [(0, .5), (0, -.5), (.5, 1), (.5, -1), (.5, 0), (.9, 1), (.9, -1), (.9, 0), (.6, 1), (-.3, .7)]:
        g, c = np.float32(g), np.float32(c)
        den = np.float32(max(np.float32(1) + g * g - np.float32(2) * g * c, np.float32(1e-6))) ** np.float32(1.5)
        assert abs(O.or_phase_hg(g, c) - (1 - g * g) / (4 * np.pi * den)) < 1e-5


def test_beam_march_steps_cover_segment():
    for seg_len, m in [(0.5, 1), (3.7, 13), (14.0, 2048), (0.001, 5)]:
        ds = np.float32(seg_len) / np.float32(m)
        total = np.float32(0)
        for _ in range(m):
            total = np.float32(total + ds)
        assert abs(total - seg_len) <= seg_len * 1e-4 + 1e-6


def test_beam_and_point_estimators_conserve_energy():
    w, h = 128, 96
    scene = mk_scene()
    beam = oracle.or_beam(F3(-2, 0, 0), F3(0, 0, 0.6), F3(0, 0.4, 0), F3(1, 0, 0))
    cam = oracle.camera_look_at((0, 0.5, 6), (0, 0, 0), (0, 1, 0), 45.0, w / h)
    p = oracle.vol_params(w, h, 7, 0.5, 0.06, 0.4, 12.0)
    zbuf = np.full(w * h, np.inf, np.float32)
    pt, _, _ = oracle.render_point(scene, cam, beam, p, 0, 20000, zbuf=zbuf, xyz=False)
    bm = np.zeros(3 * w * h, np.float32)
    O.or_render_beam(C.byref(scene.c), C.byref(cam), C.byref(beam), C.byref(p), fp(zbuf), 0, 20000, fp(bm))
    yp, yb = pt[1::3].sum(dtype=np.float64), bm[1::3].sum(dtype=np.float64)
    assert yp > 0 and yb > 0 and 0.92 <= yb / yp <= 1.08


# ---- lighttrace.rs:439-476 -----------------------------------------------------
SCREEN = np.array([4, -3, -2, 0, 0, 4, 0, 8, 0], np.float32)


def test_prism_disperses_beam_on_screen():
    beam = oracle.or_beam(F3(-3, -0.05, -0.05), F3(0, 0, 0.1), F3(0, 0.1, 0), F3(1, 0, 0))
    prism, empty = mk_scene(solids=[wedge(30.0, 1.0, 2.0)]), mk_scene()

    def landing(sc, lam):
        out = np.zeros(2, np.float32)
        assert O.or_mean_landing(C.byref(sc.c), fp(SCREEN), C.byref(beam), lam, 256, 1, fp(out)) > 0
        return out

    sep = np.linalg.norm(landing(prism, 450.0) - landing(prism, 650.0))
    sep0 = np.linalg.norm(landing(empty, 450.0) - landing(empty, 650.0))
    assert sep0 < 1e-4 and sep > 0.02


def test_screen_receives_energy():
    beam = oracle.or_beam(F3(-3, -0.05, -0.05), F3(0, 0, 0.1), F3(0, 0.1, 0), F3(1, 0, 0))
    sc = mk_scene(solids=[wedge(30.0, 1.0, 2.0)])
    p = oracle.vol_params(64, 64, 1)
    out = np.zeros(3 * 64 * 64, np.float32)
    O.or_lighttrace(C.byref(sc.c), fp(SCREEN), 64, 64, C.byref(beam), C.byref(p), 100000, fp(out))
    assert out[1::3].max() > 0


# ---- tracer.rs:561-630 ------------------------------------------------------------
def tracer_mean(scene, cam, w, h, spp, seed):
    s = np.zeros(3 * w * h, np.float32)
    O.or_tracer_accumulate_mt(C.byref(scene.c), C.byref(cam), w, h, 0, seed, spp, 0, 8, fp(s), 8)
    return s / np.float32(spp)


def test_tracer_background_integrates_to_d65():
    sc = mk_scene()
    cam = oracle.camera_look_at((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, 1.0)
    m = tracer_mean(sc, cam, 32, 32, 256, 7)
    tot = np.array([m[0::3].sum(), m[1::3].sum(), m[2::3].sum()], np.float64)
    x, y = tot[0] / tot.sum(), tot[1] / tot.sum()
    assert abs(x - 0.3127) < 6e-3 and abs(y - 0.3290) < 6e-3


def test_tracer_dispersion_collapse_preserves_brightness():
    cam = oracle.camera_look_at((0, 0, 3), (0, 0, 0), (0, 1, 0), 18.0, 1.0)
    y0 = tracer_mean(mk_scene(), cam, 8, 8, 256, 3)[1::3].mean()
    slab = mk_scene(solids=[axis_box((-5, -5, -0.1), (5, 5, 0.1))])
    slab._m[0].glass = 0  # BK7
    y1 = tracer_mean(slab, cam, 8, 8, 256, 3)[1::3].mean()
    assert y0 > 0 and 0.7 * y0 < y1 < 1.05 * y0


def test_tracer_accumulate_positive():
    sc = mk_scene(spheres=[((0, 0, -3), 1.0)])
    sc._m[0].reflectance = 0.8
    cam = oracle.camera_look_at((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, 1.0)
    assert tracer_mean(sc, cam, 16, 16, 4, 42)[1::3].sum() > 0


# ---- spectral-core/tests/raindrop.rs ----------------------------------------------
def deviation_deg(b, lam, bounces):
    nw = n(2, lam)
    sph = mk_scene(spheres=[((0, 0, 0), 1.0)])
    o, d = np.array([-3.0, b, 0.0], np.float32), np.array([1.0, 0, 0], np.float32)
    dirs = [d]
    h = hit(sph, o, d)
    if h is None:
        return None
    d = refract(d, h[2], 1.0, nw)
    if d is None:
        return None
    o = h[1]
    dirs.append(d)
    for _ in range(bounces):
        h = hit(sph, o, d)
        if h is None:
            return None
        d, o = reflect(d, h[2]), h[1]
        dirs.append(d)
    h = hit(sph, o, d)
    if h is None:
        return None
    out = refract(d, h[2], nw, 1.0)
    if out is None:
        return None
    dirs.append(out)
    tot = 0.0
    for a, c in zip(dirs, dirs[1:]):
        tot += abs(math.degrees(math.atan2(a[0] * c[1] - a[1] * c[0], a[0] * c[0] + a[1] * c[1])))
    return tot


def min_dev(lam, bounces):
    best = float("inf")
    for i in range(1, 1000, 3):
        dv = deviation_deg(i / 1000 * 0.999, lam, bounces)
        if dv is not None:
            best = min(best, dv)
    return best


def test_primary_rainbow_42_and_red_outside():
    assert abs((180 - min_dev(550, 1)) - 42.0) < 2.0
    assert 180 - min_dev(650, 1) > 180 - min_dev(450, 1)


def test_secondary_rainbow_51_reversed():
    assert abs((min_dev(550, 2) - 180) - 51.0) < 3.0
    assert min_dev(450, 2) - 180 > min_dev(650, 2) - 180


# ---- spectral-gpu/src/vol_photons.rs:1108-1166 (CPU parity evidence) ---------------
def dsotm_oracle_scene():
    k = 0.9
    planes = [((-0.8660254, 0.5, 0.0), -k), ((0.8660254, 0.5, 0.0), -k), ((0, -1, 0), -1.0), ((0, 0, 1), -1.0),
              ((0, 0, -1), -1.0)]
    return mk_scene(solids=[planes])


def test_forward_parity_tir_boundary_detected():
    sc = dsotm_oracle_scene()
    bdir = unit([0.84, 0.54, 0.0])
    bperp = unit([-0.54, 0.84, 0.0]) * np.float32(0.05)
    beam = oracle.or_beam(F3(-2.6, -0.95, -0.6), F3(0, 0, 1.2), F3(*bperp), F3(*bdir))
    p = oracle.vol_params(256, 256, 42, max_dist=14.0)
    st = np.zeros(72, np.float32)
    found = None
    for idx in range(5000):
        nv = O.or_simulate_photon_fixed(C.byref(sc.c), C.byref(beam), C.byref(p), idx, 400.0, 9, fp(st))
        nr = O.or_simulate_photon_fixed(C.byref(sc.c), C.byref(beam), C.byref(p), idx, 680.0, 9, fp(st))
        if nv != nr:
            found = idx
            break
    assert found is not None


def test_film_resolve_arithmetic():
    # film.rs:337-372: u32 x4096 -> f32 accum.
    raw = np.zeros(3 * 32 * 32, np.uint32)
    raw[[0, 1, 2, 15, 16, 17]] = [4096, 2048, 1024, 2048, 6144, 0]
    acc = raw.astype(np.float32) / np.float32(4096.0)
    assert np.allclose(acc[[0, 1, 2, 15, 16, 17]], [1.0, 0.5, 0.25, 0.5, 1.5, 0.0], atol=1 / 4096)


def test_synthetic_splat_deterministic_and_nonzero():
    a = np.zeros(3 * 32 * 32, np.uint32)
    b = np.zeros(3 * 32 * 32, np.uint32)
    O.or_synthetic_splat(32, 32, 0xDEADBEEF, 4096, a.ctypes.data_as(C.POINTER(C.c_uint32)))
    O.or_synthetic_splat(32, 32, 0xDEADBEEF, 4096, b.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert (a == b).all() and (a > 0).any()


# ---- committed fixtures of the beam estimator and the camera tracer ----------
def test_oracle_reproduces_beam_and_tracer_fixtures():
    import importlib.util
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(here, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    scene, beam, _ = mg.dsotm()
    cam = oracle.camera_look_at((0.5, -0.5, 12.0), (0.5, -0.5, 0.0), (0, 1, 0), 42.0, 1.2)
    img = oracle.render_beam(scene, cam, beam, oracle.vol_params(48, 40, 3, 0.5, 0.06, 0.5, 14.0), 0, 600)
    assert img.tobytes() == np.load(os.path.join(here, "beam_film_48x40.npz"))["img_f32"].tobytes()
    gs, gcam = mg.glass_spheres()
    acc = oracle.tracer_accumulate(gs, gcam, 32, 24, 0, 77, 8) / np.float32(8)
    assert acc.tobytes() == np.load(os.path.join(here, "tracer_glass_32x24.npz"))["mean_xyz"].tobytes()


# ---- free-flight sampling: the same single-scatter integral -------------------
def test_free_flight_and_uniform_point_estimators_agree():
    """Estimator 3 draws each haze distance from sigma_t exp(-sigma_t t) on the
    segment and weights it by 1/pdf; it estimates the same in-scatter as the
    uniform point estimator (volume.rs:130-150).  DSOTM scene with sigma_t 0.3,
    40k photons: total Y within 2 %."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    scene, beam, _ = mg.dsotm()
    cam = oracle.camera_look_at((0.5, -0.5, 12.0), (0.5, -0.5, 0.0), (0, 1, 0), 42.0, 1.0)
    ys = {}
    for est in (0, 3):
        p = oracle.vol_params(96, 96, 5, 0.5, 0.3, 0.5, 14.0, estimator=est)
        img, _, _ = oracle.render_point(scene, cam, beam, p, 0, 40_000)
        ys[est] = img[1::3].astype(np.float64).sum()
    assert ys[0] > 0 and abs(ys[3] / ys[0] - 1.0) < 0.02, ys
