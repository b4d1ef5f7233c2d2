// Device math shared by every sm_100a kernel of the spectral path.
//
// Transport arithmetic follows the reference renderer's CPU crate operation by
// operation so per-photon paths are bit-identical to it:
//   * f32 with no fused multiply-add (the library is built with -fmad=false),
//     IEEE division and square root (-prec-div/-prec-sqrt, the nvcc default);
//   * glam 0.29 scalar Vec3 order: dot = (x*x + y*y) + z*z, length = sqrt(dot),
//     normalize = v * (1 / length), cross as glam writes it;
//   * Sellmeier index in f64, cast to f32 (spectral-core/src/sellmeier.rs:28-44).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/spectral_cuda.h"

namespace sc {

constexpr int kTableN = 71;          // 5 nm CIE rows, 380..730 nm
constexpr int kTileShift = 3;        // film tiles are 8x8 pixels
constexpr int kTilePixels = 64;

struct f3 { float x, y, z; };
__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
__host__ __device__ __forceinline__ f3 ld3(const float* a) { return mk(a[0], a[1], a[2]); }
__host__ __device__ __forceinline__ f3 add(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ f3 sub(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ f3 mul(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ f3 vdiv(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__host__ __device__ __forceinline__ f3 neg(f3 a) { return mk(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float length(f3 a) { return sqrtf(dot(a, a)); }
__host__ __device__ __forceinline__ f3 normalize(f3 a) { float r = 1.0f / length(a); return mul(a, r); }
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}

// ---- counter-based PCG hash stream (spectral-core/src/rng.rs:7-40) --------
__host__ __device__ __forceinline__ uint32_t pcg32(uint32_t input) {
    uint32_t state = input * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
__host__ __device__ __forceinline__ uint32_t mix2(uint32_t a, uint32_t b) { return pcg32(a ^ pcg32(b)); }
struct Rng {
    uint32_t state;
    __host__ __device__ __forceinline__ static Rng make(uint32_t key, uint32_t seed) { Rng r; r.state = pcg32(key ^ pcg32(seed)); return r; }
    __host__ __device__ __forceinline__ uint32_t u32() { state += 1u; return pcg32(state); }
    __host__ __device__ __forceinline__ float f32() { return (float)(u32() >> 8) * (1.0f / 16777216.0f); }
};

// ---- dispersion: glass 0 BK7, 1 SF11, 2 water (Cauchy), 3 fused silica ----
struct Sellmeier { double b0, b1, b2, c0, c1, c2; };
__host__ __device__ __forceinline__ Sellmeier sellmeier_coef(uint32_t glass) {
    if (glass == 0u) return {1.03961212, 0.231792344, 1.01046945, 0.00600069867, 0.0200179144, 103.560653};
    if (glass == 1u) return {1.73759695, 0.313747346, 1.89878101, 0.013188707, 0.0623068142, 155.23629};
    // Malitson (1965) fused silica
    return {0.6961663, 0.4079426, 0.8974794, 0.0684043 * 0.0684043, 0.1162414 * 0.1162414, 9.896161 * 9.896161};
}

// Glass::n in the reference's operation order: l = nm / 1000, three divided
// terms, sqrt, cast to f32 (spectral-core/src/sellmeier.rs:28-44).
static __host__ __device__ __noinline__ float glass_n_ref(uint32_t glass, float nm) {
    double l_um = (double)nm / 1000.0;
    if (glass == 2u) return (float)(1.3238 + 0.00314 / (l_um * l_um));
    double l2 = l_um * l_um;
    const Sellmeier k = sellmeier_coef(glass);
    double t0 = k.b0 * l2 / (l2 - k.c0);
    double t1 = k.b1 * l2 / (l2 - k.c1);
    double t2 = k.b2 * l2 / (l2 - k.c2);
    return (float)sqrt(1.0 + ((t0 + t1) + t2));
}

// Glass::n with one f64 division instead of four: the three Sellmeier terms
// over a common denominator and nm^2 / 10^6 for the squared wavelength in um.
// This f64 value differs from the reference-order one by a few f64 ulps
// (below 2^-47 for n in [1, 2)).  Both round to the same f32 unless they lie
// within that distance of a rounding midpoint (f +- 2^-24 for n in [1, 2)),
// so the result is accepted only when it is more than 2^-40 away from both
// midpoints and otherwise recomputed in the reference order (about one
// evaluation in 2^16): the returned f32 is always the reference's.
__host__ __device__ __forceinline__ float glass_n(uint32_t glass, float nm) {
    const double x2 = (double)nm * (double)nm;  // exact
    double n;
    if (glass == 2u) {
        n = 1.3238 + 3140.0 / x2;
    } else {
        const Sellmeier k = sellmeier_coef(glass);
        const double l2 = x2 * 1e-6;
        const double d0 = l2 - k.c0, d1 = l2 - k.c1, d2 = l2 - k.c2;
        n = sqrt(1.0 + l2 * ((k.b0 * d1 + k.b1 * d0) * d2 + k.b2 * (d0 * d1)) / ((d0 * d1) * d2));
    }
    const float f = (float)n;
    if (f >= 1.0f && f < 2.0f && fabs(n - (double)f) < 0x1p-24 - 0x1p-40) return f;
    return glass_n_ref(glass, nm);
}

// ---- sensor table lerp, clamped (spectral-core/src/cie.rs:47-61) ----------
__host__ __device__ __forceinline__ float tab_sample(const float* col, float nm) {
    float f = (nm - 380.0f) / 5.0f;
    if (f < 0.0f) f = 0.0f;
    if (f > (float)(kTableN - 1)) f = (float)(kTableN - 1);
    if (f != f) f = 0.0f;
    int i = (int)floorf(f);
    float frac = f - (float)i;
    if (i + 1 >= kTableN) return col[kTableN - 1];
    float a = col[i], b = col[i + 1];
    return a + (b - a) * frac;
}

// ---- optics (spectral-core/src/optics.rs:8-49) ----------------------------
__device__ __forceinline__ f3 reflect3(f3 d, f3 n) { return sub(d, mul(n, 2.0f * dot(d, n))); }
__device__ __forceinline__ bool refract3(f3 d, f3 n, float n1, float n2, f3& out) {
    float eta = n1 / n2;
    f3 nn = n;
    float cos_i = -dot(d, n);
    if (cos_i < 0.0f) { nn = neg(n); cos_i = -cos_i; }
    float k = 1.0f - eta * eta * (1.0f - cos_i * cos_i);
    if (k < 0.0f) return false;
    float cos_t = sqrtf(k);
    out = normalize(add(mul(d, eta), mul(nn, eta * cos_i - cos_t)));
    return true;
}
__device__ __forceinline__ float fresnel(float cos_i, float n1, float n2) {
    cos_i = fminf(fmaxf(cos_i, 0.0f), 1.0f);
    float e = n1 / n2;
    float sin_t2 = e * e * (1.0f - cos_i * cos_i);
    if (sin_t2 >= 1.0f) return 1.0f;
    float cos_t = sqrtf(1.0f - sin_t2);
    float rs = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t);
    float rp = (n1 * cos_t - n2 * cos_i) / (n1 * cos_t + n2 * cos_i);
    return 0.5f * (rs * rs + rp * rp);
}

// ---- scene in shared memory ------------------------------------------------
struct SceneView {
    const sc_primitive* prims;
    const sc_plane* planes;
    const sc_material* mats;
    uint32_t n_prims;
};
struct Hit { float t; f3 point, normal; bool front_face; };

__device__ __forceinline__ bool sphere_hit(const sc_primitive& pr, f3 o, f3 d, float tmin, float tmax, Hit& h) {
    f3 c = ld3(pr.center);
    f3 oc = sub(o, c);
    float a = dot(d, d);
    float half_b = dot(oc, d);
    float cc = dot(oc, oc) - pr.radius * pr.radius;
    float disc = half_b * half_b - a * cc;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float t = (-half_b - sq) / a;
    if (t < tmin || t > tmax) {
        t = (-half_b + sq) / a;
        if (t < tmin || t > tmax) return false;
    }
    f3 p = add(o, mul(d, t));
    f3 outward = vdiv(sub(p, c), pr.radius);
    bool ff = dot(outward, d) < 0.0f;
    h.t = t; h.point = p; h.normal = ff ? outward : neg(outward); h.front_face = ff;
    return true;
}
__device__ __forceinline__ bool solid_hit(const SceneView& S, const sc_primitive& pr, f3 o, f3 d, float tmin, float tmax, Hit& h) {
    float t_enter = -__int_as_float(0x7f800000), t_exit = __int_as_float(0x7f800000);
    f3 en = mk(0.f, 0.f, 0.f), ex = mk(0.f, 0.f, 0.f);
    const uint32_t end = pr.plane_start + pr.plane_count;
    for (uint32_t i = pr.plane_start; i < end; ++i) {
        const sc_plane& pl = S.planes[i];
        f3 n = ld3(pl.normal);
        float denom = dot(n, d);
        float dist = dot(n, o) + pl.d;
        if (fabsf(denom) < 1e-8f) {
            if (dist > 0.0f) return false;
            continue;
        }
        float t = -dist / denom;
        if (denom < 0.0f) { if (t > t_enter) { t_enter = t; en = n; } }
        else { if (t < t_exit) { t_exit = t; ex = n; } }
    }
    if (t_enter > t_exit) return false;
    float th; f3 hn;
    if (t_enter > tmin) { th = t_enter; hn = en; }
    else if (t_exit > tmin) { th = t_exit; hn = ex; }
    else return false;
    if (th > tmax) return false;
    bool ff = dot(hn, d) < 0.0f;
    h.t = th; h.point = add(o, mul(d, th)); h.normal = ff ? hn : neg(hn); h.front_face = ff;
    return true;
}
// Scene::intersect (spectral-core/src/scene.rs:64-78): nearest hit, t_min 1e-3.
__device__ __forceinline__ bool scene_hit(const SceneView& S, f3 o, f3 d, Hit& best, uint32_t& mat) {
    bool any = false;
    float closest = __int_as_float(0x7f800000);
    for (uint32_t i = 0; i < S.n_prims; ++i) {
        const sc_primitive& pr = S.prims[i];
        Hit h;
        bool ok = pr.kind == 0u ? sphere_hit(pr, o, d, 1e-3f, closest, h)
                : (pr.kind == 1u ? solid_hit(S, pr, o, d, 1e-3f, closest, h) : false);
        if (ok) { closest = h.t; best = h; mat = pr.material; any = true; }
    }
    return any;
}

// Material::scatter (spectral-core/src/material.rs:30-82).
__device__ __forceinline__ f3 cosine_hemisphere(f3 n, Rng& r) {
    float u1 = r.f32(), u2 = r.f32();
    float rr = sqrtf(u1);
    float phi = 6.2831855f * u2;
    float x = rr * cosf(phi), y = rr * sinf(phi);
    float z = sqrtf(fmaxf(1.0f - u1, 0.0f));
    f3 a = fabsf(n.x) > 0.9f ? mk(0.f, 1.f, 0.f) : mk(1.f, 0.f, 0.f);
    f3 t = normalize(cross(n, a));
    f3 b = cross(n, t);
    return normalize(add(add(mul(t, x), mul(b, y)), mul(n, z)));
}
__device__ __forceinline__ void scatter(const sc_material& m, f3 wo, const Hit& h, float n_hero, Rng& r, f3& dir, float& w) {
    if (m.kind == 0u) { dir = cosine_hemisphere(h.normal, r); w = m.reflectance; return; }
    float cos_i = fabsf(-dot(wo, h.normal));
    float n1 = h.front_face ? 1.0f : n_hero, n2 = h.front_face ? n_hero : 1.0f;
    float R = fresnel(cos_i, n1, n2);
    w = 1.0f;
    if (r.f32() < R) { dir = reflect3(wo, h.normal); return; }
    f3 t;
    if (refract3(wo, h.normal, n1, n2, t)) dir = t; else dir = reflect3(wo, h.normal);
}

// ---- Camera::project with precomputed basis (spectral-core/src/camera.rs:50-69)
struct Proj { f3 o, u, v, w; float vw, vh; };
__host__ __device__ __forceinline__ Proj proj_make(const sc_camera& c) {
    Proj p; f3 H = ld3(c.horizontal), V = ld3(c.vertical);
    p.o = ld3(c.origin); p.u = normalize(H); p.v = normalize(V); p.vw = length(H); p.vh = length(V);
    p.w = sub(sub(sub(p.o, mul(H, 0.5f)), mul(V, 0.5f)), ld3(c.lower_left));
    return p;
}
__device__ __forceinline__ bool project(const Proj& P, f3 q, float& s, float& t) {
    f3 dir = sub(q, P.o);
    float c = dot(dir, P.w);
    if (c >= -1e-6f) return false;
    s = 0.5f + dot(dir, P.u) / (-c * P.vw);
    t = 0.5f + dot(dir, P.v) / (-c * P.vh);
    return s >= 0.0f && s < 1.0f && t >= 0.0f && t < 1.0f;
}
__device__ __forceinline__ f3 primary_dir(const sc_camera& c, float s, float t) {
    return normalize(sub(add(add(ld3(c.lower_left), mul(ld3(c.horizontal), s)), mul(ld3(c.vertical), t)), ld3(c.origin)));
}

// Henyey-Greenstein phase (spectral-core/src/volume.rs:88-92).
__device__ __forceinline__ float phase_hg(float g, float cos_theta) {
    float g2 = g * g;
    float denom = powf(fmaxf(1.0f + g2 - 2.0f * g * cos_theta, 1e-6f), 1.5f);
    return (1.0f - g2) / (4.0f * 3.14159265358979323846f * denom);
}

// Deterministic round-to-nearest fixed point (never negative, clamped below 2^62).
__device__ __forceinline__ unsigned long long to_fixed(float x, float scale) {
    float y = x * scale;
    if (!(y > 0.0f)) return 0ull;
    // below 2^23 adding 2^23 rounds y to the nearest (even) integer in the
    // mantissa, exactly as the conversion does, with two ALU operations
    if (y < 8388608.0f) return (unsigned long long)(__float_as_uint(y + 8388608.0f) - 0x4B000000u);
    // below 2^31 the 32-bit conversion rounds identically and is cheaper
    if (y < 2147483648.0f) return (unsigned long long)(unsigned)__float2int_rn(y);
    y = fminf(y, 4.0e18f);
    return (unsigned long long)__float2ll_rn(y);
}

// Film layout: 8x8-pixel tiles, tile-major, `channels` int64 per pixel.
__host__ __device__ __forceinline__ uint32_t film_tile(uint32_t px, uint32_t py, uint32_t tiles_x) {
    return (py >> kTileShift) * tiles_x + (px >> kTileShift);
}
// The pixel's index in tile-major order fits 32 bits (every entry point limits
// a film to 2^28 pixels, and beam films to 65535 x 65535: at most 2^26 tiles of
// 64 pixels), so it is formed in 32-bit integer arithmetic and widened once, by
// the multiply with the channel count.
__host__ __device__ __forceinline__ size_t film_cell(uint32_t px, uint32_t py, uint32_t tiles_x, uint32_t channels) {
    const uint32_t local = ((py & 7u) << 3) | (px & 7u);
    return (size_t)((film_tile(px, py, tiles_x) << 6) | local) * channels;
}

}  // namespace sc
