/*
 * CPU oracle: plain-C restatement of the reference renderer's CPU crate.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Every function names the reference
 * file:line it restates (paths relative to the reference checkout).
 * Build: see oracle/Makefile (-O2 -ffp-contract=off, glibc libm).
 */
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* f32 vector algebra with glam 0.29 scalar-Vec3 operation order.            */
/* ------------------------------------------------------------------------ */
typedef struct { float x, y, z; } v3;
static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 L(const float* a) { return V(a[0], a[1], a[2]); }
static inline void S(float* o, v3 a) { o[0] = a.x; o[1] = a.y; o[2] = a.z; }
static inline v3 add(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 vdiv(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static inline v3 neg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float length(v3 a) { return sqrtf(dot(a, a)); }
static inline v3 normalize(v3 a) { float r = 1.0f / length(a); return mul(a, r); }
static inline v3 cross(v3 a, v3 b) {
    return V(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}

/* Planted faults (0 = none), set only by the test that checks that the parity
 * gates catch a wrong restatement: 1 PCG multiplier, 2 Sellmeier index off by
 * 2e-4, 3 Fresnel without its p term, 4 haze weight without the 1/4, 5 HG
 * phase with g negated. */
static int g_fault = 0;
void or_set_fault(int fault) { g_fault = fault; }

/* ------------------------------------------------------------------------ */
/* rng.rs:7-40                                                               */
/* ------------------------------------------------------------------------ */
uint32_t or_pcg32(uint32_t input) {
    uint32_t state = input * (g_fault == 1 ? 747796403u : 747796405u) + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
typedef struct { uint32_t state; } rng_t;
static inline rng_t rng_new(uint32_t key, uint32_t seed) { rng_t r; r.state = or_pcg32(key ^ or_pcg32(seed)); return r; }
static inline uint32_t rng_u32(rng_t* r) { r->state += 1u; return or_pcg32(r->state); }
static inline float rng_f32(rng_t* r) { uint32_t bits = rng_u32(r) >> 8; return (float)bits * (1.0f / 16777216.0f); }
uint32_t or_mix2(uint32_t a, uint32_t b) { return or_pcg32(a ^ or_pcg32(b)); }
void or_rng_draws_u32(uint32_t key, uint32_t seed, uint32_t n, uint32_t* out) {
    rng_t r = rng_new(key, seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = rng_u32(&r);
}
void or_rng_draws_f32(uint32_t key, uint32_t seed, uint32_t n, float* out) {
    rng_t r = rng_new(key, seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = rng_f32(&r);
}

/* ------------------------------------------------------------------------ */
/* sellmeier.rs:13-44.  Glass ids: 0 BK7, 1 SF11, 2 water (Cauchy), 3 fused   */
/* silica (Malitson 1965 Sellmeier; not in the reference crate).             */
/* ------------------------------------------------------------------------ */
static float glass_n_ref(uint32_t glass, float nm);
float or_glass_n(uint32_t glass, float nm) {
    const float n = glass_n_ref(glass, nm);
    return g_fault == 2 ? n + 2e-4f : n;
}
static float glass_n_ref(uint32_t glass, float nm) {
    double l_um = (double)nm / 1000.0;
    if (glass == 2u) return (float)(1.3238 + 0.00314 / (l_um * l_um));
    double l2 = l_um * l_um;
    double b[3], c[3];
    if (glass == 0u) {
        b[0] = 1.03961212; b[1] = 0.231792344; b[2] = 1.01046945;
        c[0] = 0.00600069867; c[1] = 0.0200179144; c[2] = 103.560653;
    } else if (glass == 1u) {
        b[0] = 1.73759695; b[1] = 0.313747346; b[2] = 1.89878101;
        c[0] = 0.013188707; c[1] = 0.0623068142; c[2] = 155.23629;
    } else {
        b[0] = 0.6961663; b[1] = 0.4079426; b[2] = 0.8974794;
        c[0] = 0.0684043 * 0.0684043; c[1] = 0.1162414 * 0.1162414; c[2] = 9.896161 * 9.896161;
    }
    double t0 = b[0] * l2 / (l2 - c[0]);
    double t1 = b[1] * l2 / (l2 - c[1]);
    double t2 = b[2] * l2 / (l2 - c[2]);
    double n2 = 1.0 + ((t0 + t1) + t2);
    return (float)sqrt(n2);
}

void or_glass_n_many(uint32_t glass, const float* nm, size_t n, float* out) {
    for (size_t i = 0; i < n; ++i) out[i] = or_glass_n(glass, nm[i]);
}

/* ------------------------------------------------------------------------ */
/* cie.rs:17-144                                                             */
/* ------------------------------------------------------------------------ */
#define NT 71
static float g_tab[5][NT]; /* xbar, ybar, zbar, d65, a */
static int g_tab_loaded = 0;

int or_load_tables_csv(const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return -1;
    char line[512];
    int row = 0;
    while (fgets(line, sizeof line, f) && row < NT) {
        if (line[0] == '#' || line[0] == 'n' || line[0] == '\n') continue;
        char* p = line;
        (void)strtof(p, &p); /* nm column */
        for (int c = 0; c < 5; ++c) {
            if (*p == ',') ++p;
            g_tab[c][row] = strtof(p, &p); /* correctly rounded decimal -> f32, like str::parse */
        }
        ++row;
    }
    fclose(f);
    if (row != NT) return -2;
    g_tab_loaded = 1;
    return 0;
}
void or_get_tables(float* out) { memcpy(out, g_tab, sizeof g_tab); }

/* Table::sample (cie.rs:47-61): start 380, step 5, 71 rows. */
static inline float tab_sample(int col, float nm) {
    float f = (nm - 380.0f) / 5.0f;
    if (f < 0.0f) f = 0.0f;
    if (f > (float)(NT - 1)) f = (float)(NT - 1);
    if (f != f) f = 0.0f;
    int i = (int)floorf(f);
    float frac = f - (float)i;
    if (i + 1 >= NT) return g_tab[col][NT - 1];
    float a = g_tab[col][i], b = g_tab[col][i + 1];
    return a + (b - a) * frac;
}
void or_cmf(float nm, float out[3]) { for (int c = 0; c < 3; ++c) out[c] = tab_sample(c, nm); }
float or_illuminant(uint32_t which, float nm) { return tab_sample(which == 1u ? 4 : 3, nm); }

void or_integrate_illuminant(uint32_t which, float out[3]) { /* cie.rs:92-106 */
    const float step = 5.0f;
    float x = 0, y = 0, z = 0, k = 0, nm = 380.0f;
    while (nm <= 730.0f) {
        float s = or_illuminant(which, nm), c[3];
        or_cmf(nm, c);
        x += s * c[0] * step; y += s * c[1] * step; z += s * c[2] * step; k += s * c[1] * step;
        nm += step;
    }
    out[0] = x / k; out[1] = y / k; out[2] = z / k;
}
void or_xyz_to_linear_srgb(const float xyz[3], float out[3]) { /* cie.rs:121-128 */
    float x = xyz[0], y = xyz[1], z = xyz[2];
    out[0] = 3.2406f * x - 1.5372f * y - 0.4986f * z;
    out[1] = -0.9689f * x + 1.8758f * y + 0.0415f * z;
    out[2] = 0.0557f * x - 0.2040f * y + 1.0570f * z;
}
void or_tonemap_to_u8(const float lin[3], float exposure, uint8_t out[3]) { /* cie.rs:131-144 */
    for (int c = 0; c < 3; ++c) {
        float v = fmaxf(lin[c] * exposure, 0.0f);
        float mapped = v / (1.0f + v);
        float gm = mapped <= 0.0031308f ? 12.92f * mapped : 1.055f * powf(mapped, 1.0f / 2.4f) - 0.055f;
        gm = fminf(fmaxf(gm, 0.0f), 1.0f);
        float q = gm * 255.0f + 0.5f;
        out[c] = (uint8_t)(q >= 255.0f ? 255.0f : q);
    }
}

/* ------------------------------------------------------------------------ */
/* optics.rs:8-49                                                            */
/* ------------------------------------------------------------------------ */
static inline v3 reflect3(v3 d, v3 n) { return sub(d, mul(n, 2.0f * dot(d, n))); }
static inline int refract3(v3 d, v3 n, float n1, float n2, v3* out) {
    float eta = n1 / n2;
    v3 nn = n;
    float cos_i = -dot(d, n);
    if (cos_i < 0.0f) { nn = neg(n); cos_i = -cos_i; }
    float k = 1.0f - eta * eta * (1.0f - cos_i * cos_i);
    if (k < 0.0f) return 0;
    float cos_t = sqrtf(k);
    *out = normalize(add(mul(d, eta), mul(nn, eta * cos_i - cos_t)));
    return 1;
}
static inline float fresnel(float cos_i, float n1, float n2) {
    cos_i = fminf(fmaxf(cos_i, 0.0f), 1.0f);
    float e = n1 / n2;
    float sin_t2 = e * e * (1.0f - cos_i * cos_i);
    if (sin_t2 >= 1.0f) return 1.0f;
    float cos_t = sqrtf(1.0f - sin_t2);
    float rs = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t);
    float rp = (n1 * cos_t - n2 * cos_i) / (n1 * cos_t + n2 * cos_i);
    return g_fault == 3 ? 0.5f * (rs * rs) : 0.5f * (rs * rs + rp * rp);
}
void or_reflect(const float d[3], const float n[3], float out[3]) { S(out, reflect3(L(d), L(n))); }
int or_refract(const float d[3], const float n[3], float n1, float n2, float out[3]) {
    v3 r; int ok = refract3(L(d), L(n), n1, n2, &r);
    if (ok) S(out, r);
    return ok;
}
float or_fresnel(float cos_i, float n1, float n2) { return fresnel(cos_i, n1, n2); }

/* ------------------------------------------------------------------------ */
/* geom.rs:35-175, scene.rs:64-78                                            */
/* ------------------------------------------------------------------------ */
typedef struct { float t; v3 point, normal; int front_face; } hit_t;

static inline int sphere_hit(const or_prim* pr, v3 o, v3 d, float tmin, float tmax, hit_t* h) {
    v3 c = L(pr->center);
    v3 oc = sub(o, c);
    float a = dot(d, d);
    float half_b = dot(oc, d);
    float cc = dot(oc, oc) - pr->radius * pr->radius;
    float disc = half_b * half_b - a * cc;
    if (disc < 0.0f) return 0;
    float sq = sqrtf(disc);
    float t = (-half_b - sq) / a;
    if (t < tmin || t > tmax) {
        t = (-half_b + sq) / a;
        if (t < tmin || t > tmax) return 0;
    }
    v3 p = add(o, mul(d, t));
    v3 outward = vdiv(sub(p, c), pr->radius);
    int ff = dot(outward, d) < 0.0f;
    h->t = t; h->point = p; h->normal = ff ? outward : neg(outward); h->front_face = ff;
    return 1;
}
static inline int solid_hit(const or_scene* sc, const or_prim* pr, v3 o, v3 d, float tmin, float tmax, hit_t* h) {
    float t_enter = -INFINITY, t_exit = INFINITY;
    v3 en = V(0, 0, 0), ex = V(0, 0, 0);
    for (uint32_t i = pr->plane_start; i < pr->plane_start + pr->plane_count; ++i) {
        const or_plane* pl = &sc->planes[i];
        v3 n = L(pl->normal);
        float denom = dot(n, d);
        float dist = dot(n, o) + pl->d;
        if (fabsf(denom) < 1e-8f) {
            if (dist > 0.0f) return 0;
            continue;
        }
        float t = -dist / denom;
        if (denom < 0.0f) { if (t > t_enter) { t_enter = t; en = n; } }
        else { if (t < t_exit) { t_exit = t; ex = n; } }
    }
    if (t_enter > t_exit) return 0;
    float th; v3 hn;
    if (t_enter > tmin) { th = t_enter; hn = en; }
    else if (t_exit > tmin) { th = t_exit; hn = ex; }
    else return 0;
    if (th > tmax) return 0;
    int ff = dot(hn, d) < 0.0f;
    h->t = th; h->point = add(o, mul(d, th)); h->normal = ff ? hn : neg(hn); h->front_face = ff;
    return 1;
}
static inline int scene_hit(const or_scene* sc, v3 o, v3 d, hit_t* best, uint32_t* mat) {
    int any = 0;
    float closest = INFINITY;
    for (uint32_t i = 0; i < sc->n_prims; ++i) {
        const or_prim* pr = &sc->prims[i];
        hit_t h;
        int ok = pr->kind == 0u ? sphere_hit(pr, o, d, 1e-3f, closest, &h)
               : pr->kind == 1u ? solid_hit(sc, pr, o, d, 1e-3f, closest, &h) : 0;
        if (ok) { closest = h.t; *best = h; *mat = pr->material; any = 1; }
    }
    return any;
}
int or_scene_intersect(const or_scene* sc, const float o[3], const float d[3], float* t,
                       float point[3], float normal[3], int* front_face, uint32_t* mat) {
    hit_t h; uint32_t m = 0;
    if (!scene_hit(sc, L(o), L(d), &h, &m)) return 0;
    *t = h.t; S(point, h.point); S(normal, h.normal); *front_face = h.front_face; *mat = m;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* material.rs:30-82                                                         */
/* ------------------------------------------------------------------------ */
static inline v3 cosine_hemisphere(v3 n, rng_t* r) {
    float u1 = rng_f32(r), u2 = rng_f32(r);
    float rr = sqrtf(u1);
    float phi = 6.2831855f * u2; /* 2.0 * PI in f32 */
    float x = rr * cosf(phi), y = rr * sinf(phi);
    float z = sqrtf(fmaxf(1.0f - u1, 0.0f));
    v3 a = fabsf(n.x) > 0.9f ? V(0, 1, 0) : V(1, 0, 0);
    v3 t = normalize(cross(n, a));
    v3 b = cross(n, t);
    return normalize(add(add(mul(t, x), mul(b, y)), mul(n, z)));
}
/* Returns 1 (material.rs scatter never returns None); *tir set when the
 * refraction branch fell back to reflection. */
static inline int scatter(const or_mat* m, v3 wo, const hit_t* h, float n_hero, rng_t* r, v3* dir, float* w) {
    if (m->kind == 0u) { *dir = cosine_hemisphere(h->normal, r); *w = m->reflectance; return 1; }
    float cos_i = fabsf(-dot(wo, h->normal));
    float n1 = h->front_face ? 1.0f : n_hero, n2 = h->front_face ? n_hero : 1.0f;
    float R = fresnel(cos_i, n1, n2);
    if (rng_f32(r) < R) { *dir = reflect3(wo, h->normal); *w = 1.0f; return 1; }
    v3 t;
    if (refract3(wo, h->normal, n1, n2, &t)) *dir = t; else *dir = reflect3(wo, h->normal);
    *w = 1.0f;
    return 1;
}
static inline float hero_index(const or_mat* m, float lambda, uint32_t spectral) {
    if (m->kind != 1u) return 1.0f;
    return or_glass_n(m->glass, spectral ? lambda : 550.0f);
}

/* ------------------------------------------------------------------------ */
/* camera.rs:15-69                                                           */
/* ------------------------------------------------------------------------ */
void or_camera_look_at(const float origin[3], const float target[3], const float up[3],
                       float vfov_deg, float aspect, or_camera* out) {
    const float rads_per_deg = 3.14159265358979323846f / 180.0f;
    float theta = vfov_deg * rads_per_deg;
    float h = tanf(theta / 2.0f);
    float vh = 2.0f * h, vw = aspect * vh;
    v3 o = L(origin);
    v3 w = normalize(sub(o, L(target)));
    v3 u = normalize(cross(L(up), w));
    v3 v = cross(w, u);
    v3 hor = mul(u, vw), ver = mul(v, vh);
    v3 ll = sub(sub(sub(o, vdiv(hor, 2.0f)), vdiv(ver, 2.0f)), w);
    S(out->origin, o); S(out->lower_left, ll); S(out->horizontal, hor); S(out->vertical, ver);
}
static inline v3 primary_dir(const or_camera* c, float s, float t) {
    return normalize(sub(add(add(L(c->lower_left), mul(L(c->horizontal), s)), mul(L(c->vertical), t)), L(c->origin)));
}
void or_camera_primary_ray(const or_camera* c, float s, float t, float o[3], float d[3]) {
    S(o, L(c->origin)); S(d, primary_dir(c, s, t));
}
/* Camera::project with its per-call derived vectors precomputed (identical values). */
typedef struct { v3 o, u, v, w; float vw, vh; } proj_t;
static inline proj_t proj_make(const or_camera* c) {
    proj_t p; v3 H = L(c->horizontal), Vv = L(c->vertical);
    p.o = L(c->origin); p.u = normalize(H); p.v = normalize(Vv); p.vw = length(H); p.vh = length(Vv);
    p.w = sub(sub(sub(p.o, mul(H, 0.5f)), mul(Vv, 0.5f)), L(c->lower_left));
    return p;
}
static inline int proj(const proj_t* P, v3 p, float* s, float* t, float* depth) {
    v3 dir = sub(p, P->o);
    float c = dot(dir, P->w);
    if (c >= -1e-6f) return 0;
    float ss = 0.5f + dot(dir, P->u) / (-c * P->vw);
    float tt = 0.5f + dot(dir, P->v) / (-c * P->vh);
    if (ss >= 0.0f && ss < 1.0f && tt >= 0.0f && tt < 1.0f) { *s = ss; *t = tt; *depth = -c; return 1; }
    return 0;
}
void or_camera_proj_params(const or_camera* c, float out[16]) {
    const proj_t P = proj_make(c);
    const float v[16] = {P.o.x, P.o.y, P.o.z, 0.0f, P.u.x, P.u.y, P.u.z, P.vw,
                         P.v.x, P.v.y, P.v.z, P.vh, P.w.x, P.w.y, P.w.z, 0.0f};
    memcpy(out, v, sizeof v);
}
int or_camera_project(const or_camera* c, const float p[3], float out[3]) {
    proj_t P = proj_make(c);
    return proj(&P, L(p), &out[0], &out[1], &out[2]);
}

/* ------------------------------------------------------------------------ */
/* volume.rs                                                                 */
/* ------------------------------------------------------------------------ */
float or_phase_hg(float g, float cos_theta) { /* volume.rs:88-92 */
    if (g_fault == 5) g = -g;
    float g2 = g * g;
    float denom = powf(fmaxf(1.0f + g2 - 2.0f * g * cos_theta, 1e-6f), 1.5f);
    return (1.0f - g2) / (4.0f * 3.14159265358979323846f * denom);
}

static inline int64_t to_fixed(float x, float scale) {
    float y = x * scale;
    if (!(y > 0.0f)) return 0;
    if (y > 4.0e18f) y = 4.0e18f;
    return (int64_t)llrintf(y);
}

uint32_t or_simulate_photon(const or_scene* sc, const or_beam* beam, const or_vol_params* p,
                            uint32_t idx, uint32_t max_pairs, float* st, float* lambda_out,
                            uint32_t* tir_out) {
    rng_t r = rng_new(idx, p->seed);
    float r1 = rng_f32(&r), r2 = rng_f32(&r);
    v3 o = add(add(L(beam->corner), mul(L(beam->u), r1)), mul(L(beam->v), r2));
    float lambda = p->lambda_min + p->lambda_range * rng_f32(&r);
    v3 d = L(beam->dir);
    uint32_t n = 0, tir = 0;
#define PUSH(O, D) do { if (n < max_pairs) { float* q = st + 8 * n; q[0]=(O).x; q[1]=(O).y; q[2]=(O).z; q[3]=0; q[4]=(D).x; q[5]=(D).y; q[6]=(D).z; q[7]=0; } ++n; } while (0)
    PUSH(o, d);
    for (uint32_t b = 0; b < p->max_bounces; ++b) {
        hit_t h; uint32_t mi = 0;
        int any = scene_hit(sc, o, d, &h, &mi);
        float seg = any ? h.t : p->max_dist;
        for (int k = 0; k < 4; ++k) { float dist = rng_f32(&r) * seg; (void)dist; }
        if (!any) break;
        const or_mat* m = &sc->mats[mi];
        float nh = hero_index(m, lambda, p->spectral);
        if (m->kind == 1u) {
            float n1 = h.front_face ? 1.0f : nh, n2 = h.front_face ? nh : 1.0f;
            v3 tmp;
            if (!refract3(d, h.normal, n1, n2, &tmp)) ++tir;
        }
        v3 nd; float w;
        scatter(m, d, &h, nh, &r, &nd, &w);
        o = h.point; d = nd;
        PUSH(o, d);
    }
#undef PUSH
    *lambda_out = lambda;
    if (tir_out) *tir_out = tir;
    return n;
}

void or_render_point(const or_scene* sc, const or_camera* cam, const or_beam* beam,
                     const or_vol_params* p, const float* zbuf, uint32_t begin, uint32_t end,
                     float* img, int64_t* fxyz, int64_t* fspec) {
    const uint32_t W = p->width, H = p->height;
    proj_t P = proj_make(cam);
    const v3 cam_o = L(cam->origin);
    const float inv_4pi = 1.0f / (4.0f * 3.14159265358979323846f);
    for (uint32_t i = begin; i < end; ++i) {
        rng_t r = rng_new(i, p->seed);
        float r1 = rng_f32(&r), r2 = rng_f32(&r);
        v3 o = add(add(L(beam->corner), mul(L(beam->u), r1)), mul(L(beam->v), r2));
        float lambda = p->lambda_min + p->lambda_range * rng_f32(&r);
        float cm[3]; or_cmf(lambda, cm);
        uint32_t bin = 0;
        if (fspec) {
            float fb = (lambda - p->bin_min) * p->bin_inv_width;
            int bi = (int)fb;
            bin = fb < 0.0f ? 0u : (bi >= (int)p->bins ? p->bins - 1u : (uint32_t)bi);
        }
        v3 d = L(beam->dir);
        float power = 1.0f;
        for (uint32_t b = 0; b < p->max_bounces; ++b) {
            hit_t h; uint32_t mi = 0;
            int any = scene_hit(sc, o, d, &h, &mi);
            float seg = any ? h.t : p->max_dist;
            for (int k = 0; k < 4; ++k) {
                const float u = rng_f32(&r);
                /* free-flight estimator (3): truncated exponential distance, 1/pdf weight */
                const int ff = p->estimator == 3u && p->sigma_t > 0.0f;
                float dist = ff ? -log1pf(u * expm1f(-p->sigma_t * seg)) / p->sigma_t : u * seg;
                v3 q = add(o, mul(d, dist));
                float s, t, depth;
                if (!proj(&P, q, &s, &t, &depth)) continue;
                uint32_t px = (uint32_t)(s * (float)W); if (px > W - 1) px = W - 1;
                uint32_t py = (uint32_t)((1.0f - t) * (float)H); if (py > H - 1) py = H - 1;
                uint32_t pix = py * W + px;
                float contrib;
                if (p->estimator == 0u || p->estimator == 3u) {
                    v3 to = sub(cam_o, q);
                    float dd = fmaxf(length(to), 1e-3f);
                    if (zbuf && !(dd < zbuf[pix])) continue;
                    float cos_t = dot(d, vdiv(to, dd));
                    float phase = or_phase_hg(p->g, cos_t);
                    float trans = expf(-p->sigma_t * dd);
                    const float span = ff ? -expm1f(-p->sigma_t * seg) / (p->sigma_t * expf(-p->sigma_t * dist)) : seg;
                    contrib = power * p->sigma_s * phase * trans / (dd * dd) * span / (g_fault == 4 ? 1.0f : 4.0f);
                } else {
                    contrib = power * p->sigma_s * seg / 4.0f * inv_4pi;
                }
                if (img) for (int c = 0; c < 3; ++c) img[3 * pix + c] += cm[c] * contrib;
                if (fxyz) for (int c = 0; c < 3; ++c) fxyz[3 * pix + c] += to_fixed(cm[c] * contrib, p->scale);
                if (fspec) fspec[(size_t)pix * p->bins + bin] += to_fixed(contrib, p->scale);
            }
            if (!any) break;
            const or_mat* m = &sc->mats[mi];
            float nh = hero_index(m, lambda, p->spectral);
            v3 nd; float w;
            scatter(m, d, &h, nh, &r, &nd, &w);
            power *= w;
            o = h.point; d = nd;
        }
    }
}

typedef struct {
    const or_scene* sc; const or_camera* cam; const or_beam* beam; const or_vol_params* p;
    const float* zbuf; uint32_t begin, end; int64_t* fxyz; int64_t* fspec;
} point_job;
static void* point_worker(void* arg) {
    point_job* j = (point_job*)arg;
    or_render_point(j->sc, j->cam, j->beam, j->p, j->zbuf, j->begin, j->end, NULL, j->fxyz, j->fspec);
    return NULL;
}
void or_render_point_mt(const or_scene* sc, const or_camera* cam, const or_beam* beam,
                        const or_vol_params* p, const float* zbuf, uint32_t begin, uint32_t end,
                        int64_t* fxyz, int64_t* fspec, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    size_t npx = (size_t)p->width * p->height;
    size_t nx = fxyz ? 3 * npx : 0, ns = fspec ? npx * p->bins : 0;
    pthread_t* th = (pthread_t*)calloc(nthreads, sizeof(pthread_t));
    point_job* jobs = (point_job*)calloc(nthreads, sizeof(point_job));
    uint32_t n = end - begin;
    for (int t = 0; t < nthreads; ++t) {
        jobs[t].sc = sc; jobs[t].cam = cam; jobs[t].beam = beam; jobs[t].p = p; jobs[t].zbuf = zbuf;
        jobs[t].begin = begin + (uint32_t)((uint64_t)n * t / nthreads);
        jobs[t].end = begin + (uint32_t)((uint64_t)n * (t + 1) / nthreads);
        jobs[t].fxyz = nx ? (int64_t*)calloc(nx, 8) : NULL;
        jobs[t].fspec = ns ? (int64_t*)calloc(ns, 8) : NULL;
        pthread_create(&th[t], NULL, point_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) {
        pthread_join(th[t], NULL);
        for (size_t i = 0; i < nx; ++i) fxyz[i] += jobs[t].fxyz[i];
        for (size_t i = 0; i < ns; ++i) fspec[i] += jobs[t].fspec[i];
        free(jobs[t].fxyz); free(jobs[t].fspec);
    }
    free(th); free(jobs);
}

/* volume.rs:178-218 */
static void splat_transverse(float* img, uint32_t W, uint32_t H, float s, float t, const float col[3], float radius_px) {
    float cx = s * (float)W - 0.5f, cy = (1.0f - t) * (float)H - 0.5f;
    float r = fmaxf(radius_px, 0.5f);
    long x0 = (long)fmaxf(floorf(cx - r), 0.0f);
    long x1 = (long)ceilf(cx + r); if (x1 < 0) x1 = 0; if (x1 > (long)W - 1) x1 = W - 1;
    long y0 = (long)fmaxf(floorf(cy - r), 0.0f);
    long y1 = (long)ceilf(cy + r); if (y1 < 0) y1 = 0; if (y1 > (long)H - 1) y1 = H - 1;
    float wsum = 0.0f;
    for (long py = y0; py <= y1; ++py)
        for (long px = x0; px <= x1; ++px) {
            float dx = (float)px - cx, dy = (float)py - cy;
            wsum += fmaxf(1.0f - sqrtf(dx * dx + dy * dy) / r, 0.0f);
        }
    if (wsum <= 0.0f) {
        long px = (long)roundf(cx); if (px < 0) px = 0; if (px > (long)W - 1) px = W - 1;
        long py = (long)roundf(cy); if (py < 0) py = 0; if (py > (long)H - 1) py = H - 1;
        size_t i = (size_t)py * W + px;
        img[3 * i] += col[0]; img[3 * i + 1] += col[1]; img[3 * i + 2] += col[2];
        return;
    }
    float inv = 1.0f / wsum;
    for (long py = y0; py <= y1; ++py)
        for (long px = x0; px <= x1; ++px) {
            float dx = (float)px - cx, dy = (float)py - cy;
            float w = fmaxf(1.0f - sqrtf(dx * dx + dy * dy) / r, 0.0f) * inv;
            if (w > 0.0f) {
                size_t i = (size_t)py * W + px;
                img[3 * i] += col[0] * w; img[3 * i + 1] += col[1] * w; img[3 * i + 2] += col[2] * w;
            }
        }
}

/* volume.rs:233-329 */
void or_render_beam(const or_scene* sc, const or_camera* cam, const or_beam* beam,
                    const or_vol_params* p, const float* zbuf, uint32_t begin, uint32_t end, float* img) {
    const uint32_t W = p->width, H = p->height;
    proj_t P = proj_make(cam);
    const v3 cam_o = L(cam->origin);
    for (uint32_t i = begin; i < end; ++i) {
        rng_t r = rng_new(i, p->seed);
        float r1 = rng_f32(&r), r2 = rng_f32(&r);
        v3 o = add(add(L(beam->corner), mul(L(beam->u), r1)), mul(L(beam->v), r2));
        float lambda = p->lambda_min + p->lambda_range * rng_f32(&r);
        float cm[3]; or_cmf(lambda, cm);
        v3 d = L(beam->dir);
        float power = 1.0f;
        for (uint32_t b = 0; b < p->max_bounces; ++b) {
            hit_t h; uint32_t mi = 0;
            int any = scene_hit(sc, o, d, &h, &mi);
            float seg = any ? h.t : p->max_dist;
            v3 pend = add(o, mul(d, seg));
            float s0, t0, z0, s1, t1, z1;
            size_t m;
            if (proj(&P, o, &s0, &t0, &z0) && proj(&P, pend, &s1, &t1, &z1)) {
                float dx = (s1 - s0) * (float)W, dy = (t1 - t0) * (float)H;
                float mf = ceilf(sqrtf(dx * dx + dy * dy) * 2.0f);
                m = (size_t)mf + 1;
            } else {
                float mf = ceilf(seg * 80.0f);
                m = mf > 0.0f ? (size_t)mf : 0;
            }
            if (m < 1) m = 1;
            if (m > 4096) m = 4096;
            float ds = seg / (float)m;
            for (size_t k = 0; k < m; ++k) {
                float dist = ((float)k + 0.5f) * ds;
                v3 q = add(o, mul(d, dist));
                float s, t, depth;
                if (!proj(&P, q, &s, &t, &depth)) continue;
                uint32_t px = (uint32_t)(s * (float)W); if (px > W - 1) px = W - 1;
                uint32_t py = (uint32_t)((1.0f - t) * (float)H); if (py > H - 1) py = H - 1;
                v3 to = sub(cam_o, q);
                float dd = fmaxf(length(to), 1e-3f);
                if (zbuf && !(dd < zbuf[py * W + px])) continue;
                v3 view = vdiv(to, dd);
                float cos_t = dot(d, view);
                float phase = or_phase_hg(p->g, cos_t);
                float trans = expf(-p->sigma_t * dd);
                float weight = power * p->sigma_s * phase * trans / (dd * dd) * ds;
                float col[3] = {cm[0] * weight, cm[1] * weight, cm[2] * weight};
                v3 perp = cross(view, V(0, 1, 0));
                if (dot(perp, perp) < 1e-8f) perp = cross(view, V(1, 0, 0));
                perp = mul(normalize(perp), 0.03f);
                float s2, t2, z2, radius_px;
                if (proj(&P, add(q, perp), &s2, &t2, &z2)) {
                    float dpx = (s2 - s) * (float)W, dpy = (t2 - t) * (float)H;
                    radius_px = fminf(fmaxf(sqrtf(dpx * dpx + dpy * dpy), 1.5f), 24.0f);
                } else {
                    radius_px = 1.0f;
                }
                splat_transverse(img, W, H, s, t, col, radius_px);
            }
            if (!any) break;
            const or_mat* mt = &sc->mats[mi];
            float nh = hero_index(mt, lambda, p->spectral);
            v3 nd; float w;
            scatter(mt, d, &h, nh, &r, &nd, &w);
            power *= w;
            o = h.point; d = nd;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* lighttrace.rs:15-166                                                      */
/* ------------------------------------------------------------------------ */
void or_lighttrace(const or_scene* sc, const float scr[9], uint32_t W, uint32_t H,
                   const or_beam* beam, const or_vol_params* p, uint32_t n, float* sum) {
    v3 corner = L(scr), su = L(scr + 3), sv = L(scr + 6);
    v3 normal = normalize(cross(su, sv));
    for (uint32_t i = 0; i < n; ++i) {
        rng_t r = rng_new(i, p->seed);
        float r1 = rng_f32(&r), r2 = rng_f32(&r);
        v3 o = add(add(L(beam->corner), mul(L(beam->u), r1)), mul(L(beam->v), r2));
        float lambda = p->lambda_min + p->lambda_range * rng_f32(&r);
        v3 d = L(beam->dir);
        float power = 1.0f;
        int landed = 0; float ls = 0, lr = 0;
        for (uint32_t b = 0; b < p->max_bounces; ++b) {
            hit_t h; uint32_t mi = 0;
            int any = scene_hit(sc, o, d, &h, &mi);
            float scene_t = any ? h.t : INFINITY, screen_t = INFINITY, ss = 0, rr = 0;
            float denom = dot(d, normal);
            if (!(fabsf(denom) < 1e-8f)) {
                float t = dot(sub(corner, o), normal) / denom;
                if (!(t <= 1e-4f)) {
                    v3 q = add(o, mul(d, t));
                    v3 rel = sub(q, corner);
                    float s = dot(rel, su) / dot(su, su);
                    float rv = dot(rel, sv) / dot(sv, sv);
                    if (s >= 0.0f && s < 1.0f && rv >= 0.0f && rv < 1.0f) { screen_t = t; ss = s; rr = rv; }
                }
            }
            if (screen_t < scene_t) { landed = 1; ls = ss; lr = rr; break; }
            if (!any) break;
            const or_mat* m = &sc->mats[mi];
            float nh = hero_index(m, lambda, p->spectral);
            v3 nd; float w;
            scatter(m, d, &h, nh, &r, &nd, &w);
            power *= w;
            o = h.point; d = nd;
        }
        if (!landed) continue;
        float cm[3]; or_cmf(lambda, cm);
        float fx = ls * (float)W - 0.5f, fy = (1.0f - lr) * (float)H - 0.5f;
        fx = fminf(fmaxf(fx, 0.0f), (float)W - 1.0f);
        fy = fminf(fmaxf(fy, 0.0f), (float)H - 1.0f);
        uint32_t x0 = (uint32_t)floorf(fx), y0 = (uint32_t)floorf(fy);
        uint32_t x1 = x0 + 1 < W ? x0 + 1 : W - 1, y1 = y0 + 1 < H ? y0 + 1 : H - 1;
        float dx = fx - (float)x0, dy = fy - (float)y0;
        uint32_t xs[4] = {x0, x1, x0, x1}, ys[4] = {y0, y0, y1, y1};
        float ws[4] = {(1.0f - dx) * (1.0f - dy), dx * (1.0f - dy), (1.0f - dx) * dy, dx * dy};
        for (int q = 0; q < 4; ++q) {
            size_t idx = (size_t)ys[q] * W + xs[q];
            for (int c = 0; c < 3; ++c) sum[3 * idx + c] += cm[c] * power * ws[q];
        }
    }
}

/* Z-buffer pass of examples/prism_on_plane.rs:125-160: t of the nearer of the
 * scene hit and the floor Screen hit (screen_coords, lighttrace.rs:42-62). */
void or_scene_zbuffer(const or_scene* sc, const float* floor9, const or_camera* cam, uint32_t W, uint32_t H,
                      float* out) {
    v3 fc = {0, 0, 0}, fu = fc, fv = fc, fn = fc;
    if (floor9) { fc = L(floor9); fu = L(floor9 + 3); fv = L(floor9 + 6); fn = normalize(cross(fu, fv)); }
    for (uint32_t py = 0; py < H; ++py)
        for (uint32_t px = 0; px < W; ++px) {
            float s = ((float)px + 0.5f) / (float)W;
            float t = 1.0f - ((float)py + 0.5f) / (float)H;
            v3 o = L(cam->origin), d = primary_dir(cam, s, t);
            hit_t h; uint32_t mi;
            float t_scene = scene_hit(sc, o, d, &h, &mi) ? h.t : INFINITY, t_floor = INFINITY;
            if (floor9) {
                float denom = dot(d, fn);
                if (!(fabsf(denom) < 1e-8f)) {
                    float tt = dot(sub(fc, o), fn) / denom;
                    if (!(tt <= 1e-4f)) {
                        v3 rel = sub(add(o, mul(d, tt)), fc);
                        float ss = dot(rel, fu) / dot(fu, fu), rr = dot(rel, fv) / dot(fv, fv);
                        if (ss >= 0.0f && ss < 1.0f && rr >= 0.0f && rr < 1.0f) t_floor = tt;
                    }
                }
            }
            out[(size_t)py * W + px] = t_scene < t_floor ? t_scene : t_floor;
        }
}

/* ------------------------------------------------------------------------ */
/* tracer.rs:44-111, spectrum.rs:20-32, scene.rs:44-50                      */
/* ------------------------------------------------------------------------ */
static or_tracer_ext g_ext; /* zero: reference behaviour */
void or_tracer_set_ext(const or_tracer_ext* ext) {
    if (ext) g_ext = *ext; else memset(&g_ext, 0, sizeof g_ext);
}
static int g_spectral = 1;
void or_tracer_set_spectral(int on) { g_spectral = on ? 1 : 0; }

void or_tracer_sample(const or_scene* sc, const or_camera* cam, uint32_t W, uint32_t H,
                      uint32_t illum, uint32_t seed, uint32_t px, uint32_t py, uint32_t sidx,
                      uint32_t max_bounces, float out[3]) {
    const float LMIN = 380.0f, LRANGE = 350.0f;
    uint32_t pixel = py * W + px;
    rng_t r = rng_new(or_mix2(pixel, sidx), seed);
    float s = ((float)px + rng_f32(&r)) / (float)W;
    float t = 1.0f - ((float)py + rng_f32(&r)) / (float)H;
    float u = rng_f32(&r);
    const float step = LRANGE / 4.0f;
    float lam[4], rad[4] = {0, 0, 0, 0}, tp[4] = {1, 1, 1, 1};
    for (int j = 0; j < 4; ++j) {
        float off = fmodf(u * LRANGE + (float)j * step, LRANGE);
        if (off < 0.0f) off += LRANGE;
        lam[j] = LMIN + off;
    }
    const float pdf = 1.0f / LRANGE;
    v3 o = L(cam->origin), d = primary_dir(cam, s, t);
    uint32_t valid = 4;
    for (uint32_t b = 0; b < max_bounces; ++b) {
        hit_t h; uint32_t mi = 0;
        int any = scene_hit(sc, o, d, &h, &mi);
        if (g_ext.radius > 0.0f) {
            or_prim em = {{g_ext.center[0], g_ext.center[1], g_ext.center[2]}, g_ext.radius, 0, 0, 0, 0};
            hit_t he;
            if (sphere_hit(&em, o, d, 1e-3f, any ? h.t : INFINITY, &he)) {
                for (int k = 0; k < 4; ++k) rad[k] += tp[k] * g_ext.scale * or_illuminant(illum, lam[k]);
                break;
            }
        }
        if (!any) {
            float bg = sc->background + ((sc->has_horizon && d.y > 0.0f) ? sc->horizon : 0.0f);
            for (int k = 0; k < 4; ++k) rad[k] += tp[k] * bg * or_illuminant(illum, lam[k]);
            break;
        }
        const or_mat* m = &sc->mats[mi];
        float nh = m->kind == 1u ? or_glass_n(m->glass, g_spectral ? lam[0] : 550.0f) : 1.0f;
        v3 nd; float w;
        scatter(m, d, &h, nh, &r, &nd, &w);
        for (int k = 0; k < 4; ++k) tp[k] *= w;
        if (m->kind == 1u && valid > 1) { tp[1] = tp[2] = tp[3] = 0.0f; valid = 1; }
        o = h.point; d = nd;
        if (g_ext.rr_start && b + 1 >= g_ext.rr_start) {
            float q = fminf(tp[0], 0.95f);
            if (!(rng_f32(&r) < q)) break;
            for (int k = 0; k < 4; ++k) tp[k] = tp[k] / q;
        }
    }
    float x = 0, y = 0, z = 0;
    for (int k = 0; k < 4; ++k) {
        float c[3]; or_cmf(lam[k], c);
        float wk = rad[k] / pdf / (float)valid;
        x += c[0] * wk; y += c[1] * wk; z += c[2] * wk;
    }
    out[0] = x; out[1] = y; out[2] = z;
}

void or_tracer_accumulate(const or_scene* sc, const or_camera* cam, uint32_t W, uint32_t H,
                          uint32_t illum, uint32_t seed, uint32_t spp, uint32_t base,
                          uint32_t max_bounces, uint32_t row0, uint32_t row1, float* sum) {
    for (uint32_t py = row0; py < row1; ++py)
        for (uint32_t px = 0; px < W; ++px) {
            float acc[3] = {0, 0, 0};
            for (uint32_t k = 0; k < spp; ++k) {
                float c[3];
                or_tracer_sample(sc, cam, W, H, illum, seed, px, py, base + k, max_bounces, c);
                acc[0] += c[0]; acc[1] += c[1]; acc[2] += c[2];
            }
            size_t i = (size_t)py * W + px;
            sum[3 * i] += acc[0]; sum[3 * i + 1] += acc[1]; sum[3 * i + 2] += acc[2];
        }
}
typedef struct {
    const or_scene* sc; const or_camera* cam; uint32_t W, H, illum, seed, spp, base, mb, r0, r1; float* sum;
} tr_job;
static void* tr_worker(void* a) {
    tr_job* j = (tr_job*)a;
    or_tracer_accumulate(j->sc, j->cam, j->W, j->H, j->illum, j->seed, j->spp, j->base, j->mb, j->r0, j->r1, j->sum);
    return NULL;
}
void or_tracer_accumulate_mt(const or_scene* sc, const or_camera* cam, uint32_t W, uint32_t H,
                             uint32_t illum, uint32_t seed, uint32_t spp, uint32_t base,
                             uint32_t mb, float* sum, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    pthread_t* th = (pthread_t*)calloc(nthreads, sizeof(pthread_t));
    tr_job* jobs = (tr_job*)calloc(nthreads, sizeof(tr_job));
    for (int t = 0; t < nthreads; ++t) {
        tr_job j = {sc, cam, W, H, illum, seed, spp, base, mb,
                    (uint32_t)((uint64_t)H * t / nthreads), (uint32_t)((uint64_t)H * (t + 1) / nthreads), sum};
        jobs[t] = j;
        pthread_create(&th[t], NULL, tr_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th); free(jobs);
}

int or_scatter(uint32_t kind, float reflectance, const float wo[3], const float normal[3], int front_face,
               float n_hero, uint32_t key, uint32_t seed, float dir_out[3], float* weight) {
    or_mat m = {reflectance, 0u, kind, 0u};
    hit_t h; h.t = 1.0f; h.point = V(0, 0, 0); h.normal = L(normal); h.front_face = front_face;
    rng_t r = rng_new(key, seed);
    v3 d; float w;
    int ok = scatter(&m, L(wo), &h, n_hero, &r, &d, &w);
    S(dir_out, d); *weight = w;
    return ok;
}

uint32_t or_simulate_photon_fixed(const or_scene* sc, const or_beam* beam, const or_vol_params* p,
                                  uint32_t idx, float lambda, uint32_t max_pairs, float* st) {
    rng_t r = rng_new(idx, p->seed);
    float r1 = rng_f32(&r), r2 = rng_f32(&r);
    v3 o = add(add(L(beam->corner), mul(L(beam->u), r1)), mul(L(beam->v), r2));
    (void)rng_f32(&r);
    v3 d = L(beam->dir);
    uint32_t n = 0;
#define PUSH(O, D) do { if (n < max_pairs) { float* q = st + 8 * n; q[0]=(O).x; q[1]=(O).y; q[2]=(O).z; q[3]=0; q[4]=(D).x; q[5]=(D).y; q[6]=(D).z; q[7]=0; } ++n; } while (0)
    PUSH(o, d);
    for (uint32_t b = 0; b < p->max_bounces; ++b) {
        hit_t h; uint32_t mi = 0;
        int any = scene_hit(sc, o, d, &h, &mi);
        float seg = any ? h.t : p->max_dist;
        for (int k = 0; k < 4; ++k) { float dist = rng_f32(&r) * seg; (void)dist; }
        if (!any) break;
        const or_mat* m = &sc->mats[mi];
        float nh = m->kind == 1u ? or_glass_n(m->glass, lambda) : 1.0f;
        v3 nd; float w;
        scatter(m, d, &h, nh, &r, &nd, &w);
        o = h.point; d = nd;
        PUSH(o, d);
    }
#undef PUSH
    return n;
}

uint32_t or_mean_landing(const or_scene* sc, const float scr[9], const or_beam* beam, float lambda, uint32_t n,
                         uint32_t seed, float out[2]) {
    v3 corner = L(scr), su = L(scr + 3), sv = L(scr + 6);
    v3 normal = normalize(cross(su, sv));
    float sx = 0.0f, sr = 0.0f;
    uint32_t cnt = 0;
    for (uint32_t i = 0; i < n; ++i) {
        rng_t r = rng_new(i, seed);
        float r1 = rng_f32(&r), r2 = rng_f32(&r);
        v3 o = add(add(L(beam->corner), mul(L(beam->u), r1)), mul(L(beam->v), r2));
        v3 d = L(beam->dir);
        for (int b = 0; b < 8; ++b) {
            hit_t h; uint32_t mi = 0;
            int any = scene_hit(sc, o, d, &h, &mi);
            float scene_t = any ? h.t : INFINITY, screen_t = INFINITY, ss = 0, rr = 0;
            float denom = dot(d, normal);
            if (!(fabsf(denom) < 1e-8f)) {
                float t = dot(sub(corner, o), normal) / denom;
                if (!(t <= 1e-4f)) {
                    v3 q = add(o, mul(d, t)), rel = sub(q, corner);
                    float s = dot(rel, su) / dot(su, su), rv = dot(rel, sv) / dot(sv, sv);
                    if (s >= 0.0f && s < 1.0f && rv >= 0.0f && rv < 1.0f) { screen_t = t; ss = s; rr = rv; }
                }
            }
            if (screen_t < scene_t) { sx += ss; sr += rr; ++cnt; break; }
            if (!any) break;
            const or_mat* m = &sc->mats[mi];
            float nh = m->kind == 1u ? or_glass_n(m->glass, lambda) : 1.0f;
            v3 nd; float w;
            scatter(m, d, &h, nh, &r, &nd, &w);
            o = h.point; d = nd;
        }
    }
    out[0] = cnt ? sx / (float)cnt : 0.0f;
    out[1] = cnt ? sr / (float)cnt : 0.0f;
    return cnt;
}

/* ------------------------------------------------------------------------ */
/* vol_photons.rs:1517-1538 (surface rim), vol_splat.wgsl:58-79, viewer gather */
/* ------------------------------------------------------------------------ */
void or_surface_rim(const or_scene* sc, const or_camera* cam, uint32_t W, uint32_t H, float* out) {
    for (uint32_t py = 0; py < H; ++py)
        for (uint32_t px = 0; px < W; ++px) {
            float s = ((float)px + 0.5f) / (float)W;
            float t = 1.0f - ((float)py + 0.5f) / (float)H;
            v3 o = L(cam->origin), d = primary_dir(cam, s, t);
            hit_t h; uint32_t mi;
            size_t i = (size_t)py * W + px;
            if (scene_hit(sc, o, d, &h, &mi)) {
                float c = fminf(fmaxf(fabsf(dot(h.normal, d)), 0.0f), 1.0f);
                float rim = (1.0f - c) * (1.0f - c);
                out[3 * i] = 0.015f + rim * 0.45f; out[3 * i + 1] = 0.02f + rim * 0.5f; out[3 * i + 2] = 0.04f + rim * 0.6f;
            } else {
                out[3 * i] = out[3 * i + 1] = out[3 * i + 2] = 0.0f;
            }
        }
}

void or_synthetic_splat(uint32_t W, uint32_t H, uint32_t seed, uint32_t n, uint32_t* film) {
    uint32_t npx = W * H;
    for (uint32_t t = 0; t < n; ++t) {
        rng_t r = rng_new(t, seed);
        uint32_t idx = rng_u32(&r) % npx;
        float x = rng_f32(&r) * 2.0f, y = rng_f32(&r) * 2.0f, z = rng_f32(&r) * 2.0f;
        film[3 * idx] += (uint32_t)(fmaxf(x, 0.0f) * 4096.0f);
        film[3 * idx + 1] += (uint32_t)(fmaxf(y, 0.0f) * 4096.0f);
        film[3 * idx + 2] += (uint32_t)(fmaxf(z, 0.0f) * 4096.0f);
    }
}

void or_gather_tonemap(const float* xyz, const float* surface, uint32_t W, uint32_t H,
                       float k, float kradius, float exposure, uint8_t* rgba) {
    int radius = (int)kradius;
    float sigma = fmaxf(kradius * 0.5f, 0.5f);
    float inv2s2 = 1.0f / (2.0f * sigma * sigma);
    const float inv_gamma = (float)(1.0 / 2.2);
    for (uint32_t py = 0; py < H; ++py)
        for (uint32_t px = 0; px < W; ++px) {
            float acc[3] = {0, 0, 0}, wsum = 0.0f;
            for (int dy = -radius; dy <= radius; ++dy)
                for (int dx = -radius; dx <= radius; ++dx) {
                    int sx = (int)px + dx, sy = (int)py + dy;
                    if (sx >= 0 && sx < (int)W && sy >= 0 && sy < (int)H) {
                        size_t si = (size_t)sy * W + sx;
                        float g = expf(-(float)(dx * dx + dy * dy) * inv2s2);
                        for (int c = 0; c < 3; ++c) acc[c] = acc[c] + xyz[3 * si + c] * g;
                        wsum = wsum + g;
                    }
                }
            size_t i = (size_t)py * W + px;
            float kk = k / fmaxf(wsum, 1e-6f), comp[3], lin[3];
            for (int c = 0; c < 3; ++c) comp[c] = (acc[c] * kk + (surface ? surface[3 * i + c] : 0.0f)) * exposure;
            or_xyz_to_linear_srgb(comp, lin);
            for (int c = 0; c < 3; ++c) {
                float tt = lin[c] / (1.0f + lin[c]);
                float v = powf(fmaxf(tt, 0.0f), inv_gamma);
                v = fminf(fmaxf(v, 0.0f), 1.0f);
                rgba[4 * i + c] = (uint8_t)(v * 255.0f + 0.5f);
            }
            rgba[4 * i + 3] = 255;
        }
}
