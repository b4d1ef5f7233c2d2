// Per-photon transport shared by the plain photon kernel (photon.cu) and the
// batched persistent kernel (batch.cu): emission, bounce loop, haze samples and
// the fixed-point film deposit.  See photon.cu for the reference it restates.
#pragma once
#include "internal.h"

namespace sc {

constexpr float kInv4Pi = 1.0f / (4.0f * 3.14159265358979323846f);

// Stage the scene records and the CMF table in shared memory; when `mask_words`
// is non-zero a zeroed dirty-tile bitmask of that many words follows them.
__device__ __forceinline__ SceneView load_scene(const PhotonParams& p, unsigned char* smem, const float** cmf_out,
                                                uint32_t** mask_out = nullptr, uint32_t mask_words = 0) {
    sc_primitive* sp = reinterpret_cast<sc_primitive*>(smem);
    sc_plane* spl = reinterpret_cast<sc_plane*>(sp + p.n_prims);
    sc_material* sm = reinterpret_cast<sc_material*>(spl + p.n_planes);
    float* scmf = reinterpret_cast<float*>(sm + p.n_mats);
    uint32_t* mask = reinterpret_cast<uint32_t*>(scmf + 3 * kTableN);
    for (uint32_t i = threadIdx.x; i < p.n_prims; i += blockDim.x) sp[i] = p.prims[i];
    for (uint32_t i = threadIdx.x; i < p.n_planes; i += blockDim.x) spl[i] = p.planes[i];
    for (uint32_t i = threadIdx.x; i < p.n_mats; i += blockDim.x) sm[i] = p.mats[i];
    for (uint32_t i = threadIdx.x; i < 3u * kTableN; i += blockDim.x) scmf[i] = p.cmf[i];
    for (uint32_t i = threadIdx.x; i < mask_words; i += blockDim.x) mask[i] = 0u;
    __syncthreads();
    *cmf_out = scmf;
    if (mask_out) *mask_out = mask_words ? mask : nullptr;
    SceneView S;
    S.prims = sp; S.planes = spl; S.mats = sm; S.n_prims = p.n_prims;
    return S;
}

__device__ __forceinline__ void red_u64(unsigned long long* a, unsigned long long v) {
    if (v) atomicAdd(a, v);
}

// Exact segmented sum of 64-bit values over the lanes of `peers` using three
// 26-bit chunks (no chunk sum can overflow 32 bits for <= 32 lanes).
__device__ __forceinline__ unsigned long long peer_sum64(unsigned peers, unsigned long long v) {
    unsigned c0 = (unsigned)(v & 0x3FFFFFFull);
    unsigned c1 = (unsigned)((v >> 26) & 0x3FFFFFFull);
    unsigned c2 = (unsigned)(v >> 52);
    unsigned s0 = __reduce_add_sync(peers, c0);
    unsigned s1 = __reduce_add_sync(peers, c1);
    unsigned s2 = __reduce_add_sync(peers, c2);
    return (unsigned long long)s0 + ((unsigned long long)s1 << 26) + ((unsigned long long)s2 << 52);
}

// Dirty-tile bitmask: bits go to this CTA's shared-memory copy (flushed to the
// global mask when the CTA finishes) or, for films whose mask does not fit,
// straight to the global mask with a fire-and-forget red.or.
__device__ __forceinline__ void mark_tile(const PhotonParams& p, uint32_t* smask, uint32_t tile) {
    if (!p.flags) return;
    const uint32_t w = tile >> 5, bit = 1u << (tile & 31u);
    if (smask) {
        if (!(smask[w] & bit)) atomicOr(smask + w, bit);
    } else {
        atomicOr(p.flags + w, bit);
    }
}

// Deposit one haze sample.  AGG=1 merges lanes of the warp that hit the same
// film cell before issuing the atomic.
// `scale`: the film's 2^k, or 1 when `contrib` carries it already.
template <bool SPEC, int AGG>
__device__ __forceinline__ void deposit(const PhotonParams& p, uint32_t* smask, bool ok, uint32_t px, uint32_t py,
                                        float contrib, float cx, float cy, float cz, uint32_t bin, float scale) {
    size_t cell = 0;
    uint32_t tile = 0;
    unsigned long long v0 = 0, v1 = 0, v2 = 0;
    if (ok) {
        tile = film_tile(px, py, p.tiles_x);
        cell = film_cell(px, py, p.tiles_x, p.channels) + (SPEC ? bin : 0u);
        if (SPEC) {
            v0 = to_fixed(contrib, scale);
        } else {
            v0 = to_fixed(cx * contrib, scale);
            v1 = to_fixed(cy * contrib, scale);
            v2 = to_fixed(cz * contrib, scale);
        }
    }
    if (AGG == 0) {
        if (!ok) return;
        mark_tile(p, smask, tile);
        red_u64(p.film + cell, v0);
        if (!SPEC) { red_u64(p.film + cell + 1, v1); red_u64(p.film + cell + 2, v2); }
        return;
    }
    const unsigned mask = __activemask();
    const uint32_t key = ok ? (uint32_t)cell : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(mask, key);
    if (!ok) return;
    const unsigned lane = threadIdx.x & 31u;
    if (peers != (1u << lane)) {
        v0 = peer_sum64(peers, v0);
        if (!SPEC) { v1 = peer_sum64(peers, v1); v2 = peer_sum64(peers, v2); }
        if ((int)lane != __ffs(peers) - 1) return;
    }
    mark_tile(p, smask, tile);
    red_u64(p.film + cell, v0);
    if (!SPEC) { red_u64(p.film + cell + 1, v1); red_u64(p.film + cell + 2, v2); }
}

__device__ __forceinline__ void record_pair(sc_debug_photon* rec, uint32_t pair, f3 o, f3 d) {
    if (pair >= 9u) return;
    float* q = rec->states[2 * pair];
    q[0] = o.x; q[1] = o.y; q[2] = o.z; q[3] = 0.0f;
    q = rec->states[2 * pair + 1];
    q[0] = d.x; q[1] = d.y; q[2] = d.z; q[3] = 0.0f;
}

// Work counters of one photon (instrumented launches only): segments traced,
// haze samples that land in frame (= film splats), dielectric/diffuse scatters.
struct PhotonCounts { uint32_t segments, splats, scatters; };

// Free-flight sampling (estimator 3, no counterpart in the reference): the
// haze sample distance follows the free-flight density sigma_t exp(-sigma_t t)
// restricted to the segment, t = -log(1 - u (1 - exp(-sigma_t seg))) / sigma_t,
// and the sample is weighted by 1 / pdf(t) = (1 - exp(-sigma_t seg)) /
// (sigma_t exp(-sigma_t t)) instead of the uniform estimator's seg: the same
// single-scatter integral, with samples denser where the beam enters.  With
// sigma_t = 0 it is the uniform estimator.
// FF: free-flight distances (estimator 3 with sigma_t > 0).  Kernels are built
// with or without free-flight support (FFOK); launches of the uniform
// estimators take the kernels without it, whose code is the uniform path only.
__host__ __device__ __forceinline__ bool free_flight(const PhotonParams& p) {
    return p.estimator == 3u && p.sigma_t > 0.0f;
}
template <bool FF>
__device__ __forceinline__ float haze_distance(const PhotonParams& p, float u, float seg) {
    if (!FF) return u * seg;
    return -log1pf(u * expm1f(-p.sigma_t * seg)) / p.sigma_t;
}
template <bool FF>
__device__ __forceinline__ float haze_span(const PhotonParams& p, float dist, float seg) {
    if (!FF) return seg;
    return -expm1f(-p.sigma_t * seg) / (p.sigma_t * expf(-p.sigma_t * dist));
}

// One point-estimator haze sample at distance `dist` along a segment
// (spectral-core/src/volume.rs:130-150): camera projection, z-test, HG phase x
// transmittance / d^2 x seg/4 (x 1/pdf / 4 for free-flight samples).  Returns
// whether the sample lands in frame; `contrib`, px, py are its weight and pixel.
template <bool FF>
__device__ __forceinline__ bool haze_sample(const PhotonParams& p, f3 o, f3 d, float dist, float seg, float power,
                                            uint32_t& px, uint32_t& py, float& contrib) {
    const f3 q = add(o, mul(d, dist));
    float s, t;
    bool ok = project(p.proj, q, s, t);
    contrib = 0.0f;
    px = py = 0u;
    if (ok) {
        px = min((uint32_t)(s * (float)p.width), p.width - 1u);
        py = min((uint32_t)((1.0f - t) * (float)p.height), p.height - 1u);
        if (FF || p.estimator != 1u) {  // point estimators (the beam estimator has its own kernel)
            const f3 to = sub(p.proj.o, q);
            const float dd = fmaxf(length(to), 1e-3f);
            if (p.zbuf && !(dd < p.zbuf[py * p.width + px])) {
                ok = false;
            } else {
                // g == 0: phase_hg is exactly 1/(4 pi) (pow(1, 1.5) == 1), so the
                // direction to the camera is not needed.
                const float phase = p.g == 0.0f ? kInv4Pi : phase_hg(p.g, dot(d, vdiv(to, dd)));
                const float trans = expf(-p.sigma_t * dd);
                contrib = power * p.sigma_s * phase * trans / (dd * dd) * haze_span<FF>(p, dist, seg) / 4.0f;
            }
        } else {
            contrib = power * p.sigma_s * seg / 4.0f * kInv4Pi;
        }
    }
    return ok;
}

// ---------------------------------------------------------------------------
// Fast haze samples.  Only the transport (intersection, Fresnel / refract /
// TIR, Sellmeier) decides a photon's path; the haze samples only weight film
// deposits, so they need the film's accuracy (0.5 % relative L1), not the CPU
// crate's operation order.  Along a segment q(t) = o + d t, with D = o - o_cam
// and the camera basis (u, v, w, |horizontal|, |vertical|):
//   depth  c(t)     = D.w + (d.w) t                  (in front: c < -1e-6)
//   column s(t) * W = W/2 + (a0 + a1 t) / -c(t),  a = (D.u, d.u) * W / |horizontal|
//   row (1-t') * H  = H/2 + (b0 + b1 t) / -c(t),  b = (D.v, d.v) * -H / |vertical|
//   distance^2      = h2 + (s0 + s1 t)^2,  s1 = |d|, s0 = -|d| t*, t* = -D.d / |d|^2,
//                     h2 = |D + d t*|^2 (squared distance of closest approach: a sum of
//                     two non-negative terms, so no cancellation near the camera)
//   d . (to camera) / distance = -s1 (s0 + s1 t) / distance
// so a sample costs three fused multiply-adds for the projection, one
// reciprocal, one reciprocal square root and one exp2 (PTX approximations),
// and the constant factor k = power sigma_s seg / 4 * 2^scale * HG numerator
// is formed once per segment.  The HG denominator power 1.5 is r^3 with
// r = rsqrt(max(1 + g^2 - 2 g cos, 1e-6)).
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Per-segment constants.  `segs` is seg * 2^-24 for the uniform estimator
// (t = (draw >> 8) * segs, the same product the reference rounds) and
// expm1(-sigma_t seg) for free-flight distances.
struct HazeSeg { float c0, c1, a0, a1, b0, b1, s0, s1, h2, k, segs; };

// Dot product with fused multiply-adds (haze constants only: the transport
// keeps the reference's separate multiplies and adds).
__device__ __forceinline__ float fdot(f3 a, f3 b) { return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, a.x * b.x)); }

template <bool FF>
__device__ __forceinline__ HazeSeg haze_setup(const PhotonParams& p, f3 o, f3 d, float seg, float power) {
    const Proj& P = p.proj;
    const f3 D = sub(o, P.o);
    HazeSeg h;
    h.c0 = fdot(D, P.w);
    h.c1 = fdot(d, P.w);
    h.a0 = fdot(D, P.u) * p.hz_sx;
    h.a1 = fdot(d, P.u) * p.hz_sx;
    h.b0 = fdot(D, P.v) * p.hz_sy;
    h.b1 = fdot(d, P.v) * p.hz_sy;
    const float e2 = fdot(d, d);
    const float r2 = rsqrt_approx(e2);                 // 1 / |d|
    const float tstar = -fdot(D, d) * (r2 * r2);
    const f3 m = mk(__fmaf_rn(d.x, tstar, D.x), __fmaf_rn(d.y, tstar, D.y), __fmaf_rn(d.z, tstar, D.z));
    h.h2 = fdot(m, m);
    h.s1 = e2 * r2;                                    // |d|
    h.s0 = -h.s1 * tstar;
    if (FF) {
        const float em = expm1f(-p.sigma_t * seg);
        h.segs = em;
        h.k = power * (-em * p.hz_inv_sigma_t) * p.hz_k;  // 1/pdf numerator (1 - e^-sigma_t seg) / sigma_t
    } else {
        h.segs = seg * (1.0f / 16777216.0f);
        h.k = power * seg * (p.estimator == 1u ? p.hz_kiso : p.hz_k);
    }
    return h;
}

// One haze sample of a segment from its 24-bit draw; returns whether it lands
// in frame (and is not occluded), with its pixel and its scaled weight.
template <bool FF>
__device__ __forceinline__ bool haze_fast(const PhotonParams& p, const HazeSeg& h, uint32_t draw24, uint32_t& px,
                                          uint32_t& py, float& contrib) {
    float t;
    if (FF) t = -log1pf((float)draw24 * (1.0f / 16777216.0f) * h.segs) * p.hz_inv_sigma_t;
    else t = (float)draw24 * h.segs;
    const float c = __fmaf_rn(h.c1, t, h.c0);
    const float rc = rcp_approx(-c);
    const float x = __fmaf_rn(__fmaf_rn(h.a1, t, h.a0), rc, p.hz_hw);
    const float y = __fmaf_rn(__fmaf_rn(h.b1, t, h.b0), rc, p.hz_hh);
    contrib = 0.0f;
    px = py = 0u;
    if (!(c < -1e-6f && x >= 0.0f && x < p.hz_w && y > 0.0f && y <= p.hz_h)) return false;
    px = min((uint32_t)x, p.width - 1u);
    py = min((uint32_t)y, p.height - 1u);
    if (!FF && p.estimator == 1u) {  // isotropic estimator: no transmittance, no 1/d^2, no z-test
        contrib = h.k;
        return true;
    }
    const float q = __fmaf_rn(h.s1, t, h.s0);
    const float dd2 = fmaxf(__fmaf_rn(q, q, h.h2), 1e-6f);
    const float r = rsqrt_approx(dd2);
    const float dd = dd2 * r;
    if (p.zbuf && !(dd < p.zbuf[py * p.width + px])) return false;
    float w = h.k * ex2_approx(p.hz_kexp * (FF ? dd - t : dd)) * (r * r);
    if (p.g != 0.0f) {
        const float den = fmaxf(__fmaf_rn(p.hz_m2g, -(h.s1 * q) * r, p.hz_g2), 1e-6f);
        const float rr = rsqrt_approx(den);
        w *= rr * rr * rr;
    }
    contrib = w;
    return true;
}

// Photon-level splat payload: CMF of the photon's wavelength (XYZ film) or its bin.
__device__ __forceinline__ void photon_payload(const PhotonParams& p, const float* cmf, float lambda, float& cx,
                                               float& cy, float& cz, uint32_t& bin, bool spec) {
    if (spec) {
        float fb = (lambda - p.bin_min) * p.bin_inv_width;
        int bi = (int)fb;
        bin = fb < 0.0f ? 0u : (bi >= (int)p.bins ? p.bins - 1u : (uint32_t)bi);
    } else {
        cx = tab_sample(cmf, lambda);
        cy = tab_sample(cmf + kTableN, lambda);
        cz = tab_sample(cmf + 2 * kTableN, lambda);
    }
}

// EXACT: haze samples in the CPU crate's operation order (haze_sample);
// otherwise the fast haze samples, as the warp-split transport runs them.
template <bool SPEC, int AGG, bool DEBUG, bool COUNT = false, bool FFOK = true, bool EXACT = false>
__device__ __forceinline__ void trace_photon(const PhotonParams& p, const SceneView& S, const float* cmf,
                                             uint32_t idx, uint32_t* smask, PhotonCounts* cnt = nullptr) {
    Rng r = Rng::make(idx, p.seed);
    const float r1 = r.f32();
    const float r2 = r.f32();
    f3 o = add(add(p.corner, mul(p.bu, r1)), mul(p.bv, r2));
    const float lambda = p.lambda_min + p.lambda_range * r.f32();
    float cx = 0.f, cy = 0.f, cz = 0.f;
    uint32_t bin = 0;
    if (!DEBUG) photon_payload(p, cmf, lambda, cx, cy, cz, bin, SPEC);
    f3 d = p.bdir;
    float power = 1.0f;
    uint32_t n_glass = 0xFFFFFFFFu;
    float n_cached = 1.0f;
    sc_debug_photon* rec = nullptr;
    uint32_t pairs = 1;
    if (DEBUG) {
        rec = p.debug + idx;
        rec->lambda = lambda;
        rec->pad0 = rec->pad1 = 0u;
        record_pair(rec, 0, o, d);
    }
    for (uint32_t b = 0; b < p.max_bounces; ++b) {
        Hit h;
        uint32_t mi = 0;
        const bool any = scene_hit(S, o, d, h, mi);
        const float seg = any ? h.t : p.max_dist;
        if (COUNT) ++cnt->segments;
        const bool ff = FFOK && free_flight(p);
        if (DEBUG) {
            r.state += 4u;  // the segment's 4 distance draws
        } else if (EXACT) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const float u = r.f32();
                const float dist = ff ? haze_distance<true>(p, u, seg) : haze_distance<false>(p, u, seg);
                uint32_t px, py;
                float contrib;
                const bool ok = ff ? haze_sample<true>(p, o, d, dist, seg, power, px, py, contrib)
                                   : haze_sample<false>(p, o, d, dist, seg, power, px, py, contrib);
                if (COUNT) { if (ok) ++cnt->splats; continue; }
                deposit<SPEC, AGG>(p, smask, ok, px, py, contrib, cx, cy, cz, bin, p.scale);
            }
        } else {
            const HazeSeg hz = ff ? haze_setup<true>(p, o, d, seg, power) : haze_setup<false>(p, o, d, seg, power);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t draw24 = r.u32() >> 8;
                uint32_t px, py;
                float contrib;
                const bool ok = ff ? haze_fast<true>(p, hz, draw24, px, py, contrib)
                                   : haze_fast<false>(p, hz, draw24, px, py, contrib);
                if (COUNT) { if (ok) ++cnt->splats; continue; }
                deposit<SPEC, AGG>(p, smask, ok, px, py, contrib, cx, cy, cz, bin, 1.0f);
            }
        }
        if (!any) break;
        const sc_material& m = S.mats[mi];
        // n(lambda) depends only on the photon's wavelength and the glass: the f64
        // Sellmeier sum runs once per photon and glass, not once per hit.
        float nh = 1.0f;
        if (m.kind == 1u) {
            if (m.glass != n_glass) { n_cached = glass_n(m.glass, p.spectral ? lambda : 550.0f); n_glass = m.glass; }
            nh = n_cached;
        }
        f3 nd;
        float w;
        if (COUNT) ++cnt->scatters;
        scatter(m, d, h, nh, r, nd, w);
        power *= w;
        o = h.point;
        d = nd;
        if (DEBUG) { record_pair(rec, pairs, o, d); ++pairs; }
    }
    if (DEBUG) rec->num_states = pairs < 9u ? pairs : 9u;
}

// One photon per lane over positions [first, count) of a range, stepping `stride`
// (photon id = id(k)), written as one loop of bounce steps: a lane whose photon
// has ended starts its next photon inside the loop, so the warp reconverges at
// every bounce step instead of waiting at the end of each photon for the
// warp's longest one.  The photons, their draws and their samples are those of
// trace_photon (fast haze samples), so the film is bit-identical to it.
template <bool SPEC, int AGG, bool FFOK, class Id>
__device__ __forceinline__ void trace_lane_range(const PhotonParams& p, const SceneView& S, const float* cmf,
                                                 uint32_t first, uint32_t count, uint32_t stride, Id id,
                                                 uint32_t* smask) {
    const bool ff = FFOK && free_flight(p);
    Rng r;
    r.state = 0u;
    f3 o = mk(0.f, 0.f, 0.f), d = p.bdir;
    float lambda = 0.0f, power = 1.0f, cx = 0.f, cy = 0.f, cz = 0.f;
    uint32_t bin = 0, bounce = 0, n_glass = 0xFFFFFFFFu;
    float n_cached = 1.0f;
    bool alive = false;
    uint32_t next = first;
    for (;;) {
        if (!alive) {
            if (next >= count || p.max_bounces == 0u) break;
            r = Rng::make(id(next), p.seed);
            next += stride;
            const float r1 = r.f32();
            const float r2 = r.f32();
            o = add(add(p.corner, mul(p.bu, r1)), mul(p.bv, r2));
            d = p.bdir;
            lambda = p.lambda_min + p.lambda_range * r.f32();
            photon_payload(p, cmf, lambda, cx, cy, cz, bin, SPEC);
            power = 1.0f;
            bounce = 0;
            n_glass = 0xFFFFFFFFu;
            alive = true;
        }
        Hit h;
        uint32_t mi = 0;
        const bool any = scene_hit(S, o, d, h, mi);
        const float seg = any ? h.t : p.max_dist;
        const HazeSeg hz = ff ? haze_setup<true>(p, o, d, seg, power) : haze_setup<false>(p, o, d, seg, power);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t draw24 = r.u32() >> 8;
            uint32_t px, py;
            float contrib;
            const bool ok = ff ? haze_fast<true>(p, hz, draw24, px, py, contrib)
                               : haze_fast<false>(p, hz, draw24, px, py, contrib);
            deposit<SPEC, AGG>(p, smask, ok, px, py, contrib, cx, cy, cz, bin, 1.0f);
        }
        ++bounce;
        if (!any || bounce >= p.max_bounces) {
            alive = false;  // escaped, or its last segment: no scatter needed
            continue;
        }
        const sc_material& m = S.mats[mi];
        float nh = 1.0f;
        if (m.kind == 1u) {
            if (m.glass != n_glass) { n_cached = glass_n(m.glass, p.spectral ? lambda : 550.0f); n_glass = m.glass; }
            nh = n_cached;
        }
        f3 nd;
        float w;
        scatter(m, d, h, nh, r, nd, w);
        power *= w;
        o = h.point;
        d = nd;
    }
}

// ---------------------------------------------------------------------------
// Warp-split transport.  (a) Every lane traces its photon's path (intersect,
// Fresnel / refract / TIR scatter) and appends one record per segment to the
// warp's shared-memory segment buffer; (b) the warp then works through the 4
// haze samples of every buffered segment as one flat list, so the expensive
// camera connection runs converged even when the photons of a warp have
// different numbers of segments.  PCG is counter based: sample k of a segment
// uses draw pcg32(state_before + k + 1), exactly the draw the per-photon loop
// makes, so paths and films are bit-identical to trace_photon's.
// Segment record: the fast haze constants of the segment, the RNG state
// before its 4 distance draws, and the photon's splat payload: its bin
// (spectral films) or the CMF x, y, z of its wavelength (XYZ films).
struct alignas(16) SegRec {
    HazeSeg hz;
    uint32_t rng, bin;
    float cx, cy, cz;
};
static_assert(sizeof(SegRec) == 64, "segment record layout");
template <uint32_t SEGS>
struct alignas(16) WarpSplitSmem {
    SegRec seg[SEGS];
};
// Segments buffered per warp: 64 in the plain photon kernel, 48 in the batch
// kernel (whose warps also hold a job slot and a dirty mask).
constexpr uint32_t kWarpSegs = 64;
constexpr uint32_t kBatchWarpSegs = 48;

template <bool SPEC, int AGG, bool FF, uint32_t SEGS>
__device__ __forceinline__ void flush_loop(const PhotonParams& p, WarpSplitSmem<SEGS>& ws, uint32_t total,
                                           uint32_t* smask, uint32_t lane) {
    for (uint32_t t = lane; t < total; t += 32u) {
        const SegRec& R = ws.seg[t >> 2];
        const HazeSeg hz = R.hz;
        const uint32_t draw24 = pcg32(R.rng + (t & 3u) + 1u) >> 8;
        uint32_t px, py;
        float contrib;
        const bool ok = haze_fast<FF>(p, hz, draw24, px, py, contrib);
        if (SPEC) deposit<true, AGG>(p, smask, ok, px, py, contrib, 0.f, 0.f, 0.f, R.bin, 1.0f);
        else deposit<false, AGG>(p, smask, ok, px, py, contrib, R.cx, R.cy, R.cz, 0u, 1.0f);
    }
}

// The estimator is fixed per job: one uniform branch picks the loop.
template <bool SPEC, int AGG, bool FFOK, uint32_t SEGS>
__device__ __forceinline__ void flush_segments(const PhotonParams& p, WarpSplitSmem<SEGS>& ws, uint32_t n,
                                               uint32_t* smask, uint32_t lane) {
    __syncwarp();
    if (FFOK && free_flight(p)) flush_loop<SPEC, AGG, true>(p, ws, 4u * n, smask, lane);
    else flush_loop<SPEC, AGG, false>(p, ws, 4u * n, smask, lane);
    __syncwarp();
}

// The photons of positions [0, count) of a range (photon id = id(k)) through
// the warp-split transport.  All 32 lanes of the warp call this together.  A
// lane whose photon has ended (escaped, or out of bounces) takes the next
// unclaimed photon of the range at the next bounce, so the lanes stay busy
// through the bounce loop although photons end after different numbers of
// segments; the photons, their RNG draws and their samples are the same, so
// the film is bit-identical to the per-photon transport's.
template <bool SPEC, int AGG, bool FFOK, uint32_t SEGS, class Id>
__device__ __forceinline__ void trace_warp_range(const PhotonParams& p, const SceneView& S, const float* cmf,
                                                 uint32_t count, Id id, uint32_t* smask, WarpSplitSmem<SEGS>& ws) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    const bool ff = FFOK && free_flight(p);
    Rng r;
    r.state = 0u;
    f3 o = mk(0.f, 0.f, 0.f), d = p.bdir;
    float lambda = 0.0f, power = 1.0f, cx = 0.f, cy = 0.f, cz = 0.f;
    uint32_t bin = 0, bounce = 0, n_glass = 0xFFFFFFFFu;
    float n_cached = 1.0f;
    bool alive = false;
    uint32_t next = 0;  // first unclaimed position of the range (the same in every lane)
    uint32_t n = 0;     // buffered segments (the same in every lane)
    for (;;) {
        if (next < count) {  // idle lanes start the next photons of the range
            const unsigned idle = __ballot_sync(0xffffffffu, !alive);
            const uint32_t k = next + __popc(idle & below);
            if (!alive && k < count) {
                r = Rng::make(id(k), p.seed);
                const float r1 = r.f32();
                const float r2 = r.f32();
                o = add(add(p.corner, mul(p.bu, r1)), mul(p.bv, r2));
                d = p.bdir;
                lambda = p.lambda_min + p.lambda_range * r.f32();
                photon_payload(p, cmf, lambda, cx, cy, cz, bin, SPEC);
                power = 1.0f;
                bounce = 0;
                n_glass = 0xFFFFFFFFu;
                alive = p.max_bounces > 0u;
            }
            next += __popc(idle);
        }
        const unsigned m = __ballot_sync(0xffffffffu, alive);
        const uint32_t cnt = __popc(m);
        // one flush site (keeps the inlined haze code single): when this round's
        // segments do not fit, and once when the range is done
        if (n + cnt > SEGS || (m == 0u && n)) {
            flush_segments<SPEC, AGG, FFOK, SEGS>(p, ws, n, smask, lane);
            n = 0;
        }
        if (m == 0u) break;  // nothing alive and nothing left to start
        if (alive) {
            Hit h;
            uint32_t mi = 0;
            const bool any = scene_hit(S, o, d, h, mi);
            const float seg = any ? h.t : p.max_dist;
            SegRec& R = ws.seg[n + __popc(m & below)];
            R.hz = ff ? haze_setup<true>(p, o, d, seg, power) : haze_setup<false>(p, o, d, seg, power);
            R.rng = r.state;
            R.bin = bin;
            R.cx = cx; R.cy = cy; R.cz = cz;
            r.state += 4u;  // this segment's 4 distance draws, made by the flush
            ++bounce;
            if (!any || bounce >= p.max_bounces) {
                alive = false;  // escaped, or its last segment: no scatter needed
            } else {
                const sc_material& mt = S.mats[mi];
                float nh = 1.0f;
                if (mt.kind == 1u) {
                    if (mt.glass != n_glass) {
                        n_cached = glass_n(mt.glass, p.spectral ? lambda : 550.0f);
                        n_glass = mt.glass;
                    }
                    nh = n_cached;
                }
                f3 nd;
                float w;
                scatter(mt, d, h, nh, r, nd, w);
                power *= w;
                o = h.point;
                d = nd;
            }
        }
        n += cnt;
    }
}

}  // namespace sc
