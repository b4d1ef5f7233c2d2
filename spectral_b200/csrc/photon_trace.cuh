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
template <bool SPEC, int AGG>
__device__ __forceinline__ void deposit(const PhotonParams& p, uint32_t* smask, bool ok, uint32_t px, uint32_t py,
                                        float contrib, float cx, float cy, float cz, uint32_t bin) {
    size_t cell = 0;
    uint32_t tile = 0;
    unsigned long long v0 = 0, v1 = 0, v2 = 0;
    if (ok) {
        tile = film_tile(px, py, p.tiles_x);
        cell = film_cell(px, py, p.tiles_x, p.channels) + (SPEC ? bin : 0u);
        if (SPEC) {
            v0 = to_fixed(contrib, p.scale);
        } else {
            v0 = to_fixed(cx * contrib, p.scale);
            v1 = to_fixed(cy * contrib, p.scale);
            v2 = to_fixed(cz * contrib, p.scale);
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

template <bool SPEC, int AGG, bool DEBUG, bool COUNT = false, bool FFOK = true>
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
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const bool ff = FFOK && free_flight(p);
            const float u = r.f32();
            const float dist = ff ? haze_distance<true>(p, u, seg) : haze_distance<false>(p, u, seg);
            if (DEBUG) continue;
            uint32_t px, py;
            float contrib;
            const bool ok = ff ? haze_sample<true>(p, o, d, dist, seg, power, px, py, contrib)
                               : haze_sample<false>(p, o, d, dist, seg, power, px, py, contrib);
            if (COUNT) { if (ok) ++cnt->splats; continue; }
            deposit<SPEC, AGG>(p, smask, ok, px, py, contrib, cx, cy, cz, bin);
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

// ---------------------------------------------------------------------------
// Warp-split transport.  (a) Every lane traces its photon's path (intersect,
// Fresnel / refract / TIR scatter) and appends one record per segment to the
// warp's shared-memory segment buffer; (b) the warp then works through the 4
// haze samples of every buffered segment as one flat list, so the expensive
// camera connection runs converged even when the photons of a warp have
// different numbers of segments.  PCG is counter based: sample k of a segment
// uses draw pcg32(state_before + k + 1), exactly the draw the per-photon loop
// makes, so paths and films are bit-identical to trace_photon's.
struct SegRec { f3 o, d; float seg, power; uint32_t rng, lane; };
constexpr uint32_t kWarpSegs = 64;
struct alignas(16) WarpSplitSmem {
    SegRec seg[kWarpSegs];
    float4 payload[32];  // per lane: CMF x, y, z of the photon (XYZ film) or its bin in .w
};
static_assert(sizeof(SegRec) == 40, "segment record layout");

template <bool SPEC, int AGG, bool FF>
__device__ __forceinline__ void flush_loop(const PhotonParams& p, WarpSplitSmem& ws, uint32_t total, uint32_t* smask,
                                           uint32_t lane) {
    for (uint32_t t = lane; t < total; t += 32u) {
        const SegRec R = ws.seg[t >> 2];
        const float u = (float)(pcg32(R.rng + (t & 3u) + 1u) >> 8) * (1.0f / 16777216.0f);
        uint32_t px, py;
        float contrib;
        const bool ok = haze_sample<FF>(p, R.o, R.d, haze_distance<FF>(p, u, R.seg), R.seg, R.power, px, py, contrib);
        const float4 pl = ws.payload[R.lane];
        deposit<SPEC, AGG>(p, smask, ok, px, py, contrib, pl.x, pl.y, pl.z, __float_as_uint(pl.w));
    }
}

// The estimator is fixed per job: one uniform branch picks the loop.
template <bool SPEC, int AGG, bool FFOK>
__device__ __forceinline__ void flush_segments(const PhotonParams& p, WarpSplitSmem& ws, uint32_t n, uint32_t* smask,
                                               uint32_t lane) {
    __syncwarp();
    if (FFOK && free_flight(p)) flush_loop<SPEC, AGG, true>(p, ws, 4u * n, smask, lane);
    else flush_loop<SPEC, AGG, false>(p, ws, 4u * n, smask, lane);
    __syncwarp();
}

// All 32 lanes of the warp must call this together; lanes without a photon pass
// valid = false.
template <bool SPEC, int AGG, bool FFOK>
__device__ __forceinline__ void trace_warp_split(const PhotonParams& p, const SceneView& S, const float* cmf,
                                                 uint32_t idx, bool valid, uint32_t* smask, WarpSplitSmem& ws) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned below = (1u << lane) - 1u;
    Rng r = Rng::make(idx, p.seed);
    f3 o = mk(0.f, 0.f, 0.f), d = p.bdir;
    float lambda = 0.0f, power = 1.0f;
    if (valid) {
        const float r1 = r.f32();
        const float r2 = r.f32();
        o = add(add(p.corner, mul(p.bu, r1)), mul(p.bv, r2));
        lambda = p.lambda_min + p.lambda_range * r.f32();
        float cx = 0.f, cy = 0.f, cz = 0.f;
        uint32_t bin = 0;
        photon_payload(p, cmf, lambda, cx, cy, cz, bin, SPEC);
        ws.payload[lane] = make_float4(cx, cy, cz, __uint_as_float(bin));
    }
    bool alive = valid;
    uint32_t n = 0;  // buffered segments, the same in every lane
    uint32_t n_glass = 0xFFFFFFFFu;
    float n_cached = 1.0f;
    for (uint32_t b = 0;; ++b) {
        const unsigned m = b < p.max_bounces ? __ballot_sync(0xffffffffu, alive) : 0u;
        const uint32_t cnt = __popc(m);
        // one flush site (keeps the inlined haze code single): when this bounce's
        // segments do not fit, and once when every photon is done
        if (n + cnt > kWarpSegs || (m == 0u && n)) {
            flush_segments<SPEC, AGG, FFOK>(p, ws, n, smask, lane);
            n = 0;
        }
        if (m == 0u) break;
        Hit h;
        uint32_t mi = 0;
        bool any = false;
        float seg = 0.0f;
        if (alive) {
            any = scene_hit(S, o, d, h, mi);
            seg = any ? h.t : p.max_dist;
        }
        if (alive) {
            SegRec& R = ws.seg[n + __popc(m & below)];
            R.o = o; R.d = d; R.seg = seg; R.power = power; R.rng = r.state; R.lane = lane;
            r.state += 4u;  // this segment's 4 distance draws, made by the flush
            if (!any) {
                alive = false;
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
