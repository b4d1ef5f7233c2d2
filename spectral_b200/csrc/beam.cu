// Photon-beam estimator: render_volumetric_scene + splat_transverse
// (spectral-core/src/volume.rs:170-329).
//
// Same emission and bounce loop as the point estimator, but no per-segment
// distance draws: every segment (including the escaping one, length max_dist)
// is marched in M = ceil(2 x projected pixel length) + 1 deterministic steps
// (ceil(80 x length) when an end point is off frame; 1 <= M <= 4096).  Each step
// at distance (k + 1/2) * len / M is connected to the camera with the point
// estimator's weight (HG phase x transmittance / d^2) times the step length, and
// deposited over a tent footprint whose radius is the projected beam radius
// 0.03 (clamped to [1.5, 24] px, 1 px when the offset point leaves the frame);
// the tent weights are renormalised over the covered pixels, so a footprint
// clipped by the frame edge keeps its energy.
//
// GPU shape.  A photon has up to max_bounces segments of up to 4096 steps each,
// so per-photon work varies by three orders of magnitude.  Each warp traces 32
// photons at a time and only records segments (origin, direction, step length,
// power, M) in a per-warp shared-memory buffer; when the buffer fills (and when
// the 32 photons are done) the warp marches all buffered steps as one flat list
// -- lane t takes global step t, found by a binary search over the buffer's
// prefix sums of M -- so lanes stay busy whatever the segment lengths.  Steps
// next to each other in the list lie ~0.5 px apart on the same segment, so the
// lanes of a warp deposit into overlapping footprints; the optional warp
// aggregation merges equal film cells before the 64-bit atomics.
#include "photon_trace.cuh"

namespace sc {

namespace {

constexpr float kBeamRadius = 0.03f;  // R_BEAM (volume.rs:172)
constexpr uint32_t kMaxSteps = 4096u;

struct BeamSeg { f3 o, d; float ds, power; uint32_t m, lane; };
constexpr uint32_t kBeamSegs = 64;
struct alignas(16) BeamWarpSmem {
    BeamSeg seg[kBeamSegs];
    uint32_t start[kBeamSegs + 4];  // exclusive prefix of m; start[kBeamSegs] = total
    float4 payload[32];             // per-lane CMF (x, y, z) and bin of its photon
};

__host__ __device__ __forceinline__ size_t beam_offset(const PhotonParams& p, uint32_t mask_words) {
    const size_t b = p.n_prims * sizeof(sc_primitive) + p.n_planes * sizeof(sc_plane) +
                     p.n_mats * sizeof(sc_material) + 3 * kTableN * sizeof(float) + mask_words * sizeof(uint32_t);
    return (b + 15u) & ~size_t(15);
}

// March count of one segment (volume.rs:255-266).
__device__ __forceinline__ uint32_t march_count(const PhotonParams& p, f3 o, f3 d, float seg) {
    const f3 pend = add(o, mul(d, seg));
    float s0, t0, s1, t1;
    float mf;
    uint32_t extra;
    if (project(p.proj, o, s0, t0) && project(p.proj, pend, s1, t1)) {
        const float dx = (s1 - s0) * (float)p.width;
        const float dy = (t1 - t0) * (float)p.height;
        mf = ceilf(sqrtf(dx * dx + dy * dy) * 2.0f);
        extra = 1u;
    } else {
        mf = ceilf(seg * 80.0f);
        extra = 0u;
    }
    if (!(mf > 0.0f)) mf = 0.0f;
    mf = fminf(mf, (float)kMaxSteps);
    const uint32_t m = (uint32_t)mf + extra;
    return m < 1u ? 1u : (m > kMaxSteps ? kMaxSteps : m);
}

// splat_transverse (volume.rs:174-218): tent footprint renormalised over the
// covered pixels; value = col * w (XYZ film) or weight * w into the bin.
template <bool SPEC, int AGG>
__device__ __forceinline__ void splat_transverse(const PhotonParams& p, uint32_t* smask, float s, float t, float c0,
                                                 float c1, float c2, float weight, uint32_t bin, float radius_px) {
    const float cx = s * (float)p.width - 0.5f;
    const float cy = (1.0f - t) * (float)p.height - 0.5f;
    const float r = fmaxf(radius_px, 0.5f);
    const int wmax = (int)p.width - 1, hmax = (int)p.height - 1;
    const int x0 = (int)fmaxf(floorf(cx - r), 0.0f);
    const int x1 = min(max((int)ceilf(cx + r), 0), wmax);
    const int y0 = (int)fmaxf(floorf(cy - r), 0.0f);
    const int y1 = min(max((int)ceilf(cy + r), 0), hmax);
    float wsum = 0.0f;
    for (int py = y0; py <= y1; ++py)
        for (int px = x0; px <= x1; ++px) {
            const float dx = (float)px - cx, dy = (float)py - cy;
            wsum += fmaxf(1.0f - sqrtf(dx * dx + dy * dy) / r, 0.0f);
        }
    if (wsum <= 0.0f) {
        const int px = min(max((int)roundf(cx), 0), wmax), py = min(max((int)roundf(cy), 0), hmax);
        deposit<SPEC, AGG>(p, smask, true, (uint32_t)px, (uint32_t)py, SPEC ? weight : 1.0f, c0, c1, c2, bin);
        return;
    }
    const float inv = 1.0f / wsum;
    for (int py = y0; py <= y1; ++py)
        for (int px = x0; px <= x1; ++px) {
            const float dx = (float)px - cx, dy = (float)py - cy;
            const float w = fmaxf(1.0f - sqrtf(dx * dx + dy * dy) / r, 0.0f) * inv;
            deposit<SPEC, AGG>(p, smask, w > 0.0f, (uint32_t)px, (uint32_t)py, SPEC ? weight * w : w, c0, c1, c2,
                               bin);
        }
}

// One march step k of a buffered segment (volume.rs:268-307).
template <bool SPEC, int AGG>
__device__ __forceinline__ void beam_step(const PhotonParams& p, uint32_t* smask, const BeamSeg& B, float4 pay,
                                          uint32_t k) {
    const float dist = ((float)k + 0.5f) * B.ds;
    const f3 q = add(B.o, mul(B.d, dist));
    float s, t;
    if (!project(p.proj, q, s, t)) return;
    const uint32_t px = min((uint32_t)(s * (float)p.width), p.width - 1u);
    const uint32_t py = min((uint32_t)((1.0f - t) * (float)p.height), p.height - 1u);
    const f3 to = sub(p.proj.o, q);
    const float dd = fmaxf(length(to), 1e-3f);
    if (p.zbuf && !(dd < p.zbuf[py * p.width + px])) return;
    const f3 view = vdiv(to, dd);
    const float phase = phase_hg(p.g, dot(B.d, view));
    const float trans = expf(-p.sigma_t * dd);
    const float weight = B.power * p.sigma_s * phase * trans / (dd * dd) * B.ds;
    f3 perp = cross(view, mk(0.0f, 1.0f, 0.0f));
    if (dot(perp, perp) < 1e-8f) perp = cross(view, mk(1.0f, 0.0f, 0.0f));
    perp = mul(normalize(perp), kBeamRadius);
    float s2, t2, radius = 1.0f;
    if (project(p.proj, add(q, perp), s2, t2)) {
        const float dpx = (s2 - s) * (float)p.width, dpy = (t2 - t) * (float)p.height;
        radius = fminf(fmaxf(sqrtf(dpx * dpx + dpy * dpy), 1.5f), 24.0f);
    }
    float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
    if (!SPEC) { c0 = pay.x * weight; c1 = pay.y * weight; c2 = pay.z * weight; }
    splat_transverse<SPEC, AGG>(p, smask, s, t, c0, c1, c2, weight, __float_as_uint(pay.w), radius);
}

// March every step of the n buffered segments as one flat list.
template <bool SPEC, int AGG>
__device__ __forceinline__ void beam_flush(const PhotonParams& p, BeamWarpSmem& ws, uint32_t n, uint32_t* smask) {
    const uint32_t lane = threadIdx.x & 31u;
    __syncwarp();
    const uint32_t m0 = lane < n ? ws.seg[lane].m : 0u;
    const uint32_t m1 = lane + 32u < n ? ws.seg[lane + 32u].m : 0u;
    uint32_t i0 = m0, i1 = m1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t a = __shfl_up_sync(0xffffffffu, i0, o), b = __shfl_up_sync(0xffffffffu, i1, o);
        if ((int)lane >= o) { i0 += a; i1 += b; }
    }
    const uint32_t tot0 = __shfl_sync(0xffffffffu, i0, 31), tot1 = __shfl_sync(0xffffffffu, i1, 31);
    ws.start[lane] = i0 - m0;
    ws.start[lane + 32u] = tot0 + i1 - m1;
    if (lane == 0) ws.start[kBeamSegs] = tot0 + tot1;
    __syncwarp();
    const uint32_t total = tot0 + tot1;
    for (uint32_t t = lane; t < total; t += 32u) {
        uint32_t lo = 0, hi = n;  // start[lo] <= t < start[hi]
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (ws.start[mid] <= t) lo = mid; else hi = mid;
        }
        const BeamSeg B = ws.seg[lo];
        beam_step<SPEC, AGG>(p, smask, B, ws.payload[B.lane], t - ws.start[lo]);
    }
    __syncwarp();
}

// 32 photons of one warp (lane = photon): transport with segments recorded,
// then marched by beam_flush.
template <bool SPEC, int AGG>
__device__ __forceinline__ void trace_beam_warp(const PhotonParams& p, const SceneView& S, const float* cmf,
                                                uint32_t idx, bool valid, uint32_t* smask, BeamWarpSmem& ws) {
    const uint32_t lane = threadIdx.x & 31u;
    Rng r = Rng::make(idx, p.seed);
    const float r1 = r.f32();
    const float r2 = r.f32();
    f3 o = add(add(p.corner, mul(p.bu, r1)), mul(p.bv, r2));
    const float lambda = p.lambda_min + p.lambda_range * r.f32();
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    uint32_t bin = 0;
    photon_payload(p, cmf, lambda, cx, cy, cz, bin, SPEC);
    ws.payload[lane] = make_float4(cx, cy, cz, __uint_as_float(bin));
    f3 d = p.bdir;
    float power = 1.0f;
    bool alive = valid;
    uint32_t n = 0, n_glass = 0xFFFFFFFFu;
    float n_cached = 1.0f;
    for (uint32_t b = 0;; ++b) {
        const unsigned live = b < p.max_bounces ? __ballot_sync(0xffffffffu, alive) : 0u;
        // one flush site (keeps beam_flush inlined): when the buffer cannot take
        // another 32 segments, and once when the 32 photons are done
        if (n > kBeamSegs - 32u || (!live && n)) {
            beam_flush<SPEC, AGG>(p, ws, n, smask);
            n = 0;
        }
        if (!live) break;
        Hit h;
        uint32_t mi = 0;
        bool any = false;
        if (alive) {
            any = scene_hit(S, o, d, h, mi);
            const float seg = any ? h.t : p.max_dist;
            const uint32_t m = march_count(p, o, d, seg);
            BeamSeg& B = ws.seg[n + __popc(live & ((1u << lane) - 1u))];
            B.o = o; B.d = d; B.ds = seg / (float)m; B.power = power; B.m = m; B.lane = lane;
        }
        n += __popc(live);
        if (alive) {
            if (any) {
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
            } else {
                alive = false;
            }
        }
    }
}

template <bool SPEC, int AGG>
__global__ void __launch_bounds__(256, 4) beam_kernel(const PhotonParams p, uint32_t mask_words) {
    extern __shared__ __align__(16) unsigned char smem[];
    const float* cmf;
    uint32_t* smask;
    const SceneView S = load_scene(p, smem, &cmf, &smask, mask_words);
    BeamWarpSmem* ws = reinterpret_cast<BeamWarpSmem*>(smem + beam_offset(p, mask_words));
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + warp) * 32u; base < p.photon_count; base += warps * 32u)
        trace_beam_warp<SPEC, AGG>(p, S, cmf, p.photon_base + base + lane, base + lane < p.photon_count, smask,
                                   ws[warp]);
    if (smask) {
        __syncthreads();
        for (uint32_t w = threadIdx.x; w < mask_words; w += blockDim.x)
            if (smask[w]) atomicOr(p.flags + w, smask[w]);
    }
}

using BeamKernelFn = void (*)(const PhotonParams, uint32_t);

BeamKernelFn beam_fn(bool spec, int agg) {
    if (spec) return agg ? beam_kernel<true, 1> : beam_kernel<true, 0>;
    return agg ? beam_kernel<false, 1> : beam_kernel<false, 0>;
}

size_t beam_smem(const PhotonParams& p, uint32_t mask_words) {
    return beam_offset(p, mask_words) + 8 * sizeof(BeamWarpSmem);
}

}  // namespace

int beam_occupancy_blocks(const LaunchShape& shape, bool spectral, size_t smem) {
    int n = 0;
    const void* fn = reinterpret_cast<const void*>(beam_fn(spectral, shape.aggregate));
    const size_t total = smem + 16 + 8 * sizeof(BeamWarpSmem);
    if (total > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)total);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, (int)shape.block, total) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

cudaError_t launch_beam(const PhotonParams& p, const LaunchShape& shape, cudaStream_t s) {
    if (p.photon_count == 0) return cudaSuccess;
    const uint32_t mw = photon_mask_words(p);
    const bool spec = p.channels != 3u || p.bins != 0u;
    const uint32_t need = (p.photon_count + 255u) / 256u;
    const uint32_t grid = need < shape.grid ? need : shape.grid;
    beam_fn(spec, shape.aggregate)<<<grid, 256, beam_smem(p, mw), s>>>(p, mw);
    return cudaGetLastError();
}

}  // namespace sc
