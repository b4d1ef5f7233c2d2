// Wavefront hero-wavelength camera path tracer.
//
// Restates CpuTracer::sample_pixel / accumulate (spectral-core/src/tracer.rs:44-141;
// GPU mirror spectral-gpu/src/shaders/trace.wgsl:419-537) as a wavefront:
//   generate  one path per (pixel, sample): stream key mix2(pixel, sample index),
//             jittered primary ray, hero-comb wavelength draw (spectrum.rs:20-32);
//   intersect nearest scene hit (+ the optional spherical emitter) per ray,
//             in the kernel that shades it (primary rays where they are made;
//             later rays as the next bounce reads them from the dense queue);
//   shade     background / emission at termination, Fresnel / refract / TIR or
//             Lambertian scatter, dispersion collapse to the hero lane, optional
//             Russian roulette; survivors are compacted into the next queue with
//             warp ballots, one atomic per block and shared-memory staging so the
//             SoA writes are contiguous;
//   tail      the few paths alive after the compacted bounces finish in one
//             launch, kept compacted per CTA bounce by bounce;
//   accumulate each pixel's samples summed in sample order (the CPU's order), so
//             the image is deterministic and, for scenes without Lambertian
//             surfaces, bit-identical to the CPU tracer.
// Queue counts stay on the device: the launch sequence of an accumulate call is
// fixed, needs no host synchronisation and is replayed from a CUDA graph.
#include <algorithm>

#include "internal.h"
#include "tracer.h"

namespace sc {

namespace {

constexpr int kShadeThreads = 256;
// Shade and tail CTAs resident per SM: 5 (48 registers, small spills) hides
// more of their queue-read and shared-memory latency than 4 (64 registers):
// accumulate(64) at 1280x720 5.83 -> 5.37 ms; 6 or 8 tail CTAs spill more
// and are slower again.
constexpr int kStageCtasPerSm = 5;
constexpr float kLambdaMin = 380.0f, kLambdaRange = 350.0f;

struct TracerSmem {
    TracerParams p;
    float tables[5 * kTableN];
    sc_primitive prims[SC_MAX_PRIMS];
    sc_material mats[SC_MAX_PRIMS];
    float4 bounds[SC_MAX_PRIMS];
};

// Stage params, scene records and sensor tables in shared memory.  Planes live
// after the fixed part (dynamic size).
__device__ __forceinline__ SceneView load_tracer(const TracerParams* gp, TracerSmem& s, sc_plane* planes) {
    const uint32_t tid = threadIdx.x;
    if (tid == 0) s.p = *gp;
    for (uint32_t i = tid; i < 5u * kTableN; i += blockDim.x) s.tables[i] = gp->tables[i];
    __syncthreads();
    for (uint32_t i = tid; i < s.p.n_prims; i += blockDim.x) s.prims[i] = s.p.prims[i];
    for (uint32_t i = tid; i < s.p.n_mats; i += blockDim.x) s.mats[i] = s.p.mats[i];
    for (uint32_t i = tid; i < s.p.n_prims; i += blockDim.x) s.bounds[i] = s.p.bounds[i];
    for (uint32_t i = tid; i < s.p.n_planes; i += blockDim.x) planes[i] = s.p.planes[i];
    __syncthreads();
    SceneView S;
    S.prims = s.prims; S.planes = planes; S.mats = s.mats; S.n_prims = s.p.n_prims;
    return S;
}

__device__ __forceinline__ float lane_lambda(float u, int k) {
    // SpectralSample::from_hero_u: (u*RANGE + k*RANGE/4).rem_euclid(RANGE).
    // For 0 <= x < 2 RANGE (every u in [0, 1)) the remainder is x or x - RANGE,
    // and x - RANGE is exact there (RANGE <= x < 2 RANGE), so it equals fmodf's
    // exact remainder without its general loop.
    const float x = u * kLambdaRange + (float)k * (kLambdaRange / 4.0f);
    float off;
    if (x >= 0.0f && x < 2.0f * kLambdaRange) {
        off = x >= kLambdaRange ? x - kLambdaRange : x;
    } else {
        off = fmodf(x, kLambdaRange);
        if (off < 0.0f) off += kLambdaRange;
    }
    return kLambdaMin + off;
}

// XYZ of a terminated comb whose lanes carry radiance rad_k = tp_k * e * S(lambda_k).
__device__ __forceinline__ void comb_xyz(const TracerSmem& s, float u, float tp, uint32_t valid, float e,
                                         float out[3]) {
    const float pdf = 1.0f / kLambdaRange;
    const float* ill = s.tables + (s.p.illuminant == 1u ? 4 : 3) * kTableN;
    // dividing by 1 or 4 lanes is scaling by a power of two: the same rounded
    // quotient as the division
    const bool pow2 = valid == 1u || valid == 4u;
    const float inv_valid = valid == 4u ? 0.25f : 1.0f;
    float x = 0.0f, y = 0.0f, z = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float lam = lane_lambda(u, k);
        const float tk = (k == 0 || valid > 1u) ? tp : 0.0f;
        const float rad = 0.0f + tk * e * tab_sample(ill, lam);
        const float q = rad / pdf;
        const float wk = pow2 ? q * inv_valid : q / (float)valid;
        x += tab_sample(s.tables, lam) * wk;
        y += tab_sample(s.tables + kTableN, lam) * wk;
        z += tab_sample(s.tables + 2 * kTableN, lam) * wk;
    }
    out[0] = x; out[1] = y; out[2] = z;
}

// Whether a ray certainly misses a bounding sphere (centre, radius^2 in b):
// the origin is outside it and the line's closest approach at t >= 0 is
// outside it.  The sphere is inflated on the host (1 % + 1e-3) far beyond the
// rounding of these products; origins farther than 100 radii are not culled
// (the products would cancel), so a culled solid is one that solid_hit would
// not hit either.
__device__ __forceinline__ bool misses_bound(float4 b, f3 o, f3 d) {
    if (!(b.w < __int_as_float(0x7f800000))) return false;
    const f3 oc = mk(b.x - o.x, b.y - o.y, b.z - o.z);
    const float l2 = dot(oc, oc);
    if (!(l2 > b.w) || l2 > 1e4f * b.w) return false;
    const float bb = dot(oc, d);
    if (bb <= 0.0f) return true;  // moving away from the centre, from outside
    return (l2 - b.w) * dot(d, d) > bb * bb;
}

// Scene::intersect (scene_hit) skipping convex solids whose bounding sphere
// the ray misses: the same nearest hit, fewer plane tests.
__device__ __forceinline__ bool scene_hit_bounded(const TracerSmem& s, const SceneView& S, f3 o, f3 d, Hit& best,
                                                  uint32_t& mat) {
    bool any = false;
    float closest = __int_as_float(0x7f800000);
    for (uint32_t i = 0; i < S.n_prims; ++i) {
        const sc_primitive& pr = S.prims[i];
        if (pr.kind == 1u && misses_bound(s.bounds[i], o, d)) continue;
        Hit h;
        bool ok = pr.kind == 0u ? sphere_hit(pr, o, d, 1e-3f, closest, h)
                : (pr.kind == 1u ? solid_hit(S, pr, o, d, 1e-3f, closest, h) : false);
        if (ok) { closest = h.t; best = h; mat = pr.material; any = true; }
    }
    return any;
}

// Nearest hit of one ray: scene records and the optional emitter sphere.
// info = material | front_face << 16 | kind << 24 (0 miss, 1 surface, 2 emitter).
__device__ __forceinline__ void trace_hit(const TracerSmem& s, const SceneView& S, f3 o, f3 d, float& t, f3& n,
                                          uint32_t& info) {
    Hit h;
    uint32_t mi = 0;
    const bool any = scene_hit_bounded(s, S, o, d, h, mi);
    uint32_t kind = any ? 1u : 0u;
    t = any ? h.t : __int_as_float(0x7f800000);
    if (s.p.em_radius > 0.0f) {
        sc_primitive em;
        em.center[0] = s.p.em_center.x; em.center[1] = s.p.em_center.y; em.center[2] = s.p.em_center.z;
        em.radius = s.p.em_radius;
        Hit he;
        if (sphere_hit(em, o, d, 1e-3f, t, he)) { kind = 2u; t = he.t; }
    }
    n = h.normal;
    info = mi | (((any && h.front_face) ? 1u : 0u) << 16) | (kind << 24);
}

// State of one path between bounces (the ray queue's fields).
struct PathState {
    f3 o, d;
    float tp, u;
    uint32_t rs, id, flags;  // RNG state, path id, valid lanes | depth << 8
};

// Shade one path at `bounce` given its hit: background / emission ends the
// path (its XYZ goes to result[id]); a surface scatters it (Fresnel / refract /
// TIR or Lambertian, dispersion collapse, Russian roulette).  Returns whether
// the path continues.
__device__ __forceinline__ bool shade_path(const TracerSmem& s, const SceneView& S, uint32_t bounce, PathState& P,
                                           float t, f3 n, uint32_t info, float* result) {
    const uint32_t kind = info >> 24;
    uint32_t valid = P.flags & 0xFFu;
    if (kind != 1u) {
        float e;
        if (kind == 0u) e = s.p.background + ((s.p.has_horizon && P.d.y > 0.0f) ? s.p.horizon : 0.0f);
        else e = s.p.em_scale;
        float xyz[3];
        comb_xyz(s, P.u, P.tp, valid, e, xyz);
        result[3 * P.id] = xyz[0]; result[3 * P.id + 1] = xyz[1]; result[3 * P.id + 2] = xyz[2];
        return false;
    }
    const sc_material& m = S.mats[info & 0xFFFFu];
    Hit h;
    h.t = t;
    h.point = add(P.o, mul(P.d, t));
    h.normal = n;
    h.front_face = ((info >> 16) & 1u) != 0u;
    const float nh = m.kind == 1u ? glass_n(m.glass, s.p.spectral ? lane_lambda(P.u, 0) : 550.0f) : 1.0f;
    Rng r;
    r.state = P.rs;
    f3 nd;
    float w;
    scatter(m, P.d, h, nh, r, nd, w);
    P.tp *= w;
    if (m.kind == 1u && valid > 1u) valid = 1u;
    const uint32_t depth = bounce + 1u;
    bool survive = depth < s.p.max_depth;
    if (s.p.rr_start && depth >= s.p.rr_start) {
        const float qv = fminf(P.tp, 0.95f);
        if (!(r.f32() < qv)) survive = false;
        else P.tp = P.tp / qv;
    }
    P.o = h.point; P.d = nd; P.rs = r.state;
    P.flags = valid | (depth << 8);
    return survive;
}

// One compacted bounce: each path's ray is intersected and shaded here, and
// the survivors are compacted into the next ray queue (no hit queue: the
// bounce that reads a ray intersects it, from the dense queue).
// GEN: the first bounce with no queue in: each path's primary ray is made here
// (stream key mix2(pixel, sample index), jittered through the pixel, hero-comb
// draw), intersected in place and shaded.  Paths of a wave are numbered
// sample-major (path i = sample s of wave pixel j with i = s * n_pixels + j):
// neighbouring threads trace neighbouring pixels, and the per-pixel sums read
// the results coalesced.  counts[1..] are zero at entry.
template <bool GEN>
__global__ void __launch_bounds__(kShadeThreads, kStageCtasPerSm) tr_shade(const TracerParams* __restrict__ gp, uint32_t bounce,
                                                          RayQueue q, RayQueue out,
                                                          uint32_t* counts, float* result, uint32_t first_pixel,
                                                          uint32_t n_pixels, uint32_t n_paths,
                                                          const uint32_t* __restrict__ base) {
    __shared__ TracerSmem s;
    __shared__ uint32_t warp_base[kShadeThreads / 32 + 1];
    __shared__ uint32_t block_base;
    __shared__ float st_f[8][kShadeThreads];      // staged survivors: ox oy oz dx dy dz tp u
    __shared__ uint32_t st_u[3][kShadeThreads];   // rng id flags
    extern __shared__ __align__(16) unsigned char dyn[];
    if (GEN && blockIdx.x == 0 && threadIdx.x == 0) counts[0] = n_paths;
    const uint32_t n = GEN ? n_paths : counts[bounce];
    if (blockIdx.x * blockDim.x >= n) return;  // nothing queued for this CTA (late bounces)
    const SceneView S = load_tracer(gp, s, reinterpret_cast<sc_plane*>(dyn));
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t b0 = GEN ? *base : 0u;
    for (uint32_t tile = blockIdx.x * blockDim.x; tile < n; tile += gridDim.x * blockDim.x) {
        const uint32_t i = tile + threadIdx.x;
        bool survive = false;
        PathState P;
        P.o = P.d = mk(0.0f, 0.0f, 0.0f);
        P.tp = P.u = 0.0f;
        P.rs = P.id = P.flags = 0u;
        if (i < n && GEN) {
            const uint32_t smp = i / n_pixels, pixel = first_pixel + (i - smp * n_pixels);
            const uint32_t px = pixel % s.p.width, py = pixel / s.p.width;
            Rng r = Rng::make(mix2(pixel, b0 + smp), s.p.seed);
            const float fs = ((float)px + r.f32()) / (float)s.p.width;
            const float ft = 1.0f - ((float)py + r.f32()) / (float)s.p.height;
            P.u = r.f32();
            P.o = ld3(s.p.cam.origin);
            P.d = primary_dir(s.p.cam, fs, ft);
            P.rs = r.state; P.tp = 1.0f; P.id = i; P.flags = 4u;
            result[3 * i] = 0.0f; result[3 * i + 1] = 0.0f; result[3 * i + 2] = 0.0f;
            float t;
            f3 nrm;
            uint32_t info;
            trace_hit(s, S, P.o, P.d, t, nrm, info);
            if ((info >> 24) != 1u) nrm = mk(0.0f, 0.0f, 0.0f);
            survive = shade_path(s, S, 0u, P, t, nrm, info, result);
        } else if (i < n) {
            P.o = mk(q.ox[i], q.oy[i], q.oz[i]);
            P.d = mk(q.dx[i], q.dy[i], q.dz[i]);
            P.tp = q.tp[i]; P.u = q.u[i]; P.rs = q.rng[i]; P.id = q.id[i]; P.flags = q.flags[i];
            float t;
            f3 nrm;
            uint32_t info;
            trace_hit(s, S, P.o, P.d, t, nrm, info);
            if ((info >> 24) != 1u) nrm = mk(0.0f, 0.0f, 0.0f);
            survive = shade_path(s, S, bounce, P, t, nrm, info, result);
        }
        const f3 o = P.o, d = P.d;
        const float tp = P.tp, u = P.u;
        const uint32_t rs = P.rs, id = P.id, flags = P.flags;
        // block-level compaction: ballot per warp, prefix over warps, one atomic
        const unsigned ball = __ballot_sync(0xffffffffu, survive);
        const uint32_t rank = __popc(ball & ((1u << lane) - 1u));
        if (lane == 0) warp_base[warp] = __popc(ball);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
            for (int w = 0; w < kShadeThreads / 32; ++w) { const uint32_t c = warp_base[w]; warp_base[w] = acc; acc += c; }
            warp_base[kShadeThreads / 32] = acc;
            block_base = acc ? atomicAdd(&counts[bounce + 1], acc) : 0u;
        }
        __syncthreads();
        if (survive) {
            const uint32_t j = warp_base[warp] + rank;
            st_f[0][j] = o.x; st_f[1][j] = o.y; st_f[2][j] = o.z;
            st_f[3][j] = d.x; st_f[4][j] = d.y; st_f[5][j] = d.z;
            st_f[6][j] = tp; st_f[7][j] = u;
            st_u[0][j] = rs; st_u[1][j] = id; st_u[2][j] = flags;
        }
        __syncthreads();
        const uint32_t total = warp_base[kShadeThreads / 32];
        if (threadIdx.x < total) {
            const uint32_t j = threadIdx.x, g = block_base + j;
            out.ox[g] = st_f[0][j]; out.oy[g] = st_f[1][j]; out.oz[g] = st_f[2][j];
            out.dx[g] = st_f[3][j]; out.dy[g] = st_f[4][j]; out.dz[g] = st_f[5][j];
            out.tp[g] = st_f[6][j]; out.u[g] = st_f[7][j];
            out.rng[g] = st_u[0][j]; out.id[g] = st_u[1][j]; out.flags[g] = st_u[2][j];
        }
        __syncthreads();
    }
}

// Late bounces: by the third bounce only a few per cent of a wave's paths are
// alive, and a launch pair per bounce costs more than the work.  The tail runs
// them in one launch: each CTA holds up to 256 paths in shared memory with the
// live ones at the front, runs one bounce of all of them (the same hit and
// shade code, so the image is unchanged), compacts the survivors with warp
// ballots, and refills the free slots from the queue with one claim per CTA
// (counter counts[max_depth + 1], zero at entry), so its warps stay full while
// the paths end after different numbers of bounces.  Segments after each
// path's first tail bounce are added to counts[first + 1].
__global__ void __launch_bounds__(256, kStageCtasPerSm) tr_tail(const TracerParams* __restrict__ gp, uint32_t first,
                                                                RayQueue q, uint32_t* counts, float* result) {
    __shared__ TracerSmem s;
    __shared__ float sf[8][256];    // ox oy oz dx dy dz tp u
    __shared__ uint32_t su[3][256]; // rng id flags
    __shared__ uint32_t warp_base[8 + 1];
    __shared__ uint32_t claim_base;
    extern __shared__ __align__(16) unsigned char dyn[];
    const uint32_t n = counts[first];
    if (blockIdx.x * blockDim.x >= n) return;
    const SceneView S = load_tracer(gp, s, reinterpret_cast<sc_plane*>(dyn));
    uint32_t* claim = counts + s.p.max_depth + 1;
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    uint32_t live = 0, segs = 0;
    for (;;) {
        if (t == 0) claim_base = atomicAdd(claim, 256u - live);
        __syncthreads();
        const uint32_t base = claim_base;
        const uint32_t got = base >= n ? 0u : min(256u - live, n - base);
        if (t >= live && t < live + got) {  // coalesced: consecutive slots take consecutive paths
            const uint32_t i = base + (t - live);
            sf[0][t] = q.ox[i]; sf[1][t] = q.oy[i]; sf[2][t] = q.oz[i];
            sf[3][t] = q.dx[i]; sf[4][t] = q.dy[i]; sf[5][t] = q.dz[i];
            sf[6][t] = q.tp[i]; sf[7][t] = q.u[i];
            su[0][t] = q.rng[i]; su[1][t] = q.id[i]; su[2][t] = q.flags[i];
        }
        live += got;
        __syncthreads();
        if (live == 0) break;
        bool survive = false;
        PathState P;
        P.o = P.d = mk(0.0f, 0.0f, 0.0f);
        P.tp = P.u = 0.0f;
        P.rs = P.id = P.flags = 0u;
        if (t < live) {
            P.o = mk(sf[0][t], sf[1][t], sf[2][t]);
            P.d = mk(sf[3][t], sf[4][t], sf[5][t]);
            P.tp = sf[6][t]; P.u = sf[7][t]; P.rs = su[0][t]; P.id = su[1][t]; P.flags = su[2][t];
            const uint32_t b = (P.flags >> 8) & 0xFFu;  // the bounce this path is at
            float th;
            f3 nrm;
            uint32_t info;
            trace_hit(s, S, P.o, P.d, th, nrm, info);
            if (b > first) ++segs;  // counts[first] already holds the first tail bounce's rays
            survive = shade_path(s, S, b, P, th, nrm, info, result);
        }
        const unsigned ball = __ballot_sync(0xffffffffu, survive);
        if (lane == 0) warp_base[warp] = __popc(ball);
        __syncthreads();  // every slot has been read
        if (t == 0) {
            uint32_t acc = 0;
            for (int w = 0; w < 8; ++w) { const uint32_t c = warp_base[w]; warp_base[w] = acc; acc += c; }
            warp_base[8] = acc;
        }
        __syncthreads();
        if (survive) {
            const uint32_t j = warp_base[warp] + __popc(ball & ((1u << lane) - 1u));
            sf[0][j] = P.o.x; sf[1][j] = P.o.y; sf[2][j] = P.o.z;
            sf[3][j] = P.d.x; sf[4][j] = P.d.y; sf[5][j] = P.d.z;
            sf[6][j] = P.tp; sf[7][j] = P.u;
            su[0][j] = P.rs; su[1][j] = P.id; su[2][j] = P.flags;
        }
        live = warp_base[8];
        __syncthreads();  // the survivors are in place (and warp_base is read) before the next claim
    }
    for (int o = 16; o > 0; o >>= 1) segs += __shfl_xor_sync(0xffffffffu, segs, o);
    if (lane == 0 && segs) atomicAdd(counts + first + 1, segs);
}

// Per-pixel sample sum in sample order (tracer.rs:121-135), added to the running
// sum.  One thread per (pixel, channel) of the wave: consecutive threads read
// consecutive floats of each sample (coalesced), and each adds its samples in
// sample order.
__global__ void __launch_bounds__(256) tr_accumulate(uint32_t first_pixel, uint32_t n_pixels, uint32_t spp,
                                                     const float* __restrict__ result, float* sum,
                                                     const uint32_t* __restrict__ counts, uint32_t max_depth,
                                                     unsigned long long* segments) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j == 0) {
        unsigned long long t = 0;
        for (uint32_t b = 0; b < max_depth; ++b) t += counts[b];
        atomicAdd(segments, t);  // both wave chains add here
    }
    const uint32_t n = 3u * n_pixels;
    if (j >= n) return;
    float a = 0.0f;
#pragma unroll 16
    for (uint32_t s = 0; s < spp; ++s) a += result[(size_t)s * n + j];  // loads run ahead; adds in sample order
    sum[3u * (size_t)first_pixel + j] += a;
}

// AccumBuffer::mean (spectral-core/src/lib.rs:16-20): each sum divided by the
// sample count (an IEEE division, as the host would do it).
__global__ void __launch_bounds__(256) tr_mean(const float* __restrict__ sum, float* __restrict__ out, size_t n,
                                               float count) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = sum[i] / count;
}

}  // namespace

cudaError_t launch_tracer_mean(const float* sum, float* out, size_t n, float count, int sms, cudaStream_t st) {
    const size_t blocks = std::min<size_t>((n + 255) / 256, (size_t)sms * 8);
    if (blocks == 0) return cudaSuccess;
    tr_mean<<<(unsigned)blocks, 256, 0, st>>>(sum, out, n, count);
    return cudaGetLastError();
}

size_t tracer_dyn_smem(uint32_t n_planes) { return (size_t)(n_planes ? n_planes : 1u) * sizeof(sc_plane); }

int tracer_grid(int sms) {
    int a = 0, b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, tr_tail, 256, tracer_dyn_smem(SC_MAX_PLANES));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, tr_shade<false>, kShadeThreads,
                                                  tracer_dyn_smem(SC_MAX_PLANES));
    int c = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, tr_shade<true>, kShadeThreads,
                                                  tracer_dyn_smem(SC_MAX_PLANES));
    int k = a < b ? a : b;
    k = k < c ? k : c;
    return sms * (k > 0 ? k : 1);
}

cudaError_t launch_tracer_wave(const TracerParams* d_params, const TracerLaunch& L, uint32_t first_pixel,
                               uint32_t n_pixels, cudaStream_t st) {
    const uint32_t n_paths = n_pixels * L.spp;
    const size_t dyn = tracer_dyn_smem(L.n_planes);
    // wavefront with compaction for the first bounces, then the tail in place;
    // the first bounce makes, intersects and shades the primary rays in one kernel
    const uint32_t wave_bounces = L.max_depth < L.wave_bounces ? L.max_depth : L.wave_bounces;
    // bounce b intersects and shades the rays of bounce b and queues its
    // compacted survivors (ray queues alternate)
    for (uint32_t b = 0; b < wave_bounces; ++b) {
        const RayQueue& in = (b & 1u) ? L.qb : L.qa;
        const RayQueue& out = (b & 1u) ? L.qa : L.qb;
        if (b == 0) {
            // the first bounce makes its primary rays itself: no queue in; later
            // bounces (and the tail's claim counter) count from zero
            cudaError_t e = cudaMemsetAsync(L.counts + 1, 0, (L.max_depth + 1) * sizeof(uint32_t), st);
            if (e != cudaSuccess) return e;
            tr_shade<true><<<L.grid, kShadeThreads, dyn, st>>>(d_params, 0u, in, out, L.counts, L.result, first_pixel,
                                                              n_pixels, n_paths, L.d_base);
        } else {
            tr_shade<false><<<L.grid, kShadeThreads, dyn, st>>>(d_params, b, in, out, L.counts, L.result, 0u, 1u, 0u,
                                                               L.d_base);
        }
    }
    if (L.max_depth > wave_bounces)
        tr_tail<<<L.grid, 256, dyn, st>>>(d_params, wave_bounces, (wave_bounces & 1u) ? L.qb : L.qa, L.counts,
                                          L.result);
    tr_accumulate<<<(3 * n_pixels + 255) / 256, 256, 0, st>>>(first_pixel, n_pixels, L.spp, L.result, L.sum, L.counts,
                                                               L.max_depth, L.segments);
    return cudaGetLastError();
}

}  // namespace sc
