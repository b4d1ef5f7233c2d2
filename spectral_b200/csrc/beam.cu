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
// the 32 photons are done) the warp marches all buffered steps as one flat list:
// 32 steps at a time are set up one per lane (step t found by a binary search
// over the buffer's prefix sums of M), then each in-frame step is splatted by
// the whole warp, lanes spread over its footprint box (the tent sum is added
// up by the step's own lane during the setup, row by row like the reference).
// Lanes stay converged whatever the segment lengths and footprint sizes, and
// the 32 atomics of one warp instruction hit 32 distinct pixels.  Film width
// and height are below 2^16 (the box corner is packed into one word).
// |d| is d2 * rsqrt(d2) (within 2 ulp), |d| / r a multiply by 1/r and the
// tent's two sums fused, so a deposit can differ from the reference's in the
// last few bits.
#include "photon_trace.cuh"

namespace sc {

namespace {

constexpr float kBeamRadius = 0.03f;  // R_BEAM (volume.rs:172)
constexpr uint32_t kMaxSteps = 4096u;

struct BeamSeg { f3 o, d; float ds, power; uint32_t m, lane; };
// One march step ready to splat: footprint centre and 1 / radius in pixels,
// the step's colour (XYZ film) or weight and bin (spectral film), times the
// film's fixed-point scale (a power of two: exact, so a pixel's deposit
// fixed_scaled(c * w) is to_fixed(c_unscaled * w, scale)), the footprint
// box [x0, x0 + bw) x [y0, y0 + bh), the warp's lane layout over it (`rows` rows
// of bw lanes per pass; lane / bw = (lane * magic) >> 16) and the tent sum,
// all worked out one step per lane so the warp-wide splat does no division.
struct StepRec {
    float cx, cy, inv_r, c0, c1, c2;
    uint32_t bin, valid;  // valid: 0 none, 1 footprint, 2 whole colour on the centre pixel
    uint32_t x0y0;        // x0 | y0 << 16
    uint32_t box;         // bw | bh << 8 | rows << 16 | passes << 24 (bw, bh <= 49)
    uint32_t magic;       // ceil(2^16 / bw)
    float inv_wsum;       // 1 / sum of the tent over the box
};
constexpr uint32_t kBeamSegs = 64;
struct alignas(16) BeamWarpSmem {
    BeamSeg seg[kBeamSegs];
    uint32_t start[kBeamSegs + 4];  // exclusive prefix of m; start[kBeamSegs] = total
    float4 payload[32];             // per-lane CMF (x, y, z) and bin of its photon
    StepRec step[32];               // 32 march steps set up for splatting
};

// Work counters of an instrumented launch: segments, march steps, steps in
// frame (and not occluded), footprint pixels deposited.
struct BeamCounts { unsigned long long segments, steps, in_frame, deposits; };

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

// Tent weight max(1 - |d| / r, 0); the division is a multiply by 1/r (within
// an ulp of the reference's quotient), both sums fused multiply-adds.
__device__ __forceinline__ float tent(float dx2, float dy, float inv_r) {
    const float d2 = __fmaf_rn(dy, dy, dx2);
    const float d = d2 > 0.0f ? d2 * rsqrtf(d2) : 0.0f;  // |d| within 2 ulp
    return fmaxf(__fmaf_rn(-d, inv_r, 1.0f), 0.0f);
}

// Fixed-point value of an already scaled, non-negative deposit: the same
// integer as to_fixed(x, scale) for y = x * scale (scale a power of two), with
// the common case (y < 2^23) in two ALU operations and no sign test.
__device__ __forceinline__ unsigned long long fixed_scaled(float y) {
    if (y < 8388608.0f) return (unsigned long long)(__float_as_uint(y + 8388608.0f) - 0x4B000000u);
    return to_fixed(y, 1.0f);
}

// Dirty bits of the tiles under a footprint box, set by the step's own lane
// during the setup (most are already set, and mark_tile reads before it
// writes): its corners' tiles when it spans at most 2 tiles per axis, else
// every tile.
__device__ __forceinline__ void mark_box(const PhotonParams& p, uint32_t* smask, int x0, int y0, int x1, int y1) {
    const int tx0 = x0 >> 3, ty0 = y0 >> 3, tx1 = x1 >> 3, ty1 = y1 >> 3;
    if (tx1 - tx0 <= 1 && ty1 - ty0 <= 1) {
        mark_tile(p, smask, (uint32_t)(ty0 * (int)p.tiles_x + tx0));
        mark_tile(p, smask, (uint32_t)(ty0 * (int)p.tiles_x + tx1));
        mark_tile(p, smask, (uint32_t)(ty1 * (int)p.tiles_x + tx0));
        mark_tile(p, smask, (uint32_t)(ty1 * (int)p.tiles_x + tx1));
    } else {
        for (int ty = ty0; ty <= ty1; ++ty)
            for (int tx = tx0; tx <= tx1; ++tx) mark_tile(p, smask, (uint32_t)(ty * (int)p.tiles_x + tx));
    }
}

// Per-step setup (volume.rs:268-300), one lane per step: the step point, its
// projection, z-test, camera-connection weight and projected beam radius.
template <bool SPEC, bool COUNT>
__device__ __forceinline__ StepRec beam_step(const PhotonParams& p, uint32_t* smask, const BeamSeg& B, float4 pay,
                                             uint32_t k, BeamCounts& cnt) {
    StepRec R;
    R.valid = 0u;
    const float dist = ((float)k + 0.5f) * B.ds;
    const f3 q = add(B.o, mul(B.d, dist));
    float s, t;
    if (!project(p.proj, q, s, t)) return R;
    const uint32_t px = min((uint32_t)(s * (float)p.width), p.width - 1u);
    const uint32_t py = min((uint32_t)((1.0f - t) * (float)p.height), p.height - 1u);
    const f3 to = sub(p.proj.o, q);
    const float dd = fmaxf(length(to), 1e-3f);
    if (p.zbuf && !(dd < p.zbuf[py * p.width + px])) return R;
    if (COUNT) ++cnt.in_frame;
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
    // splat_transverse (volume.rs:174-186): centre, radius and box in pixels
    R.cx = s * (float)p.width - 0.5f;
    R.cy = (1.0f - t) * (float)p.height - 0.5f;
    const float r = fmaxf(radius, 0.5f);
    R.inv_r = 1.0f / r;
    const int x0 = (int)fmaxf(floorf(R.cx - r), 0.0f);
    const int x1 = min(max((int)ceilf(R.cx + r), 0), (int)p.width - 1);
    const int y0 = (int)fmaxf(floorf(R.cy - r), 0.0f);
    const int y1 = min(max((int)ceilf(R.cy + r), 0), (int)p.height - 1);
    const uint32_t bw = (uint32_t)(x1 - x0 + 1), bh = (uint32_t)(y1 - y0 + 1);
    R.x0y0 = (uint32_t)x0 | ((uint32_t)y0 << 16);
    const uint32_t rows = bw <= 32u ? 32u / bw : 1u;
    R.box = bw | (bh << 8) | (rows << 16) | (((bh + rows - 1u) / rows) << 24);
    R.magic = (65536u + bw - 1u) / bw;
    if (SPEC) { R.c0 = weight * p.scale; R.c1 = R.c2 = 0.0f; }
    else { R.c0 = pay.x * weight * p.scale; R.c1 = pay.y * weight * p.scale; R.c2 = pay.z * weight * p.scale; }
    R.bin = __float_as_uint(pay.w);
    // the tent sum over the box, row by row as the reference adds it
    float wsum = 0.0f;
    for (int py = y0; py <= y1; ++py) {
        const float dy = (float)py - R.cy;
        for (int px = x0; px <= x1; ++px) {
            const float dx = (float)px - R.cx;
            wsum += tent(dx * dx, dy, R.inv_r);
        }
    }
    R.valid = wsum > 0.0f ? 1u : 2u;
    if (!COUNT) mark_box(p, smask, x0, y0, x1, y1);  // covers the centre pixel of an empty tent too
    R.inv_wsum = wsum > 0.0f ? 1.0f / wsum : 0.0f;
    return R;
}

// Add one footprint pixel's share (w = tent / wsum) to the film.
template <bool SPEC>
__device__ __forceinline__ void deposit_pixel(const PhotonParams& p, uint32_t px, uint32_t py, const StepRec& R,
                                              float w) {
    unsigned long long* c = p.film + film_cell(px, py, p.tiles_x, p.channels);
    if (SPEC) {
        red_u64(c + R.bin, fixed_scaled(R.c0 * w));
    } else {
        red_u64(c, fixed_scaled(R.c0 * w));
        red_u64(c + 1, fixed_scaled(R.c1 * w));
        red_u64(c + 2, fixed_scaled(R.c2 * w));
    }
}

// Consecutive march steps often share a footprint box (steps are ~0.5 px apart,
// a box moves every pixel).  Over such a run each lane keeps its pixels'
// fixed-point sums in registers and issues one atomic per cell at the end of
// the run: the same integers reach the film, with fewer atomics.  Runs cover
// boxes up to 32 wide and 2 passes (footprint radius up to ~7 px).
struct BoxRun {
    uint32_t x0y0, box, bin;  // key; box == 0: no open run
    unsigned long long acc[2][3];
};

template <bool SPEC>
__device__ __forceinline__ void run_flush(const PhotonParams& p, BoxRun& run, uint32_t lane) {
    if (run.box == 0u) return;
    const int x0 = (int)(run.x0y0 & 0xFFFFu), y0 = (int)(run.x0y0 >> 16);
    const int bw = (int)(run.box & 0xFFu), bh = (int)((run.box >> 8) & 0xFFu), rows = (int)((run.box >> 16) & 0xFFu);
    const int lrow = (int)lane / bw, lcol = (int)lane - lrow * bw;
    if (lrow < rows) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int py = y0 + lrow + k * rows;
            if (py < y0 + bh) {
                unsigned long long* c = p.film + film_cell((uint32_t)(x0 + lcol), (uint32_t)py, p.tiles_x, p.channels);
                if (SPEC) {
                    red_u64(c + run.bin, run.acc[k][0]);
                } else {
                    red_u64(c, run.acc[k][0]);
                    red_u64(c + 1, run.acc[k][1]);
                    red_u64(c + 2, run.acc[k][2]);
                }
            }
        }
    }
    run.box = 0u;
}

// Whether a step can join a run (a footprint of at most 2 passes of <= 32 lanes).
__device__ __forceinline__ bool runnable(const StepRec& R) {
    return R.valid == 1u && (R.box & 0xFFu) <= 32u && (R.box >> 24) <= 2u;
}

template <bool SPEC>
__device__ __forceinline__ void run_add(const PhotonParams& p, BoxRun& run, const StepRec& R, uint32_t lane) {
    const uint32_t bin = SPEC ? R.bin : 0u;
    if (R.x0y0 != run.x0y0 || R.box != run.box || bin != run.bin) {
        run_flush<SPEC>(p, run, lane);
        run.x0y0 = R.x0y0; run.box = R.box; run.bin = bin;
#pragma unroll
        for (int k = 0; k < 2; ++k) run.acc[k][0] = run.acc[k][1] = run.acc[k][2] = 0ull;
    }
    const int x0 = (int)(R.x0y0 & 0xFFFFu), y0 = (int)(R.x0y0 >> 16);
    const int bw = (int)(R.box & 0xFFu), bh = (int)((R.box >> 8) & 0xFFu), rows = (int)((R.box >> 16) & 0xFFu);
    const int lrow = (int)((lane * R.magic) >> 16), lcol = (int)lane - lrow * bw;
    if (lrow >= rows) return;
    const float dx = (float)(x0 + lcol) - R.cx, dx2 = dx * dx, inv_r = R.inv_r, inv = R.inv_wsum;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int py = y0 + lrow + k * rows;
        if (py < y0 + bh) {
            const float w = tent(dx2, (float)py - R.cy, inv_r) * inv;
            if (w > 0.0f) {
                run.acc[k][0] += fixed_scaled(R.c0 * w);
                if (!SPEC) {
                    run.acc[k][1] += fixed_scaled(R.c1 * w);
                    run.acc[k][2] += fixed_scaled(R.c2 * w);
                }
            }
        }
    }
}

// splat_transverse (volume.rs:174-218) by the whole warp, its tent sum already
// known: lanes cover the footprint box (rows packed 32 / width at a time, or
// 32-column chunks of one row for boxes wider than 32) and deposit their pixels'
// renormalised shares (the step's lane marked the tiles under the box).
template <bool SPEC, bool COUNT>
__device__ __forceinline__ void splat_warp(const PhotonParams& p, const StepRec& R, uint32_t lane, BeamCounts& cnt) {
    const float cx = R.cx, cy = R.cy;
    if (R.valid == 2u) {  // empty tent sum: the whole colour to the centre pixel
        if (lane == 0) {
            const uint32_t px = (uint32_t)min(max((int)roundf(cx), 0), (int)p.width - 1);
            const uint32_t py = (uint32_t)min(max((int)roundf(cy), 0), (int)p.height - 1);
            if (COUNT) { ++cnt.deposits; return; }
            deposit_pixel<SPEC>(p, px, py, R, 1.0f);
        }
        return;
    }
    const uint32_t x0y0 = R.x0y0, box = R.box;
    const int x0 = (int)(x0y0 & 0xFFFFu), y0 = (int)(x0y0 >> 16);
    const int bw = (int)(box & 0xFFu), bh = (int)((box >> 8) & 0xFFu), rows = (int)((box >> 16) & 0xFFu);
    const int x1 = x0 + bw - 1, y1 = y0 + bh - 1;
    const float inv_r = R.inv_r, inv = R.inv_wsum;
    const int lrow = bw <= 32 ? (int)((lane * R.magic) >> 16) : 0;
    const int lcol = (int)lane - lrow * bw;
    if (lrow >= rows) return;
    const int chunks = bw <= 32 ? 1 : (bw + 31) / 32;
    for (int ch = 0; ch < chunks; ++ch) {
        const int px = x0 + ch * 32 + lcol;
        if (px > x1) break;
        const float dx = (float)px - cx, dx2 = dx * dx;
        for (int py = y0 + lrow; py <= y1; py += rows) {
            const float w = tent(dx2, (float)py - cy, inv_r) * inv;
            if (w > 0.0f) {
                if (COUNT) ++cnt.deposits;
                else deposit_pixel<SPEC>(p, (uint32_t)px, (uint32_t)py, R, w);
            }
        }
    }
}

// March every step of the n buffered segments as one flat list: 32 steps at a
// time are set up one per lane, then splatted one at a time by the whole warp.
template <bool SPEC, bool COUNT>
__device__ __forceinline__ void beam_flush(const PhotonParams& p, BeamWarpSmem& ws, uint32_t n, uint32_t* smask,
                                           BeamCounts& cnt) {
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
    if (COUNT && lane == 0) { cnt.segments += n; cnt.steps += total; }
    for (uint32_t t0 = 0; t0 < total; t0 += 32u) {
        const uint32_t t = t0 + lane;
        StepRec R;
        R.valid = 0u;
        if (t < total) {
            uint32_t lo = 0, hi = n;  // start[lo] <= t < start[hi]
            while (hi - lo > 1u) {
                const uint32_t mid = (lo + hi) >> 1;
                if (ws.start[mid] <= t) lo = mid; else hi = mid;
            }
            const BeamSeg B = ws.seg[lo];
            R = beam_step<SPEC, COUNT>(p, smask, B, ws.payload[B.lane], t - ws.start[lo], cnt);
        }
        ws.step[lane] = R;
        unsigned todo = __ballot_sync(0xffffffffu, R.valid != 0u);
        __syncwarp();
        BoxRun run;
        run.box = 0u;
        while (todo) {
            const uint32_t j = __ffs(todo) - 1u;
            todo &= todo - 1u;
            const StepRec Rj = ws.step[j];
            if (!COUNT && runnable(Rj)) {
                run_add<SPEC>(p, run, Rj, lane);
            } else {
                if (!COUNT) run_flush<SPEC>(p, run, lane);
                splat_warp<SPEC, COUNT>(p, Rj, lane, cnt);
            }
        }
        if (!COUNT) run_flush<SPEC>(p, run, lane);
        __syncwarp();
    }
}

// 32 photons of one warp (lane = photon): transport with segments recorded,
// then marched by beam_flush.
template <bool SPEC, bool COUNT>
__device__ __forceinline__ void trace_beam_warp(const PhotonParams& p, const SceneView& S, const float* cmf,
                                                uint32_t idx, bool valid, uint32_t* smask, BeamWarpSmem& ws,
                                                BeamCounts& cnt) {
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
            beam_flush<SPEC, COUNT>(p, ws, n, smask, cnt);
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

template <bool SPEC>
__global__ void __launch_bounds__(256, 3) beam_kernel(const PhotonParams p, uint32_t mask_words) {
    extern __shared__ __align__(16) unsigned char smem[];
    const float* cmf;
    uint32_t* smask;
    const SceneView S = load_scene(p, smem, &cmf, &smask, mask_words);
    BeamWarpSmem* ws = reinterpret_cast<BeamWarpSmem*>(smem + beam_offset(p, mask_words));
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    BeamCounts cnt = {0, 0, 0, 0};
    for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + warp) * 32u; base < p.photon_count; base += warps * 32u)
        trace_beam_warp<SPEC, false>(p, S, cmf, p.photon_base + base + lane, base + lane < p.photon_count, smask,
                                          ws[warp], cnt);
    if (smask) {
        __syncthreads();
        for (uint32_t w = threadIdx.x; w < mask_words; w += blockDim.x)
            if (smask[w]) atomicOr(p.flags + w, smask[w]);
    }
}

// Instrumented pass: same transport and march, no film writes; sums the work
// counters into out[0..4] = photons, segments, steps, in-frame steps, deposits.
__global__ void __launch_bounds__(256, 3) beam_count_kernel(const PhotonParams p, unsigned long long* out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const float* cmf;
    const SceneView S = load_scene(p, smem, &cmf);
    BeamWarpSmem* ws = reinterpret_cast<BeamWarpSmem*>(smem + beam_offset(p, 0));
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    BeamCounts cnt = {0, 0, 0, 0};
    unsigned long long ph = 0;
    for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + warp) * 32u; base < p.photon_count; base += warps * 32u) {
        trace_beam_warp<false, true>(p, S, cmf, p.photon_base + base + lane, base + lane < p.photon_count, nullptr,
                                        ws[warp], cnt);
        ph += base + lane < p.photon_count;
    }
    unsigned long long v[5] = {ph, cnt.segments, cnt.steps, cnt.in_frame, cnt.deposits};
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
        if (lane == 0 && v[i]) atomicAdd(out + i, v[i]);
    }
}

using BeamKernelFn = void (*)(const PhotonParams, uint32_t);

BeamKernelFn beam_fn(bool spec) { return spec ? beam_kernel<true> : beam_kernel<false>; }

size_t beam_smem(const PhotonParams& p, uint32_t mask_words) {
    return beam_offset(p, mask_words) + 8 * sizeof(BeamWarpSmem);
}

}  // namespace

int beam_occupancy_blocks(const LaunchShape& shape, bool spectral, size_t smem) {
    return occupancy_blocks(reinterpret_cast<const void*>(beam_fn(spectral)), (int)shape.block,
                            smem + 16 + 8 * sizeof(BeamWarpSmem));
}

cudaError_t launch_beam_count(const PhotonParams& p, unsigned long long* out, uint32_t grid, cudaStream_t s) {
    if (p.photon_count == 0) return cudaSuccess;
    const uint32_t need = (p.photon_count + 255u) / 256u;
    const size_t smem = beam_smem(p, 0);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(reinterpret_cast<const void*>(beam_count_kernel),
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    beam_count_kernel<<<need < grid ? need : grid, 256, smem, s>>>(p, out);
    return cudaGetLastError();
}

cudaError_t launch_beam(const PhotonParams& p, const LaunchShape& shape, cudaStream_t s) {
    if (p.photon_count == 0) return cudaSuccess;
    const uint32_t mw = photon_mask_words(p);
    const bool spec = p.channels != 3u || p.bins != 0u;
    const uint32_t need = (p.photon_count + 255u) / 256u;
    const uint32_t grid = need < shape.grid ? need : shape.grid;
    beam_fn(spec)<<<grid, 256, beam_smem(p, mw), s>>>(p, mw);
    return cudaGetLastError();
}

}  // namespace sc
