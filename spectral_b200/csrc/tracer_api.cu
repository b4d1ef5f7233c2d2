// extern "C" camera tracer object: GpuTracer (spectral-gpu/src/lib.rs:165-389)
// over the wavefront kernels of tracer.cu.
#include <algorithm>
#include <array>
#include <cmath>
#include <limits>
#include <vector>

#include "host_util.h"
#include "solid_bound.h"
#include "tracer.h"

using namespace sc;

namespace {
// Waves run on chains (one stream and one queue set each), so one wave's short
// late-bounce launches overlap other waves' full-width ones.  Measured on the
// 1280x720, 64 spp workload (accumulate(64)): 2 chains of 2^19-path waves
// (queues in L2) 7.47 ms, 3 x 2^20 6.39 ms, 3 x 2^22 6.11 ms, 2 x 2^24
// 6.14 ms: large waves give the in-place tail enough paths to fill the GPU, and
// the stages are bound by latency and issue, not by the queues' DRAM traffic.
// With the first shade making its own rays and 5 stage CTAs per SM: 2 x 2^22
// 5.52 ms, 3 x 2^21 5.47, 3 x 2^22 5.39, 4 x 2^23 5.35 (within run-to-run
// spread of 3 x 2^22); two compacted bounces before the tail stay best (one
// 6.45, three 5.75, four 5.67 ms).
constexpr uint32_t kMaxChains = 4;
constexpr uint32_t kDefaultChains = 3;
constexpr uint32_t kDefaultWaveLog2 = 22;  // paths per wave and chain: 2^22

}

struct sc_tracer {
    sc_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;                    // chain 0: the tracer's stream
    cudaStream_t extra[kMaxChains - 1] = {};          // chains 1..
    cudaEvent_t fork = nullptr, join[kMaxChains - 1] = {};
    uint32_t chains = kDefaultChains, wave_paths = 1u << kDefaultWaveLog2;
    std::mutex mu;
    uint32_t w = 0, h = 0, samples = 0;
    uint32_t row0 = 0, row1 = 0;  // rows traced by accumulate (all by default)
    TracerParams hp{};
    DevBuf<TracerParams> params;
    DevBuf<float> tables;
    DevBuf<sc_primitive> prims;
    DevBuf<sc_plane> planes;
    DevBuf<sc_material> mats;
    DevBuf<float4> bounds;
    DevBuf<float> sum, result, qbuf;
    DevBuf<float> mean;  // per-pixel means staged for read_xyz (allocated by its first call)
    DevBuf<uint32_t> counts, base;
    DevBuf<unsigned long long> segments;
    DevBuf<uint32_t> qbuf_u;
    uint32_t wave_cap = 0;  // paths per wave the queues are sized for
    TracerLaunch L[kMaxChains]{};
    cudaGraphExec_t graph = nullptr;
    uint32_t graph_spp = 0;
    uint64_t last_paths = 0, last_segments = 0;

    void release_streams() {
        if (stream) cudaStreamDestroy(stream);
        for (uint32_t c = 0; c + 1 < kMaxChains; ++c) {
            if (extra[c]) cudaStreamDestroy(extra[c]);
            if (join[c]) cudaEventDestroy(join[c]);
        }
        if (fork) cudaEventDestroy(fork);
        stream = nullptr;
        fork = nullptr;
    }
    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        graph_spp = 0;
    }
    int upload_params() {
        SC_CUDA(cudaMemcpyAsync(params.p, &hp, sizeof hp, cudaMemcpyHostToDevice, stream));
        return SC_OK;
    }
    int ensure_queues(uint32_t paths) {
        if (paths <= wave_cap) return SC_OK;
        drop_graph();
        const size_t n = paths;
        // per chain: 2 ray queues x 8 floats, result 3; 2 ray queues x 3 u32
        SC_CUDA(qbuf.alloc(chains * (n * 8 * 2 + 3 * n)));
        SC_CUDA(qbuf_u.alloc(chains * (n * 3 * 2)));
        float* f = qbuf.p;
        uint32_t* u = qbuf_u.p;
        for (uint32_t c = 0; c < chains; ++c) {
            TracerLaunch& Lc = L[c];
            RayQueue* qs[2] = {&Lc.qa, &Lc.qb};
            for (RayQueue* q : qs) {
                q->ox = f; q->oy = f + n; q->oz = f + 2 * n; q->dx = f + 3 * n; q->dy = f + 4 * n;
                q->dz = f + 5 * n; q->tp = f + 6 * n; q->u = f + 7 * n;
                f += 8 * n;
                q->rng = u; q->id = u + n; q->flags = u + 2 * n;
                u += 3 * n;
            }
            Lc.result = f;
            f += 3 * n;
        }
        wave_cap = paths;
        return SC_OK;
    }
    int run(uint32_t spp) {
        const uint32_t px0 = row0 * w, px1 = row1 * w, npx = px1 - px0;
        const uint32_t px_per_wave = std::max(1u, wave_paths / spp);
        int rc = ensure_queues(std::max(1u, std::min(npx, px_per_wave)) * spp);
        if (rc != SC_OK) return rc;
        for (uint32_t c = 0; c < chains; ++c) L[c].spp = spp;
        SC_CUDA(cudaMemcpyAsync(base.p, &samples, 4, cudaMemcpyHostToDevice, stream));
        if (!graph || graph_spp != spp) {
            drop_graph();
            cudaGraph_t g = nullptr;
            SC_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            // fork the other chains off the tracer's stream, deal waves round robin, join them back
            cudaError_t e = cudaEventRecord(fork, stream);
            for (uint32_t c = 1; c < chains && e == cudaSuccess; ++c) e = cudaStreamWaitEvent(extra[c - 1], fork, 0);
            uint32_t wave = 0;
            for (uint32_t first = px0; first < px1 && e == cudaSuccess; first += px_per_wave, ++wave) {
                const uint32_t c = wave % chains;
                e = launch_tracer_wave(params.p, L[c], first, std::min(px_per_wave, px1 - first),
                                       c ? extra[c - 1] : stream);
            }
            for (uint32_t c = 1; c < chains && e == cudaSuccess; ++c) {
                e = cudaEventRecord(join[c - 1], extra[c - 1]);
                if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, join[c - 1], 0);
            }
            cudaError_t e2 = cudaStreamEndCapture(stream, &g);
            if (e == cudaSuccess) e = e2;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&graph, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                graph = nullptr;
                set_error("tracer graph capture failed: %s", cudaGetErrorString(e));
                return SC_E_CUDA;
            }
            graph_spp = spp;
        }
        SC_CUDA(cudaGraphLaunch(graph, stream));
        samples += spp;
        last_paths = (uint64_t)npx * spp;
        return SC_OK;
    }
};

extern "C" {

int sc_tracer_create(sc_ctx* ctx, const sc_primitive* prims, uint32_t n_prims, const sc_plane* planes,
                     uint32_t n_planes, const sc_material* mats, uint32_t n_mats, float background, int has_horizon,
                     float horizon, const sc_camera* cam, uint32_t width, uint32_t height, uint32_t illuminant,
                     uint32_t seed, const sc_tracer_options* opts, sc_tracer** out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && cam && out, SC_E_INVALID, "null argument");
    *out = nullptr;
    SC_REQUIRE(n_prims <= SC_MAX_PRIMS && n_planes <= SC_MAX_PLANES && n_mats <= SC_MAX_PRIMS, SC_E_LIMIT,
               "scene exceeds %d primitives / %d planes", SC_MAX_PRIMS, SC_MAX_PLANES);
    SC_REQUIRE((n_prims == 0 || prims) && (n_planes == 0 || planes) && (n_mats == 0 || mats), SC_E_INVALID,
               "null scene array");
    for (uint32_t i = 0; i < n_prims; ++i) {
        SC_REQUIRE(prims[i].kind <= 1u && prims[i].material < n_mats, SC_E_INVALID, "primitive %u invalid", i);
        if (prims[i].kind == 1u)
            SC_REQUIRE((uint64_t)prims[i].plane_start + prims[i].plane_count <= n_planes, SC_E_INVALID,
                       "primitive %u plane range", i);
    }
    for (uint32_t i = 0; i < n_mats; ++i)
        SC_REQUIRE(mats[i].kind <= 1u && (mats[i].kind == 0u || mats[i].glass <= 3u), SC_E_INVALID, "material %u", i);
    SC_REQUIRE(width > 0 && height > 0 && (uint64_t)width * height <= (1ull << 26), SC_E_INVALID, "image %ux%u",
               width, height);
    SC_REQUIRE(illuminant <= 1u, SC_E_INVALID, "illuminant %u (0 D65, 1 A)", illuminant);
    sc_tracer_options o{};
    if (opts) o = *opts;
    if (o.max_depth == 0) o.max_depth = 8;
    SC_REQUIRE(o.max_depth <= 64, SC_E_LIMIT, "max_depth %u > 64", o.max_depth);
    SC_REQUIRE(o.wave_bounces <= 64, SC_E_INVALID, "wave_bounces %u > 64", o.wave_bounces);
    SC_REQUIRE(o.chains <= kMaxChains, SC_E_INVALID, "chains %u > %u", o.chains, kMaxChains);
    SC_REQUIRE(o.wave_paths_log2 == 0 || (o.wave_paths_log2 >= 12 && o.wave_paths_log2 <= 24), SC_E_INVALID,
               "wave_paths_log2 %u outside 12..24", o.wave_paths_log2);
    sc_tracer* t = new sc_tracer();
    t->ctx = ctx; t->w = width; t->h = height;
    t->chains = o.chains ? o.chains : kDefaultChains;
    t->wave_paths = 1u << (o.wave_paths_log2 ? o.wave_paths_log2 : kDefaultWaveLog2);
    DeviceGuard g(ctx->device);
    auto fail = [&](cudaError_t e) {
        set_error("tracer setup failed: %s", cudaGetErrorString(e));
        t->release_streams();
        delete t;
        return e == cudaErrorMemoryAllocation ? SC_E_NOMEM : SC_E_CUDA;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e);
    for (uint32_t c = 1; c < t->chains; ++c) {
        if ((e = cudaStreamCreateWithFlags(&t->extra[c - 1], cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
        if ((e = cudaEventCreateWithFlags(&t->join[c - 1], cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    }
    if ((e = cudaEventCreateWithFlags(&t->fork, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    if ((e = t->params.alloc(1)) != cudaSuccess) return fail(e);
    if ((e = t->tables.alloc(5 * kTableN)) != cudaSuccess) return fail(e);
    if ((e = t->prims.alloc(std::max(1u, n_prims))) != cudaSuccess) return fail(e);
    if ((e = t->planes.alloc(std::max(1u, n_planes))) != cudaSuccess) return fail(e);
    if ((e = t->mats.alloc(std::max(1u, n_mats))) != cudaSuccess) return fail(e);
    if ((e = t->bounds.alloc(std::max(1u, n_prims))) != cudaSuccess) return fail(e);
    if ((e = t->sum.alloc(3ull * width * height)) != cudaSuccess) return fail(e);
    // per chain: max_depth + 1 queue counts and the tail's claim counter
    if ((e = t->counts.alloc(t->chains * (o.max_depth + 2))) != cudaSuccess) return fail(e);
    if ((e = t->base.alloc(1)) != cudaSuccess) return fail(e);
    if ((e = t->segments.alloc(1)) != cudaSuccess) return fail(e);
    cudaMemcpy(t->tables.p, ctx->tables, 5 * kTableN * sizeof(float), cudaMemcpyHostToDevice);
    if (n_prims) cudaMemcpy(t->prims.p, prims, n_prims * sizeof(sc_primitive), cudaMemcpyHostToDevice);
    if (n_planes) cudaMemcpy(t->planes.p, planes, n_planes * sizeof(sc_plane), cudaMemcpyHostToDevice);
    if (n_mats) cudaMemcpy(t->mats.p, mats, n_mats * sizeof(sc_material), cudaMemcpyHostToDevice);
    {
        std::vector<float4> hb(std::max(1u, n_prims));
        for (uint32_t i = 0; i < n_prims; ++i) {
            float b[4] = {0.0f, 0.0f, 0.0f, std::numeric_limits<float>::infinity()};
            if (prims[i].kind == 1u) solid_bound(planes + prims[i].plane_start, prims[i].plane_count, b);
            hb[i] = make_float4(b[0], b[1], b[2], b[3]);
        }
        if ((e = cudaMemcpy(t->bounds.p, hb.data(), hb.size() * sizeof(float4), cudaMemcpyHostToDevice)) != cudaSuccess)
            return fail(e);
    }
    cudaMemset(t->sum.p, 0, t->sum.bytes());
    cudaMemset(t->segments.p, 0, 8);
    t->row0 = 0; t->row1 = height;
    TracerParams& hp = t->hp;
    hp.cam = *cam; hp.width = width; hp.height = height; hp.seed = seed; hp.illuminant = illuminant;
    hp.background = background; hp.horizon = horizon; hp.has_horizon = has_horizon ? 1u : 0u;
    hp.max_depth = o.max_depth; hp.rr_start = o.rr_start;
    hp.spectral = 1u;
    hp.em_center = ld3(o.emitter_center); hp.em_radius = o.emitter_radius; hp.em_scale = o.emitter_scale;
    hp.prims = t->prims.p; hp.planes = t->planes.p; hp.mats = t->mats.p;
    hp.n_prims = n_prims; hp.n_planes = n_planes; hp.n_mats = n_mats;
    hp.tables = t->tables.p;
    hp.bounds = t->bounds.p;
    for (uint32_t c = 0; c < t->chains; ++c) {
        TracerLaunch& L = t->L[c];
        L.counts = t->counts.p + c * (o.max_depth + 2); L.sum = t->sum.p; L.d_base = t->base.p;
        L.segments = t->segments.p;
        L.max_depth = o.max_depth; L.n_planes = n_planes; L.grid = (uint32_t)tracer_grid(ctx->sms);
        L.wave_bounces = o.wave_bounces ? o.wave_bounces : 2u;
    }
    if ((e = cudaMemcpy(t->params.p, &hp, sizeof hp, cudaMemcpyHostToDevice)) != cudaSuccess) return fail(e);
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail(e);
    *out = t;
    return SC_OK;
    SC_GUARD_END
}

int sc_tracer_destroy(sc_tracer* t) {
    SC_GUARD_BEGIN
    if (!t) return SC_OK;
    {
        DeviceGuard g(t->ctx->device);
        if (t->stream) cudaStreamSynchronize(t->stream);
        t->drop_graph();
        t->params.reset(); t->tables.reset(); t->prims.reset(); t->planes.reset(); t->mats.reset(); t->bounds.reset();
        t->sum.reset(); t->result.reset(); t->qbuf.reset(); t->qbuf_u.reset(); t->counts.reset(); t->base.reset();
        t->segments.reset(); t->mean.reset();
        t->release_streams();
    }
    delete t;
    return SC_OK;
    SC_GUARD_END
}

#define TR_LOCK(t)                                           \
    SC_REQUIRE((t), SC_E_INVALID, "null tracer");            \
    std::lock_guard<std::mutex> _lk((t)->mu);                \
    DeviceGuard _dg((t)->ctx->device)

int sc_tracer_accumulate(sc_tracer* t, uint32_t spp) {
    SC_GUARD_BEGIN
    TR_LOCK(t);
    if (spp == 0) return SC_OK;
    SC_REQUIRE(spp <= (1u << 16), SC_E_INVALID, "spp %u > 65536", spp);
    return t->run(spp);
    SC_GUARD_END
}

int sc_tracer_read_xyz(sc_tracer* t, float* out) {
    SC_GUARD_BEGIN
    TR_LOCK(t);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    // AccumBuffer::mean (spectral-core/src/lib.rs:16-20): sum / max(samples, 1), on the device
    const size_t n = 3ull * t->w * t->h;
    if (t->mean.n < n) SC_CUDA(t->mean.alloc(n));
    SC_CUDA(launch_tracer_mean(t->sum.p, t->mean.p, n, (float)std::max(t->samples, 1u), t->ctx->sms, t->stream));
    SC_CUDA(cudaMemcpyAsync(out, t->mean.p, n * sizeof(float), cudaMemcpyDeviceToHost, t->stream));
    SC_CUDA(cudaStreamSynchronize(t->stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_tracer_set_camera(sc_tracer* t, const sc_camera* cam) {
    SC_GUARD_BEGIN
    TR_LOCK(t);
    SC_REQUIRE(cam, SC_E_INVALID, "null camera");
    t->hp.cam = *cam;
    return t->upload_params();
    SC_GUARD_END
}

int sc_tracer_set_rows(sc_tracer* t, uint32_t row_begin, uint32_t row_end) {
    SC_GUARD_BEGIN
    TR_LOCK(t);
    SC_REQUIRE(row_begin <= row_end && row_end <= t->h, SC_E_INVALID, "rows [%u, %u) outside [0, %u)", row_begin,
               row_end, t->h);
    if (row_begin != t->row0 || row_end != t->row1) {
        t->row0 = row_begin;
        t->row1 = row_end;
        t->drop_graph();  // the captured waves cover the old rows
    }
    return SC_OK;
    SC_GUARD_END
}

int sc_tracer_set_spectral(sc_tracer* t, int on) {
    SC_GUARD_BEGIN
    TR_LOCK(t);
    t->hp.spectral = on ? 1u : 0u;
    return t->upload_params();
    SC_GUARD_END
}

int sc_tracer_clear_accum(sc_tracer* t) {
    SC_GUARD_BEGIN
    TR_LOCK(t);
    SC_CUDA(cudaMemsetAsync(t->sum.p, 0, t->sum.bytes(), t->stream));
    t->samples = 0;
    return SC_OK;
    SC_GUARD_END
}

int sc_tracer_stream(sc_tracer* t, void** stream) {
    SC_GUARD_BEGIN
    SC_REQUIRE(t && stream, SC_E_INVALID, "null argument");
    *stream = t->stream;
    return SC_OK;
    SC_GUARD_END
}

int sc_tracer_dims(sc_tracer* t, uint32_t* w, uint32_t* h) {
    SC_GUARD_BEGIN
    SC_REQUIRE(t, SC_E_INVALID, "null tracer");
    if (w) *w = t->w;
    if (h) *h = t->h;
    return SC_OK;
    SC_GUARD_END
}

int sc_tracer_last_stats(sc_tracer* t, uint64_t* paths, uint64_t* segments) {
    SC_GUARD_BEGIN
    TR_LOCK(t);
    unsigned long long s = 0;
    SC_CUDA(cudaMemcpyAsync(&s, t->segments.p, 8, cudaMemcpyDeviceToHost, t->stream));
    SC_CUDA(cudaStreamSynchronize(t->stream));
    if (paths) *paths = t->last_paths;
    if (segments) *segments = s;
    return SC_OK;
    SC_GUARD_END
}

}  // extern "C"
