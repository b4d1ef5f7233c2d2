// extern "C" batch object: many uneven scenes in one persistent, graph-captured
// launch (batch.cu), the same work as plain per-scene launches for comparison,
// and an autotuner that picks chunk size (work-queue granularity), threads per
// CTA, register bound, splat aggregation and transport by timing the batch
// itself.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "batch.h"
#include "host_util.h"

using namespace sc;

namespace {

struct JobGeom {
    uint32_t w, h, channels, tiles_x, tiles_y, words;
    size_t cells() const { return (size_t)tiles_x * tiles_y * kTilePixels * channels; }
};

int check_job(const sc_scene_job& j, uint32_t i) {
    SC_REQUIRE(j.n_prims <= kBatchPrims && j.n_planes <= kBatchPlanes && j.n_mats <= kBatchPrims, SC_E_LIMIT,
               "job %u: batch scenes hold at most %u primitives / %u planes", i, kBatchPrims, kBatchPlanes);
    for (uint32_t k = 0; k < j.n_prims; ++k) {
        const sc_primitive& p = j.prims[k];
        SC_REQUIRE(p.kind <= 1u && p.material < j.n_mats, SC_E_INVALID, "job %u primitive %u invalid", i, k);
        if (p.kind == 1u)
            SC_REQUIRE((uint64_t)p.plane_start + p.plane_count <= j.n_planes, SC_E_INVALID,
                       "job %u primitive %u plane range", i, k);
    }
    for (uint32_t k = 0; k < j.n_mats; ++k)
        SC_REQUIRE(j.mats[k].kind <= 1u && (j.mats[k].kind == 0u || j.mats[k].glass <= 3u), SC_E_INVALID,
                   "job %u material %u", i, k);
    SC_REQUIRE(j.width > 0 && j.height > 0 && (uint64_t)j.width * j.height <= (1ull << 26), SC_E_INVALID,
               "job %u film %ux%u", i, j.width, j.height);
    SC_REQUIRE(j.opts.bins >= 1 && j.opts.bins <= SC_MAX_BINS, SC_E_INVALID,
               "job %u: batch films are spectral (1..%d bins)", i, SC_MAX_BINS);
    const float lmin = j.opts.lambda_min ? j.opts.lambda_min : 380.0f, lmax = j.opts.lambda_max ? j.opts.lambda_max : 730.0f;
    SC_REQUIRE(lmax > lmin, SC_E_INVALID, "job %u band", i);
    SC_REQUIRE(j.opts.max_bounces <= 64 && j.opts.scale_log2 <= 50 && (j.opts.estimator <= 1 || j.opts.estimator == 3), SC_E_INVALID,
               "job %u options", i);
    SC_REQUIRE(j.opts.haze_exact == 0u, SC_E_INVALID, "job %u: batches run the fast haze samples (haze_exact 0)", i);
    return SC_OK;
}

}  // namespace

struct sc_batch {
    sc_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    // Pipelined read-back: `ran` is recorded after every pass, `copied` after
    // every asynchronous image copy.  Job uploads wait for the last pass, a
    // pass's drain (which rewrites the images) waits for the last copy, and a
    // copy waits for the last pass, so the copy of pass k overlaps the tracing
    // of pass k + 1.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ran = nullptr, copied = nullptr;
    cudaEvent_t uploaded = nullptr;  // orders a pass on a caller's stream after work on the batch's own stream
    std::mutex mu;
    std::vector<sc_scene_job> jobs;
    std::vector<JobGeom> geom;
    std::vector<size_t> film_off, flag_off, xyz_off, binw_off;
    DevBuf<unsigned long long> films;
    DevBuf<uint32_t> flags;
    DevBuf<float> xyz, binw;
    DevBuf<BatchJobDev> d_jobs;
    DevBuf<WorkItem> d_items;
    DevBuf<FilmDesc> d_descs;
    DevBuf<DirtyTile> dirty_list;  // reduce scratch: room for every tile, and its counter
    DevBuf<uint32_t> counter, dirty_count;
    std::vector<BatchJobDev> h_jobs;
    // Pinned copy of the job table for its upload, so the host returns at once
    // (a copy from pageable memory would first wait for the pass before it);
    // `staged` follows the last upload, which must have read it before the
    // host rewrites it.
    BatchJobDev* h_stage = nullptr;
    cudaEvent_t staged = nullptr;
    void free_stage() {
        if (h_stage) cudaFreeHost(h_stage);
        if (staged) cudaEventDestroy(staged);
        h_stage = nullptr;
        staged = nullptr;
    }
    uint32_t n_items = 0, total_tiles = 0, total_words = 0, max_channels = 0;
    uint64_t total_photons = 0;
    sc_batch_tuning tuning{};
    uint32_t grid = 0;
    bool ff = false;  // some job samples free-flight distances: the kernel built with them

    bool any_free_flight() const {
        for (const sc_scene_job& j : jobs)
            if (j.opts.estimator == 3u && j.weights.sigma_t > 0.0f) return true;
        return false;
    }
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;

    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
    }

    PhotonParams job_params(uint32_t j) const {
        const sc_scene_job& J = jobs[j];
        const JobGeom& g = geom[j];
        sc_film_options o = J.opts;
        if (o.lambda_min == 0.0f) o.lambda_min = 380.0f;
        if (o.lambda_max == 0.0f) o.lambda_max = 730.0f;
        if (o.max_bounces == 0u) o.max_bounces = 8u;
        if (o.scale_log2 == 0u) o.scale_log2 = 32u;
        PhotonParams p;
        std::memset(&p, 0, sizeof p);
        p.corner = ld3(J.beam.corner); p.bu = ld3(J.beam.u); p.bv = ld3(J.beam.v); p.bdir = ld3(J.beam.dir);
        p.proj = make_proj(J.cam);
        p.width = g.w; p.height = g.h; p.tiles_x = g.tiles_x; p.channels = g.channels;
        p.photon_base = 0; p.photon_count = J.n_photons; p.seed = J.seed; p.max_bounces = o.max_bounces;
        p.sigma_s = J.weights.sigma_s; p.sigma_t = J.weights.sigma_t; p.g = J.weights.g; p.max_dist = J.max_dist;
        p.lambda_min = o.lambda_min; p.lambda_range = o.lambda_max - o.lambda_min;
        p.bins = o.bins; p.bin_min = o.lambda_min; p.bin_inv_width = (float)o.bins / p.lambda_range;
        p.scale = std::ldexp(1.0f, (int)o.scale_log2);
        p.spectral = J.spectral; p.estimator = o.estimator;
        p.film = films.p + film_off[j];
        p.flags = flags.p + flag_off[j];
        p.n_prims = J.n_prims; p.n_planes = J.n_planes; p.n_mats = J.n_mats;
        p.cmf = ctx->cmf.p;
        set_haze_consts(p);
        return p;
    }

    int upload_jobs() {
        h_jobs.resize(jobs.size());
        for (uint32_t j = 0; j < jobs.size(); ++j) {
            BatchJobDev& d = h_jobs[j];
            std::memset(&d, 0, sizeof d);
            d.slot_image.p = job_params(j);
            std::memcpy(d.slot_image.prims, jobs[j].prims, sizeof d.slot_image.prims);
            std::memcpy(d.slot_image.planes, jobs[j].planes, sizeof d.slot_image.planes);
            std::memcpy(d.slot_image.mats, jobs[j].mats, sizeof d.slot_image.mats);
            d.flags = flags.p + flag_off[j];
            d.mask_words = geom[j].words;
        }
        if (!h_stage || !staged) {
            free_stage();
            cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&h_stage), h_jobs.size() * sizeof(BatchJobDev));
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&staged, cudaEventDisableTiming);
            if (e != cudaSuccess) {
                free_stage();
                SC_CUDA(e);
            }
        } else {
            SC_CUDA(cudaEventSynchronize(staged));  // the last upload has read the pinned copy
        }
        std::memcpy(h_stage, h_jobs.data(), h_jobs.size() * sizeof(BatchJobDev));
        SC_CUDA(cudaStreamWaitEvent(stream, ran, 0));  // the previous pass still reads the table
        SC_CUDA(cudaMemcpyAsync(d_jobs.p, h_stage, h_jobs.size() * sizeof(BatchJobDev), cudaMemcpyHostToDevice,
                                stream));
        SC_CUDA(cudaEventRecord(staged, stream));
        return SC_OK;
    }

    int build_items(uint32_t chunk) {
        std::vector<uint32_t> order(jobs.size());
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t a, uint32_t b) { return jobs[a].n_photons > jobs[b].n_photons; });
        std::vector<WorkItem> items;
        for (uint32_t j : order)
            for (uint32_t b = 0; b < jobs[j].n_photons; b += chunk)
                items.push_back(WorkItem{j, b, std::min(chunk, jobs[j].n_photons - b)});
        n_items = (uint32_t)items.size();
        if (d_items.n < items.size()) SC_CUDA(d_items.alloc(items.size()));
        if (!items.empty())
            SC_CUDA(cudaMemcpyAsync(d_items.p, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                                    stream));
        SC_CUDA(cudaStreamSynchronize(stream));
        return SC_OK;
    }

    int apply_tuning(const sc_batch_tuning& t) {
        sc_batch_tuning n = t;
        if (n.chunk_photons == 0) n.chunk_photons = 2048;
        n.chunk_photons = std::max(32u, (n.chunk_photons + 31u) / 32u * 32u);
        if (n.minb == 0) n.minb = 4;
        n.minb = n.minb >= 5 ? 5 : 4;
        n.aggregate = n.aggregate ? 1 : 0;
        n.per_photon = n.per_photon ? 1 : 0;
        n.block = n.block == 128u ? 128u : 256u;
        ff = any_free_flight();
        const int occ = batch_occupancy((int)n.aggregate, (int)n.minb, n.per_photon ? 0 : 1, kBatchMaskWords, n.block,
                                        ff);
        grid = n.grid ? n.grid : (uint32_t)(ctx->sms * occ);
        if (n.chunk_photons != tuning.chunk_photons || n_items == 0) {
            int rc = build_items(n.chunk_photons);
            if (rc != SC_OK) return rc;
        }
        n.grid = grid;
        tuning = n;
        drop_graph();
        return SC_OK;
    }

    int enqueue_batch(cudaStream_t s) {
        SC_CUDA(launch_batch(d_jobs.p, d_items.p, n_items, counter.p, ctx->cmf.p, kBatchMaskWords,
                             (int)tuning.aggregate, (int)tuning.minb, tuning.per_photon ? 0 : 1, grid, s,
                             tuning.block, ff));
        // the drain rewrites the images: wait for the last asynchronous copy of them
        SC_CUDA(cudaStreamWaitEvent(s, copied, cudaEventWaitExternal));
        SC_CUDA(launch_reduce_many(d_descs.p, (uint32_t)jobs.size(), total_words, true, max_channels, dirty_list.p,
                                   dirty_count.p, s));
        return SC_OK;
    }

    int run(cudaStream_t s) {
        if (!graph || graph_stream != s) {
            drop_graph();
            cudaGraph_t g = nullptr;
            SC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            int rc = enqueue_batch(s);
            cudaError_t e = cudaStreamEndCapture(s, &g);
            if (rc != SC_OK) { if (g) cudaGraphDestroy(g); return rc; }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&graph, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                graph = nullptr;
                set_error("batch graph capture failed: %s", cudaGetErrorString(e));
                return SC_E_CUDA;
            }
            graph_stream = s;
        }
        SC_CUDA(cudaGraphLaunch(graph, s));
        SC_CUDA(cudaEventRecord(ran, s));
        return SC_OK;
    }

    int run_plain(cudaStream_t s) {
        SC_CUDA(cudaStreamWaitEvent(s, copied, 0));  // the drains rewrite the images
        for (uint32_t j = 0; j < jobs.size(); ++j) {
            PhotonParams p = job_params(j);
            p.prims = reinterpret_cast<const sc_primitive*>(
                reinterpret_cast<const unsigned char*>(d_jobs.p + j) + offsetof(BatchSlotImage, prims));
            p.planes = reinterpret_cast<const sc_plane*>(
                reinterpret_cast<const unsigned char*>(d_jobs.p + j) + offsetof(BatchSlotImage, planes));
            p.mats = reinterpret_cast<const sc_material*>(
                reinterpret_cast<const unsigned char*>(d_jobs.p + j) + offsetof(BatchSlotImage, mats));
            // the transport the batch's tuning chose (measured on these scenes, it
            // beats the single-film default of warp-split transport plus the
            // wavelength-ordered dispatch for films larger than L2)
            LaunchShape shape;
            shape.block = 256; shape.aggregate = 0; shape.minb = 4; shape.split = tuning.per_photon ? 0 : 1;
            const size_t smem = scene_smem_bytes(p.n_prims, p.n_planes, p.n_mats) +
                                (geom[j].words <= kMaxSmemMaskWords ? geom[j].words * 4u : 0u);
            shape.grid = (uint32_t)(ctx->sms * photon_occupancy_blocks(shape, true, smem));
            SC_CUDA(launch_photons(p, shape, s));
            ReduceParams r;
            r.film = p.film; r.flags = p.flags; r.xyz = xyz.p + xyz_off[j]; r.width = geom[j].w; r.height = geom[j].h;
            r.tiles_x = geom[j].tiles_x; r.tiles_y = geom[j].tiles_y; r.channels = geom[j].channels;
            r.binw = binw.p + binw_off[j];
            r.inv_scale = std::ldexp(1.0, -(int)(jobs[j].opts.scale_log2 ? jobs[j].opts.scale_log2 : 32u));
            SC_CUDA(launch_reduce(r, true, s));
        }
        SC_CUDA(cudaEventRecord(ran, s));
        return SC_OK;
    }
};

extern "C" {

int sc_batch_create(sc_ctx* ctx, const sc_scene_job* jobs, uint32_t n_jobs, const sc_batch_tuning* tuning,
                    sc_batch** out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && jobs && out && n_jobs > 0, SC_E_INVALID, "null argument or empty batch");
    *out = nullptr;
    for (uint32_t i = 0; i < n_jobs; ++i) {
        int rc = check_job(jobs[i], i);
        if (rc != SC_OK) return rc;
    }
    sc_batch* b = new sc_batch();
    b->ctx = ctx;
    b->jobs.assign(jobs, jobs + n_jobs);
    size_t cells = 0, words = 0, px = 0, bw = 0;
    uint32_t tiles = 0;
    for (uint32_t i = 0; i < n_jobs; ++i) {
        JobGeom g;
        g.w = jobs[i].width; g.h = jobs[i].height; g.channels = jobs[i].opts.bins;
        g.tiles_x = (g.w + 7u) / 8u; g.tiles_y = (g.h + 7u) / 8u; g.words = flag_words(g.w, g.h);
        b->geom.push_back(g);
        b->film_off.push_back(cells); b->flag_off.push_back(words); b->xyz_off.push_back(3 * px);
        b->binw_off.push_back(bw);
        cells += g.cells(); words += g.words; px += (size_t)g.w * g.h; bw += 3 * g.channels;
        tiles += g.tiles_x * g.tiles_y;
        b->max_channels = std::max(b->max_channels, g.channels);
        b->total_photons += jobs[i].n_photons;
    }
    b->total_tiles = tiles;
    b->total_words = (uint32_t)words;
    DeviceGuard g(ctx->device);
    auto fail = [&](cudaError_t e) {
        set_error("batch setup failed: %s", cudaGetErrorString(e));
        if (b->stream) cudaStreamDestroy(b->stream);
        if (b->copy_stream) cudaStreamDestroy(b->copy_stream);
        if (b->ran) cudaEventDestroy(b->ran);
        if (b->copied) cudaEventDestroy(b->copied);
        if (b->uploaded) cudaEventDestroy(b->uploaded);
        b->free_stage();
        delete b;
        return e == cudaErrorMemoryAllocation ? SC_E_NOMEM : SC_E_CUDA;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e);
    if ((e = cudaStreamCreateWithFlags(&b->copy_stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreateWithFlags(&b->ran, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreateWithFlags(&b->copied, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreateWithFlags(&b->uploaded, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    if ((e = cudaEventRecord(b->ran, b->stream)) != cudaSuccess) return fail(e);
    if ((e = cudaEventRecord(b->copied, b->stream)) != cudaSuccess) return fail(e);
    if ((e = b->films.alloc(cells)) != cudaSuccess) return fail(e);
    if ((e = b->flags.alloc(words)) != cudaSuccess) return fail(e);
    if ((e = b->xyz.alloc(3 * px)) != cudaSuccess) return fail(e);
    if ((e = b->binw.alloc(bw)) != cudaSuccess) return fail(e);
    if ((e = b->d_jobs.alloc(n_jobs)) != cudaSuccess) return fail(e);
    if ((e = b->d_descs.alloc(n_jobs)) != cudaSuccess) return fail(e);
    if ((e = b->counter.alloc(1)) != cudaSuccess) return fail(e);
    if ((e = b->dirty_list.alloc(tiles)) != cudaSuccess) return fail(e);
    if ((e = b->dirty_count.alloc(1)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(b->films.p, 0, b->films.bytes(), b->stream)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(b->flags.p, 0, b->flags.bytes(), b->stream)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(b->xyz.p, 0, b->xyz.bytes(), b->stream)) != cudaSuccess) return fail(e);
    std::vector<float> hw(bw);
    std::vector<FilmDesc> descs(n_jobs);
    for (uint32_t i = 0; i < n_jobs; ++i) {
        const sc_film_options& o = jobs[i].opts;
        bin_weights(ctx->tables, o.bins, o.lambda_min ? o.lambda_min : 380.0f, o.lambda_max ? o.lambda_max : 730.0f,
                    hw.data() + b->binw_off[i]);
        FilmDesc& d = descs[i];
        d.film = b->films.p + b->film_off[i]; d.flags = b->flags.p + b->flag_off[i]; d.xyz = b->xyz.p + b->xyz_off[i];
        d.binw = b->binw.p + b->binw_off[i];
        d.width = b->geom[i].w; d.height = b->geom[i].h; d.tiles_x = b->geom[i].tiles_x; d.tiles_y = b->geom[i].tiles_y;
        d.channels = b->geom[i].channels; d.word_begin = (uint32_t)b->flag_off[i];
        d.inv_scale = std::ldexp(1.0, -(int)(o.scale_log2 ? o.scale_log2 : 32u));
    }
    if ((e = cudaMemcpyAsync(b->binw.p, hw.data(), bw * sizeof(float), cudaMemcpyHostToDevice, b->stream)) != cudaSuccess)
        return fail(e);
    if ((e = cudaMemcpyAsync(b->d_descs.p, descs.data(), n_jobs * sizeof(FilmDesc), cudaMemcpyHostToDevice,
                             b->stream)) != cudaSuccess)
        return fail(e);
    int rc = b->upload_jobs();
    if (rc == SC_OK) rc = b->apply_tuning(tuning ? *tuning : sc_batch_tuning{});
    if (rc == SC_OK && (e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return fail(e);
    if (rc != SC_OK) {
        std::string msg = sc_last_error();
        if (b->stream) cudaStreamDestroy(b->stream);
        if (b->copy_stream) cudaStreamDestroy(b->copy_stream);
        if (b->ran) cudaEventDestroy(b->ran);
        if (b->copied) cudaEventDestroy(b->copied);
        if (b->uploaded) cudaEventDestroy(b->uploaded);
        b->free_stage();
        delete b;
        set_error("%s", msg.c_str());
        return rc;
    }
    *out = b;
    return SC_OK;
    SC_GUARD_END
}

int sc_batch_destroy(sc_batch* b) {
    SC_GUARD_BEGIN
    if (!b) return SC_OK;
    {
        DeviceGuard g(b->ctx->device);
        if (b->stream) cudaStreamSynchronize(b->stream);
        if (b->graph_stream) cudaStreamSynchronize(b->graph_stream);
        if (b->copy_stream) cudaStreamSynchronize(b->copy_stream);
        b->drop_graph();
        b->films.reset(); b->flags.reset(); b->xyz.reset(); b->binw.reset(); b->d_jobs.reset(); b->d_items.reset();
        b->d_descs.reset(); b->counter.reset();
        if (b->stream) cudaStreamDestroy(b->stream);
        if (b->copy_stream) cudaStreamDestroy(b->copy_stream);
        if (b->ran) cudaEventDestroy(b->ran);
        if (b->copied) cudaEventDestroy(b->copied);
        if (b->uploaded) cudaEventDestroy(b->uploaded);
        b->free_stage();
    }
    delete b;
    return SC_OK;
    SC_GUARD_END
}

#define BATCH_LOCK(b)                                        \
    SC_REQUIRE((b), SC_E_INVALID, "null batch");             \
    std::lock_guard<std::mutex> _lk((b)->mu);                \
    DeviceGuard _dg((b)->ctx->device)

int sc_batch_set_tuning(sc_batch* b, const sc_batch_tuning* t) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    SC_REQUIRE(t, SC_E_INVALID, "null tuning");
    SC_CUDA(cudaStreamSynchronize(b->stream));
    if (b->graph_stream) SC_CUDA(cudaStreamSynchronize(b->graph_stream));
    return b->apply_tuning(*t);
    SC_GUARD_END
}

int sc_batch_get_tuning(sc_batch* b, sc_batch_tuning* t) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    SC_REQUIRE(t, SC_E_INVALID, "null output");
    *t = b->tuning;
    return SC_OK;
    SC_GUARD_END
}

int sc_batch_autotune(sc_batch* b, sc_batch_tuning* chosen) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    cudaEvent_t e0, e1;
    SC_CUDA(cudaEventCreate(&e0));
    SC_CUDA(cudaEventCreate(&e1));
    sc_batch_tuning best{};
    float best_ms = 1e30f;
    for (uint32_t block : {256u, 128u})
    for (uint32_t per_photon : {0u, 1u})
    for (uint32_t chunk : {512u, 2048u, 8192u})
        for (uint32_t minb : {4u, 5u})
            for (uint32_t agg : {0u, 1u}) {
                sc_batch_tuning t{chunk, minb, agg, 0, per_photon, block};
                int rc = b->apply_tuning(t);
                if (rc == SC_OK) rc = b->run(b->stream);  // warm-up (also builds the graph)
                if (rc != SC_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
                SC_CUDA(cudaEventRecord(e0, b->stream));
                for (int k = 0; k < 2; ++k) {
                    rc = b->run(b->stream);
                    if (rc != SC_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
                }
                SC_CUDA(cudaEventRecord(e1, b->stream));
                SC_CUDA(cudaEventSynchronize(e1));
                float ms = 0.0f;
                SC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best_ms) { best_ms = ms; best = b->tuning; }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    best.grid = 0;
    int rc = b->apply_tuning(best);
    if (rc != SC_OK) return rc;
    if (chosen) *chosen = b->tuning;
    return SC_OK;
    SC_GUARD_END
}

int sc_batch_update_jobs(sc_batch* b, const sc_scene_job* jobs, uint32_t n) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    SC_REQUIRE(jobs && n == b->jobs.size(), SC_E_INVALID, "expected %zu jobs", b->jobs.size());
    for (uint32_t i = 0; i < n; ++i) {
        int rc = check_job(jobs[i], i);
        if (rc != SC_OK) return rc;
        const sc_scene_job& o = b->jobs[i];
        SC_REQUIRE(jobs[i].width == o.width && jobs[i].height == o.height && jobs[i].n_photons == o.n_photons &&
                       jobs[i].opts.bins == o.opts.bins && jobs[i].opts.lambda_min == o.opts.lambda_min &&
                       jobs[i].opts.lambda_max == o.opts.lambda_max,
                   SC_E_STATE, "job %u changes its film or photon budget; create a new batch", i);
    }
    b->jobs.assign(jobs, jobs + n);
    if (b->any_free_flight() != b->ff) {  // another kernel: new grid and graph
        const int rc = b->apply_tuning(b->tuning);
        if (rc != SC_OK) return rc;
    }
    return b->upload_jobs();  // stream-ordered before the next run on the same stream
    SC_GUARD_END
}

int sc_batch_run(sc_batch* b, void* stream) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
    if (s != b->stream) {  // order after uploads made on the batch's own stream
        SC_CUDA(cudaEventRecord(b->uploaded, b->stream));
        SC_CUDA(cudaStreamWaitEvent(s, b->uploaded, 0));
    }
    return b->run(s);
    SC_GUARD_END
}

int sc_batch_run_plain(sc_batch* b, void* stream) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    return b->run_plain(stream ? static_cast<cudaStream_t>(stream) : b->stream);
    SC_GUARD_END
}

int sc_batch_synchronize(sc_batch* b) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    SC_CUDA(cudaStreamSynchronize(b->stream));
    if (b->graph_stream) SC_CUDA(cudaStreamSynchronize(b->graph_stream));
    SC_CUDA(cudaStreamSynchronize(b->copy_stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_batch_read_xyz(sc_batch* b, uint32_t job, float* out) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    SC_REQUIRE(out && job < b->jobs.size(), SC_E_INVALID, "bad job %u or null output", job);
    SC_CUDA(cudaDeviceSynchronize());
    SC_CUDA(cudaMemcpy(out, b->xyz.p + b->xyz_off[job], 3ull * b->geom[job].w * b->geom[job].h * sizeof(float),
                       cudaMemcpyDeviceToHost));
    return SC_OK;
    SC_GUARD_END
}

int sc_batch_read_all_xyz(sc_batch* b, float* out, size_t capacity, void* stream) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    SC_REQUIRE(out && capacity >= b->xyz.n, SC_E_INVALID, "output holds %zu floats, need %zu", capacity, b->xyz.n);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->stream;
    SC_CUDA(cudaStreamWaitEvent(s, b->ran, 0));
    SC_CUDA(cudaMemcpyAsync(out, b->xyz.p, b->xyz.bytes(), cudaMemcpyDeviceToHost, s));
    SC_CUDA(cudaStreamSynchronize(s));
    return SC_OK;
    SC_GUARD_END
}

int sc_batch_read_all_xyz_async(sc_batch* b, float* out, size_t capacity, void* stream) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    SC_REQUIRE(out && capacity >= b->xyz.n, SC_E_INVALID, "output holds %zu floats, need %zu", capacity, b->xyz.n);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b->copy_stream;
    SC_CUDA(cudaStreamWaitEvent(s, b->ran, 0));
    SC_CUDA(cudaMemcpyAsync(out, b->xyz.p, b->xyz.bytes(), cudaMemcpyDeviceToHost, s));
    SC_CUDA(cudaEventRecord(b->copied, s));
    return SC_OK;
    SC_GUARD_END
}

int sc_batch_info(sc_batch* b, uint64_t* total_photons, uint64_t* film_bytes, uint64_t* xyz_floats,
                  uint64_t* job_table_bytes) {
    SC_GUARD_BEGIN
    SC_REQUIRE(b, SC_E_INVALID, "null batch");
    if (job_table_bytes) *job_table_bytes = b->jobs.size() * sizeof(BatchJobDev);
    if (total_photons) *total_photons = b->total_photons;
    if (film_bytes) *film_bytes = b->films.bytes();
    if (xyz_floats) *xyz_floats = b->xyz.n;
    return SC_OK;
    SC_GUARD_END
}

int sc_batch_stats(sc_batch* b, uint64_t out[6]) {
    SC_GUARD_BEGIN
    BATCH_LOCK(b);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    DevBuf<unsigned long long> d;
    SC_CUDA(d.alloc(4));
    SC_CUDA(cudaMemsetAsync(d.p, 0, 32, b->stream));
    for (uint32_t j = 0; j < b->jobs.size(); ++j) {
        PhotonParams p = b->job_params(j);
        const unsigned char* base = reinterpret_cast<const unsigned char*>(b->d_jobs.p + j);
        p.prims = reinterpret_cast<const sc_primitive*>(base + offsetof(BatchSlotImage, prims));
        p.planes = reinterpret_cast<const sc_plane*>(base + offsetof(BatchSlotImage, planes));
        p.mats = reinterpret_cast<const sc_material*>(base + offsetof(BatchSlotImage, mats));
        SC_CUDA(launch_photon_count(p, d.p, (uint32_t)b->ctx->sms * 8u, b->stream));
    }
    unsigned long long c[4];
    SC_CUDA(cudaMemcpyAsync(c, d.p, 32, cudaMemcpyDeviceToHost, b->stream));
    // dirty tiles of one pass: trace only, count the set bits, then drain
    SC_CUDA(launch_batch(b->d_jobs.p, b->d_items.p, b->n_items, b->counter.p, b->ctx->cmf.p, kBatchMaskWords,
                         (int)b->tuning.aggregate, (int)b->tuning.minb, b->tuning.per_photon ? 0 : 1, b->grid,
                         b->stream, b->tuning.block, b->ff));
    std::vector<uint32_t> fl(b->flags.n);
    SC_CUDA(cudaMemcpyAsync(fl.data(), b->flags.p, b->flags.bytes(), cudaMemcpyDeviceToHost, b->stream));
    SC_CUDA(cudaStreamSynchronize(b->stream));
    uint64_t dirty = 0, dirty_bytes = 0;
    for (uint32_t j = 0; j < b->jobs.size(); ++j) {
        uint64_t dj = 0;
        for (uint32_t w = 0; w < b->geom[j].words; ++w) dj += __builtin_popcount(fl[b->flag_off[j] + w]);
        dirty += dj;
        dirty_bytes += dj * kTilePixels * b->geom[j].channels * 8u;
    }
    SC_CUDA(launch_reduce_many(b->d_descs.p, (uint32_t)b->jobs.size(), b->total_words, true, b->max_channels,
                               b->dirty_list.p, b->dirty_count.p, b->stream));
    SC_CUDA(cudaStreamSynchronize(b->stream));
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[3]; out[4] = dirty; out[5] = dirty_bytes;
    return SC_OK;
    SC_GUARD_END
}

int sc_batch_device_xyz(sc_batch* b, uint32_t job, const float** xyz_dev) {
    SC_GUARD_BEGIN
    SC_REQUIRE(b && xyz_dev && job < b->jobs.size(), SC_E_INVALID, "bad argument");
    *xyz_dev = b->xyz.p + b->xyz_off[job];
    return SC_OK;
    SC_GUARD_END
}

}  // extern "C"
