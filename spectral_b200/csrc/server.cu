// Serving loop: continuous batching of render requests.
//
// * Memory: one device arena of the configured HBM budget, carved by a best-fit
//   free list on the host, so admitting and retiring requests never calls
//   cudaMalloc / cudaFree (which would stall the device).
// * Admission: queued requests are admitted in arrival order whenever a slot is
//   free and their film + flags + image fit in the arena (first fit: a request
//   that does not fit yet does not block smaller ones behind it).  A request
//   that could never fit the budget is rejected at submission.
// * Step: the current frame of EVERY active request is traced by one persistent
//   batch launch (batch.cu) and drained/sensor-reduced by one launch over all
//   active films; newly arrived requests join at the next step.
// * State on the device per request: its film, dirty mask and image.  The RNG
//   state of a request is its photon index: frame f traces photons
//   [f*N, (f+1)*N) of the request's own stream, so a request's result does not
//   depend on what else is in the batch.
// * Orbit sessions move the camera by a fixed azimuth step around their target
//   every frame (the film restarts each frame, as the reference viewer resets
//   its accumulation on a camera move); the last frame's image is returned.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <map>
#include <vector>

#include "batch.h"
#include "host_util.h"

using namespace sc;

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Best-fit allocator over [0, capacity) with coalescing; offsets aligned to 256 B.
class Arena {
  public:
    void reset(uint64_t cap) { free_.clear(); free_[0] = cap; cap_ = cap; used_ = 0; }
    bool alloc(uint64_t bytes, uint64_t& off) {
        bytes = (bytes + 255u) & ~uint64_t(255);
        auto best = free_.end();
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= bytes && (best == free_.end() || it->second < best->second)) best = it;
        if (best == free_.end()) return false;
        off = best->first;
        const uint64_t rest = best->second - bytes;
        free_.erase(best);
        if (rest) free_[off + bytes] = rest;
        used_ += bytes;
        return true;
    }
    void release(uint64_t off, uint64_t bytes) {
        bytes = (bytes + 255u) & ~uint64_t(255);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) { it->second += nx->second; free_.erase(nx); }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) { pv->second += it->second; free_.erase(it); }
        }
    }
    uint64_t used() const { return used_; }
    uint64_t capacity() const { return cap_; }

  private:
    std::map<uint64_t, uint64_t> free_;
    uint64_t cap_ = 0, used_ = 0;
};

struct Request {
    uint64_t id = 0;
    sc_request r{};
    uint32_t frame = 0;
    double t_submit = 0, t_admit = 0, t_first = 0, t_done = 0;
    uint64_t off = 0, bytes = 0;
    uint32_t tiles_x = 0, tiles_y = 0, words = 0;
    size_t film_cells = 0;
    std::vector<float> result;
};

uint64_t request_bytes(const sc_scene_job& j, uint32_t& tiles_x, uint32_t& tiles_y, uint32_t& words, size_t& cells) {
    tiles_x = (j.width + 7u) / 8u;
    tiles_y = (j.height + 7u) / 8u;
    words = flag_words(j.width, j.height);
    cells = (size_t)tiles_x * tiles_y * kTilePixels * j.opts.bins;
    auto up = [](uint64_t b) { return (b + 255u) & ~uint64_t(255); };
    return up(cells * 8) + up(words * 4ull) + up(3ull * j.width * j.height * 4) + up(3ull * j.opts.bins * 4);
}

}  // namespace

struct sc_server {
    sc_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    sc_server_config cfg{};
    Arena arena;
    DevBuf<unsigned char> mem;
    DevBuf<BatchJobDev> d_jobs;
    DevBuf<FilmDesc> d_descs;
    DevBuf<WorkItem> d_items;
    DevBuf<DirtyTile> dirty_list;  // reduce scratch, grown to the active films' tiles
    DevBuf<uint32_t> counter, dirty_count;
    std::deque<Request*> queue;
    std::vector<Request*> active;
    std::deque<Request*> finished;
    uint64_t next_id = 1, photons = 0;
    uint32_t grid = 0;
    std::vector<BatchJobDev> h_jobs;
    std::vector<FilmDesc> h_descs;
    std::vector<WorkItem> h_items;

    unsigned long long* film_ptr(const Request* q) { return reinterpret_cast<unsigned long long*>(mem.p + q->off); }
    uint32_t* flags_ptr(const Request* q) {
        return reinterpret_cast<uint32_t*>(mem.p + q->off + ((q->film_cells * 8 + 255u) & ~size_t(255)));
    }
    float* xyz_ptr(const Request* q) {
        return reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(flags_ptr(q)) +
                                        ((q->words * 4ull + 255u) & ~uint64_t(255)));
    }
    float* binw_ptr(const Request* q) {
        const sc_scene_job& j = q->r.job;
        return reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(xyz_ptr(q)) +
                                        ((3ull * j.width * j.height * 4 + 255u) & ~uint64_t(255)));
    }

    sc_camera frame_camera(const Request* q) const {
        const sc_request& r = q->r;
        if (r.orbit_deg == 0.0f || q->frame == 0) return r.job.cam;
        const double a = (double)r.orbit_deg * q->frame * 3.14159265358979323846 / 180.0;
        const double dx = r.job.cam.origin[0] - r.orbit_target[0], dz = r.job.cam.origin[2] - r.orbit_target[2];
        float o[3] = {(float)(r.orbit_target[0] + dx * std::cos(a) + dz * std::sin(a)), r.job.cam.origin[1],
                      (float)(r.orbit_target[2] - dx * std::sin(a) + dz * std::cos(a))};
        sc_camera c;
        sc_camera_look_at(o, r.orbit_target, r.orbit_up, r.vfov_deg, (float)r.job.width / (float)r.job.height, &c);
        return c;
    }

    int admit(double t) {
        for (auto it = queue.begin(); it != queue.end();) {
            if (active.size() >= cfg.max_slots) break;
            Request* q = *it;
            uint64_t off;
            if (!arena.alloc(q->bytes, off)) { ++it; continue; }
            q->off = off;
            q->t_admit = t;
            SC_CUDA(cudaMemsetAsync(film_ptr(q), 0, q->film_cells * 8, stream));
            SC_CUDA(cudaMemsetAsync(flags_ptr(q), 0, q->words * 4ull, stream));
            std::vector<float> w(3 * q->r.job.opts.bins);
            bin_weights(ctx->tables, q->r.job.opts.bins, q->r.job.opts.lambda_min, q->r.job.opts.lambda_max, w.data());
            SC_CUDA(cudaMemcpyAsync(binw_ptr(q), w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
            SC_CUDA(cudaStreamSynchronize(stream));  // the host vector goes out of scope
            active.push_back(q);
            it = queue.erase(it);
        }
        return SC_OK;
    }

    int step(uint32_t* n_active) {
        const double t0 = now_s();
        int rc = admit(t0);
        if (rc != SC_OK) return rc;
        if (active.empty()) { if (n_active) *n_active = 0; return SC_OK; }
        const uint32_t n = (uint32_t)active.size();
        h_jobs.resize(n);
        h_descs.resize(n);
        h_items.clear();
        uint32_t tiles = 0, words = 0, maxc = 0;
        uint64_t step_photons = 0;
        std::vector<uint32_t> order(n);
        for (uint32_t i = 0; i < n; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
            return active[a]->r.job.n_photons > active[b]->r.job.n_photons;
        });
        for (uint32_t i = 0; i < n; ++i) {
            Request* q = active[i];
            const sc_scene_job& J = q->r.job;
            PhotonParams p;
            std::memset(&p, 0, sizeof p);
            const sc_camera cam = frame_camera(q);
            p.corner = ld3(J.beam.corner); p.bu = ld3(J.beam.u); p.bv = ld3(J.beam.v); p.bdir = ld3(J.beam.dir);
            p.proj = make_proj(cam);
            p.width = J.width; p.height = J.height; p.tiles_x = q->tiles_x; p.channels = J.opts.bins;
            p.photon_count = J.n_photons; p.seed = J.seed;
            p.max_bounces = J.opts.max_bounces ? J.opts.max_bounces : 8u;
            p.sigma_s = J.weights.sigma_s; p.sigma_t = J.weights.sigma_t; p.g = J.weights.g; p.max_dist = J.max_dist;
            p.lambda_min = J.opts.lambda_min; p.lambda_range = J.opts.lambda_max - J.opts.lambda_min;
            p.bins = J.opts.bins; p.bin_min = J.opts.lambda_min; p.bin_inv_width = (float)J.opts.bins / p.lambda_range;
            p.scale = std::ldexp(1.0f, (int)(J.opts.scale_log2 ? J.opts.scale_log2 : 32u));
            p.spectral = J.spectral; p.estimator = J.opts.estimator;
            p.film = film_ptr(q); p.flags = flags_ptr(q);
            p.n_prims = J.n_prims; p.n_planes = J.n_planes; p.n_mats = J.n_mats;
            p.cmf = ctx->cmf.p;
            BatchJobDev& d = h_jobs[i];
            std::memset(&d, 0, sizeof d);
            d.slot_image.p = p;
            std::memcpy(d.slot_image.prims, J.prims, sizeof d.slot_image.prims);
            std::memcpy(d.slot_image.planes, J.planes, sizeof d.slot_image.planes);
            std::memcpy(d.slot_image.mats, J.mats, sizeof d.slot_image.mats);
            d.flags = p.flags;
            d.mask_words = q->words;
            FilmDesc& fd = h_descs[i];
            fd.film = p.film; fd.flags = p.flags; fd.xyz = xyz_ptr(q); fd.binw = binw_ptr(q);
            fd.width = J.width; fd.height = J.height; fd.tiles_x = q->tiles_x; fd.tiles_y = q->tiles_y;
            fd.channels = J.opts.bins; fd.word_begin = words;
            fd.inv_scale = std::ldexp(1.0, -(int)(J.opts.scale_log2 ? J.opts.scale_log2 : 32u));
            tiles += q->tiles_x * q->tiles_y;
            words += q->words;
            maxc = std::max(maxc, J.opts.bins);
            step_photons += J.n_photons;
        }
        const uint32_t chunk = cfg.chunk_photons;
        for (uint32_t i : order) {
            const Request* q = active[i];
            const uint32_t N = q->r.job.n_photons, base = q->frame * N;
            for (uint32_t b = 0; b < N; b += chunk) h_items.push_back(WorkItem{i, base + b, std::min(chunk, N - b)});
        }
        if (d_items.n < h_items.size()) SC_CUDA(d_items.alloc(h_items.size() * 2));
        if (dirty_list.n < tiles) SC_CUDA(dirty_list.alloc(tiles * 2ull));
        SC_CUDA(cudaMemcpyAsync(d_jobs.p, h_jobs.data(), n * sizeof(BatchJobDev), cudaMemcpyHostToDevice, stream));
        SC_CUDA(cudaMemcpyAsync(d_descs.p, h_descs.data(), n * sizeof(FilmDesc), cudaMemcpyHostToDevice, stream));
        SC_CUDA(cudaMemcpyAsync(d_items.p, h_items.data(), h_items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                                stream));
        SC_CUDA(launch_batch(d_jobs.p, d_items.p, (uint32_t)h_items.size(), counter.p, ctx->cmf.p, kBatchMaskWords, 0,
                             4, 1, grid, stream));
        SC_CUDA(launch_reduce_many(d_descs.p, n, words, true, maxc, dirty_list.p, dirty_count.p, stream));
        SC_CUDA(cudaStreamSynchronize(stream));
        const double t1 = now_s();
        photons += step_photons;
        std::vector<Request*> still;
        for (Request* q : active) {
            if (q->frame == 0) q->t_first = t1;
            ++q->frame;
            if (q->frame >= q->r.frames) {
                const size_t nf = 3ull * q->r.job.width * q->r.job.height;
                q->result.resize(nf);
                SC_CUDA(cudaMemcpy(q->result.data(), xyz_ptr(q), nf * sizeof(float), cudaMemcpyDeviceToHost));
                q->t_done = now_s();
                arena.release(q->off, q->bytes);
                finished.push_back(q);
            } else {
                still.push_back(q);
            }
        }
        active.swap(still);
        if (n_active) *n_active = (uint32_t)active.size();
        return SC_OK;
    }
};

extern "C" {

int sc_server_create(sc_ctx* ctx, const sc_server_config* cfg, sc_server** out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && cfg && out, SC_E_INVALID, "null argument");
    SC_REQUIRE(cfg->hbm_budget_bytes >= (1u << 20), SC_E_INVALID, "budget below 1 MiB");
    *out = nullptr;
    sc_server* s = new sc_server();
    s->ctx = ctx;
    s->cfg = *cfg;
    if (s->cfg.max_slots == 0) s->cfg.max_slots = 256;
    if (s->cfg.chunk_photons == 0) s->cfg.chunk_photons = 2048;
    s->cfg.chunk_photons = std::max(32u, (s->cfg.chunk_photons + 31u) / 32u * 32u);
    DeviceGuard g(ctx->device);
    auto fail = [&](cudaError_t e) {
        set_error("server setup failed: %s", cudaGetErrorString(e));
        if (s->stream) cudaStreamDestroy(s->stream);
        delete s;
        return e == cudaErrorMemoryAllocation ? SC_E_NOMEM : SC_E_CUDA;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e);
    if ((e = s->mem.alloc(cfg->hbm_budget_bytes)) != cudaSuccess) return fail(e);
    if ((e = s->d_jobs.alloc(s->cfg.max_slots)) != cudaSuccess) return fail(e);
    if ((e = s->d_descs.alloc(s->cfg.max_slots)) != cudaSuccess) return fail(e);
    if ((e = s->counter.alloc(1)) != cudaSuccess) return fail(e);
    if ((e = s->dirty_count.alloc(1)) != cudaSuccess) return fail(e);
    s->arena.reset(cfg->hbm_budget_bytes);
    s->grid = (uint32_t)(ctx->sms * batch_occupancy(0, 4, 1, kBatchMaskWords));
    *out = s;
    return SC_OK;
    SC_GUARD_END
}

int sc_server_destroy(sc_server* s) {
    SC_GUARD_BEGIN
    if (!s) return SC_OK;
    {
        DeviceGuard g(s->ctx->device);
        if (s->stream) cudaStreamSynchronize(s->stream);
        for (Request* q : s->queue) delete q;
        for (Request* q : s->active) delete q;
        for (Request* q : s->finished) delete q;
        s->mem.reset(); s->d_jobs.reset(); s->d_descs.reset(); s->d_items.reset(); s->counter.reset();
        if (s->stream) cudaStreamDestroy(s->stream);
    }
    delete s;
    return SC_OK;
    SC_GUARD_END
}

#define SERVER_LOCK(s)                                       \
    SC_REQUIRE((s), SC_E_INVALID, "null server");            \
    std::lock_guard<std::mutex> _lk((s)->mu);                \
    DeviceGuard _dg((s)->ctx->device)

int sc_server_submit(sc_server* s, const sc_request* r, uint64_t* id) {
    SC_GUARD_BEGIN
    SERVER_LOCK(s);
    SC_REQUIRE(r && id, SC_E_INVALID, "null argument");
    const sc_scene_job& j = r->job;
    SC_REQUIRE(j.n_prims <= kBatchPrims && j.n_planes <= kBatchPlanes && j.n_mats <= kBatchPrims, SC_E_LIMIT,
               "request scene exceeds %u primitives / %u planes", kBatchPrims, kBatchPlanes);
    for (uint32_t k = 0; k < j.n_prims; ++k)
        SC_REQUIRE(j.prims[k].kind <= 1u && j.prims[k].material < j.n_mats &&
                       (j.prims[k].kind == 0u || (uint64_t)j.prims[k].plane_start + j.prims[k].plane_count <= j.n_planes),
                   SC_E_INVALID, "request primitive %u invalid", k);
    for (uint32_t k = 0; k < j.n_mats; ++k)
        SC_REQUIRE(j.mats[k].kind <= 1u && (j.mats[k].kind == 0u || j.mats[k].glass <= 3u), SC_E_INVALID,
                   "request material %u invalid", k);
    SC_REQUIRE(j.width > 0 && j.height > 0 && (uint64_t)j.width * j.height <= (1ull << 26), SC_E_INVALID, "film");
    SC_REQUIRE(j.opts.bins >= 1 && j.opts.bins <= SC_MAX_BINS, SC_E_INVALID, "bins %u", j.opts.bins);
    SC_REQUIRE(j.opts.lambda_max > j.opts.lambda_min && j.opts.lambda_min > 0.0f, SC_E_INVALID, "band");
    SC_REQUIRE(r->frames >= 1 && (uint64_t)r->frames * j.n_photons <= 0xFFFFFFFFull, SC_E_INVALID,
               "frames x photons must fit 32-bit photon indices");
    Request* q = new Request();
    q->r = *r;
    q->bytes = request_bytes(j, q->tiles_x, q->tiles_y, q->words, q->film_cells);
    if (q->bytes > s->arena.capacity()) {
        set_error("request needs %llu bytes, budget is %llu", (unsigned long long)q->bytes,
                  (unsigned long long)s->arena.capacity());
        delete q;
        return SC_E_NOMEM;
    }
    q->id = s->next_id++;
    q->t_submit = now_s();
    s->queue.push_back(q);
    *id = q->id;
    return SC_OK;
    SC_GUARD_END
}

int sc_server_step(sc_server* s, uint32_t* active) {
    SC_GUARD_BEGIN
    SERVER_LOCK(s);
    return s->step(active);
    SC_GUARD_END
}

int sc_server_poll(sc_server* s, uint64_t* id, float* xyz_out, size_t capacity, uint32_t* width, uint32_t* height,
                   double times[4]) {
    SC_GUARD_BEGIN
    SERVER_LOCK(s);
    SC_REQUIRE(id, SC_E_INVALID, "null id");
    if (s->finished.empty()) { set_error("no finished request"); return SC_E_STATE; }
    Request* q = s->finished.front();
    if (xyz_out) {
        SC_REQUIRE(capacity >= q->result.size(), SC_E_INVALID, "output holds %zu floats, need %zu", capacity,
                   q->result.size());
        std::memcpy(xyz_out, q->result.data(), q->result.size() * sizeof(float));
    }
    *id = q->id;
    if (width) *width = q->r.job.width;
    if (height) *height = q->r.job.height;
    if (times) { times[0] = q->t_submit; times[1] = q->t_admit; times[2] = q->t_first; times[3] = q->t_done; }
    s->finished.pop_front();
    delete q;
    return SC_OK;
    SC_GUARD_END
}

int sc_server_cancel(sc_server* s, uint64_t id) {
    SC_GUARD_BEGIN
    SERVER_LOCK(s);
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it)
        if ((*it)->id == id) { delete *it; s->queue.erase(it); return SC_OK; }
    for (auto it = s->active.begin(); it != s->active.end(); ++it)
        if ((*it)->id == id) {  // between steps nothing of this request is in flight
            s->arena.release((*it)->off, (*it)->bytes);
            delete *it;
            s->active.erase(it);
            return SC_OK;
        }
    set_error("request %llu is not queued or active", (unsigned long long)id);
    return SC_E_STATE;
    SC_GUARD_END
}

int sc_server_stats(sc_server* s, uint64_t* photons_traced, uint64_t* bytes_in_use, uint32_t* queued,
                    uint32_t* active, uint32_t* finished) {
    SC_GUARD_BEGIN
    SERVER_LOCK(s);
    if (photons_traced) *photons_traced = s->photons;
    if (bytes_in_use) *bytes_in_use = s->arena.used();
    if (queued) *queued = (uint32_t)s->queue.size();
    if (active) *active = (uint32_t)s->active.size();
    if (finished) *finished = (uint32_t)s->finished.size();
    return SC_OK;
    SC_GUARD_END
}

}  // extern "C"
