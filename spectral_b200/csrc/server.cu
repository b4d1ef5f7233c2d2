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
// * Pipelining: a step only queues its work on the server's stream (tables go
//   up from pinned staging, two sets used in turn) and returns, so the host
//   prepares step k + 1 while the device runs step k.  Everything a request
//   owns on the device is touched only by work on that one stream, in order,
//   so its arena range can be handed to the next request as soon as its last
//   frame is queued.  The images of requests that finished in a step are
//   copied behind the step into a pinned host ring (allocated once), and the
//   request becomes pollable once that copy is done.
// * State on the device per request: its film, dirty mask and image.  The RNG
//   state of a request is its photon index: frame f traces photons
//   [f*N, (f+1)*N) of the request's own stream, so a request's result does not
//   depend on what else is in the batch.
// * Progressive sessions (several frames, a fixed camera) add every frame into
//   the request's resident film, as the reference viewer accumulates frame
//   after frame (spectral-viewer/src/main.rs:395-419): that film is never
//   drained, and each frame's image is the accumulated film over the frames so
//   far, scaled by 1 / frames (the viewer's normalisation by total photons, at
//   the per-frame photon count), so it keeps the brightness of one frame.
//   Orbit sessions move the camera by a fixed azimuth step around their target
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

// Pinned host memory for finished images: one ring allocated at creation.
// Images are taken in the order requests finish and given back in the order
// they are polled, which is the same order, so the ring is a FIFO of ranges.
class PinnedRing {
  public:
    cudaError_t init(size_t floats) {
        cap_ = floats;
        return cudaMallocHost(reinterpret_cast<void**>(&base_), cap_ * sizeof(float));
    }
    float* get(size_t n) {
        if (!base_ || n > cap_) return nullptr;
        if (live_.empty()) { live_.push_back({0, n}); return base_; }
        const size_t t = live_.front().first, h = live_.back().first + live_.back().second;
        size_t at;
        if (h > t) {  // free: [h, cap) and [0, t)
            if (cap_ - h >= n) at = h;
            else if (t >= n) at = 0;
            else return nullptr;
        } else {      // wrapped: free [h, t)
            if (t - h >= n) at = h;
            else return nullptr;
        }
        live_.push_back({at, n});
        return base_ + at;
    }
    void pop() { if (!live_.empty()) live_.pop_front(); }
    size_t capacity() const { return cap_; }
    void release() {
        if (base_) cudaFreeHost(base_);
        base_ = nullptr;
        live_.clear();
    }

  private:
    float* base_ = nullptr;
    size_t cap_ = 0;
    std::deque<std::pair<size_t, size_t>> live_;
};
constexpr size_t kRingFloats = size_t(64) << 20;  // 256 MB: twenty 1024x1024 images

struct Request {
    uint64_t id = 0;
    sc_request r{};
    uint32_t frame = 0;
    double t_submit = 0, t_admit = 0, t_first = 0, t_done = 0;
    uint64_t off = 0, bytes = 0;
    uint32_t tiles_x = 0, tiles_y = 0, words = 0;
    size_t film_cells = 0;
    const float* binw = nullptr;  // bin-averaged CMF of its (bins, band), shared through the context
    float* image = nullptr;       // pinned copy of the last frame's XYZ image
    bool image_own = false;       // its own pinned allocation (larger than the ring), not a ring range
};

// Film, dirty mask and image of one request in the arena.
uint64_t request_bytes(const sc_scene_job& j, uint32_t& tiles_x, uint32_t& tiles_y, uint32_t& words, size_t& cells) {
    tiles_x = (j.width + 7u) / 8u;
    tiles_y = (j.height + 7u) / 8u;
    words = flag_words(j.width, j.height);
    cells = (size_t)tiles_x * tiles_y * kTilePixels * j.opts.bins;
    auto up = [](uint64_t b) { return (b + 255u) & ~uint64_t(255); };
    return up(cells * 8) + up(words * 4ull) + up(3ull * j.width * j.height * 4);
}

// One set of pinned upload tables; `used` is recorded after the copies that
// read it, so the host rewrites the set only after they ran.
struct HostStage {
    BatchJobDev* jobs = nullptr;
    FilmDesc* descs = nullptr;
    WorkItem* items = nullptr;
    size_t items_cap = 0;
    cudaEvent_t used = nullptr;
};

// A queued step: its completion event, the requests whose first frame it
// traces and those whose last frame it traces (their image copies follow it).
struct StepRecord {
    cudaEvent_t done = nullptr;
    std::vector<Request*> first, last;
};

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
    std::deque<StepRecord> inflight;  // queued steps, oldest first
    std::deque<Request*> finished;
    // Requests whose last frame is traced but whose image waits for room in
    // the ring (results not yet polled); they keep their arena range, so a
    // caller that does not poll holds admission back instead of pinning more
    // host memory.
    std::deque<Request*> unread;
    uint64_t next_id = 1, photons = 0;
    uint32_t grid = 0;
    HostStage stage[2];
    uint32_t stage_k = 0;
    PinnedRing ring;
    std::vector<cudaEvent_t> spare_events;
    std::vector<WorkItem> h_items;

    unsigned long long* film_ptr(const Request* q) { return reinterpret_cast<unsigned long long*>(mem.p + q->off); }
    uint32_t* flags_ptr(const Request* q) {
        return reinterpret_cast<uint32_t*>(mem.p + q->off + ((q->film_cells * 8 + 255u) & ~size_t(255)));
    }
    float* xyz_ptr(const Request* q) {
        return reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(flags_ptr(q)) +
                                        ((q->words * 4ull + 255u) & ~uint64_t(255)));
    }
    // Bin-averaged CMF of a (bins, band) on the device, kept by the context.
    int binw_for(const sc_film_options& o, const float** out) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        const auto key = std::make_tuple(o.bins, o.lambda_min, o.lambda_max);
        auto it = ctx->binw_cache.find(key);
        if (it == ctx->binw_cache.end()) {
            std::vector<float> w(3 * o.bins);
            bin_weights(ctx->tables, o.bins, o.lambda_min, o.lambda_max, w.data());
            std::unique_ptr<DevBuf<float>> buf(new DevBuf<float>());
            SC_CUDA(buf->alloc(w.size()));
            SC_CUDA(cudaMemcpy(buf->p, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
            it = ctx->binw_cache.emplace(key, std::move(buf)).first;
        }
        *out = it->second->p;
        return SC_OK;
    }

    cudaError_t event(cudaEvent_t* e) {
        if (!spare_events.empty()) {
            *e = spare_events.back();
            spare_events.pop_back();
            return cudaSuccess;
        }
        return cudaEventCreateWithFlags(e, cudaEventDisableTiming);
    }

    // Retire queued steps that are done (all of them, in order, when `wait`):
    // first-frame and done times; finished requests become pollable.
    int collect(bool wait) {
        while (!inflight.empty()) {
            StepRecord& r = inflight.front();
            if (wait) {
                SC_CUDA(cudaEventSynchronize(r.done));
            } else {
                const cudaError_t e = cudaEventQuery(r.done);
                if (e == cudaErrorNotReady) break;
                SC_CUDA(e);
            }
            const double t = now_s();
            for (Request* q : r.first) q->t_first = t;
            for (Request* q : r.last) {
                q->t_done = t;
                finished.push_back(q);
            }
            spare_events.push_back(r.done);
            inflight.pop_front();
        }
        return SC_OK;
    }

    // Requests whose images are still being produced or copied.
    uint32_t retiring() const {
        size_t n = unread.size();
        for (const StepRecord& r : inflight) n += r.last.size();
        return (uint32_t)n;
    }

    // Queue the image copies of waiting requests, oldest first, while the ring
    // has room; each joins `rec`, whose event follows the copies.  An image
    // larger than the whole ring, or every waiting image when `own` (nothing
    // else is left to trace), gets a pinned buffer of its own.
    int issue_unread(StepRecord& rec, bool own) {
        while (!unread.empty()) {
            Request* q = unread.front();
            const size_t nf = 3ull * q->r.job.width * q->r.job.height;
            q->image = ring.get(nf);
            if (!q->image) {
                if (!own && nf <= ring.capacity()) break;  // room comes back as results are polled
                SC_CUDA(cudaMallocHost(reinterpret_cast<void**>(&q->image), nf * sizeof(float)));
                q->image_own = true;
            }
            SC_CUDA(cudaMemcpyAsync(q->image, xyz_ptr(q), nf * sizeof(float), cudaMemcpyDeviceToHost, stream));
            arena.release(q->off, q->bytes);  // later users of the range queue behind this copy
            rec.last.push_back(q);
            unread.pop_front();
        }
        return SC_OK;
    }

    void free_image(Request* q) {
        if (!q->image) return;
        if (q->image_own) cudaFreeHost(q->image);
        else ring.pop();
        q->image = nullptr;
    }

    // Several frames on a fixed camera: the frames accumulate.
    static bool progressive(const Request* q) { return q->r.frames > 1u && q->r.orbit_deg == 0.0f; }

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
            int rc = binw_for(q->r.job.opts, &q->binw);
            if (rc != SC_OK) { arena.release(off, q->bytes); return rc; }
            // behind every earlier use of this range on the same stream
            SC_CUDA(cudaMemsetAsync(film_ptr(q), 0, q->film_cells * 8, stream));
            SC_CUDA(cudaMemsetAsync(flags_ptr(q), 0, q->words * 4ull, stream));
            active.push_back(q);
            it = queue.erase(it);
        }
        return SC_OK;
    }

    // The pinned table set for this step, with room for `items` work items.
    int stage_for(uint32_t items, HostStage** out) {
        HostStage& h = stage[stage_k];
        stage_k ^= 1u;
        if (!h.used) SC_CUDA(cudaEventCreateWithFlags(&h.used, cudaEventDisableTiming));
        else SC_CUDA(cudaEventSynchronize(h.used));  // its previous copies ran
        if (!h.jobs) {
            SC_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h.jobs), cfg.max_slots * sizeof(BatchJobDev)));
            SC_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h.descs), cfg.max_slots * sizeof(FilmDesc)));
        }
        if (h.items_cap < items) {
            if (h.items) cudaFreeHost(h.items);
            h.items = nullptr;
            h.items_cap = 0;
            SC_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h.items), (size_t)items * 2 * sizeof(WorkItem)));
            h.items_cap = (size_t)items * 2;
        }
        *out = &h;
        return SC_OK;
    }

    void release_all() {
        for (HostStage& h : stage) {
            if (h.jobs) cudaFreeHost(h.jobs);
            if (h.descs) cudaFreeHost(h.descs);
            if (h.items) cudaFreeHost(h.items);
            if (h.used) cudaEventDestroy(h.used);
            h = HostStage{};
        }
        for (StepRecord& r : inflight) spare_events.push_back(r.done);
        inflight.clear();
        for (cudaEvent_t e : spare_events) cudaEventDestroy(e);
        spare_events.clear();
        ring.release();
    }

    int step(uint32_t* n_active) {
        const double t0 = now_s();
        int rc = collect(false);
        if (rc == SC_OK) rc = admit(t0);
        if (rc != SC_OK) return rc;
        if (active.empty()) {
            // nothing to trace: finish what is still queued (a drain loop ends
            // here, also one that polls only at the end)
            if (!unread.empty()) {
                StepRecord rec;
                rc = issue_unread(rec, true);
                if (rc != SC_OK) return rc;
                SC_CUDA(event(&rec.done));
                SC_CUDA(cudaEventRecord(rec.done, stream));
                inflight.push_back(std::move(rec));
            }
            rc = collect(true);
            if (n_active) *n_active = 0;
            return rc;
        }
        const uint32_t n = (uint32_t)active.size();
        std::vector<uint32_t> order(n);
        for (uint32_t i = 0; i < n; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
            return active[a]->r.job.n_photons > active[b]->r.job.n_photons;
        });
        const uint32_t chunk = cfg.chunk_photons;
        h_items.clear();
        for (uint32_t i : order) {
            const Request* q = active[i];
            const uint32_t N = q->r.job.n_photons, base = q->frame * N;
            for (uint32_t b = 0; b < N; b += chunk) h_items.push_back(WorkItem{i, base + b, std::min(chunk, N - b)});
        }
        HostStage* h = nullptr;
        rc = stage_for((uint32_t)h_items.size(), &h);
        if (rc != SC_OK) return rc;
        std::memcpy(h->items, h_items.data(), h_items.size() * sizeof(WorkItem));
        uint32_t tiles = 0, words = 0, maxc = 0;
        uint64_t step_photons = 0;
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
            set_haze_consts(p);
            BatchJobDev& d = h->jobs[i];
            std::memset(&d, 0, sizeof d);
            d.slot_image.p = p;
            std::memcpy(d.slot_image.prims, J.prims, sizeof d.slot_image.prims);
            std::memcpy(d.slot_image.planes, J.planes, sizeof d.slot_image.planes);
            std::memcpy(d.slot_image.mats, J.mats, sizeof d.slot_image.mats);
            d.flags = p.flags;
            d.mask_words = q->words;
            FilmDesc& fd = h->descs[i];
            fd.film = p.film; fd.flags = p.flags; fd.xyz = xyz_ptr(q); fd.binw = q->binw;
            fd.width = J.width; fd.height = J.height; fd.tiles_x = q->tiles_x; fd.tiles_y = q->tiles_y;
            fd.channels = J.opts.bins; fd.word_begin = words;
            fd.keep = progressive(q) ? 1u : 0u;
            fd.inv_scale = std::ldexp(1.0, -(int)(J.opts.scale_log2 ? J.opts.scale_log2 : 32u)) /
                           (progressive(q) ? (double)(q->frame + 1u) : 1.0);
            tiles += q->tiles_x * q->tiles_y;
            words += q->words;
            maxc = std::max(maxc, J.opts.bins);
            step_photons += J.n_photons;
        }
        if (d_items.n < h_items.size() || dirty_list.n < tiles) {
            SC_CUDA(cudaStreamSynchronize(stream));  // queued steps still read the old tables (growth only)
            if (d_items.n < h_items.size()) SC_CUDA(d_items.alloc(h_items.size() * 2));
            if (dirty_list.n < tiles) SC_CUDA(dirty_list.alloc(tiles * 2ull));
        }
        SC_CUDA(cudaMemcpyAsync(d_jobs.p, h->jobs, n * sizeof(BatchJobDev), cudaMemcpyHostToDevice, stream));
        SC_CUDA(cudaMemcpyAsync(d_descs.p, h->descs, n * sizeof(FilmDesc), cudaMemcpyHostToDevice, stream));
        SC_CUDA(cudaMemcpyAsync(d_items.p, h->items, h_items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                                stream));
        SC_CUDA(cudaEventRecord(h->used, stream));
        bool ff = false;  // some request samples free-flight distances: the kernel built with them
        for (const Request* q : active) ff = ff || (q->r.job.opts.estimator == 3u && q->r.job.weights.sigma_t > 0.0f);
        SC_CUDA(launch_batch(d_jobs.p, d_items.p, (uint32_t)h_items.size(), counter.p, ctx->cmf.p, kBatchMaskWords, 0,
                             4, cfg.warp_split ? 1 : 0, grid, stream, 256, ff));
        SC_CUDA(launch_reduce_many(d_descs.p, n, words, true, maxc, dirty_list.p, dirty_count.p, stream));
        photons += step_photons;
        StepRecord rec;
        std::vector<Request*> still;
        for (Request* q : active) {
            if (q->frame == 0) rec.first.push_back(q);
            ++q->frame;
            if (q->frame >= q->r.frames) unread.push_back(q);
            else still.push_back(q);
        }
        active.swap(still);
        rc = issue_unread(rec, false);
        if (rc != SC_OK) return rc;
        SC_CUDA(event(&rec.done));
        SC_CUDA(cudaEventRecord(rec.done, stream));
        inflight.push_back(std::move(rec));
        // Queue depth: with requests waiting for admission, up to two steps
        // queued (the device never idles between steps); otherwise one, so a
        // new arrival waits behind at most the step being traced.
        const size_t depth = queue.empty() ? 1u : 2u;
        if (inflight.size() > depth) {
            rc = collect(false);
            while (rc == SC_OK && inflight.size() > depth) {
                SC_CUDA(cudaEventSynchronize(inflight.front().done));
                rc = collect(false);
            }
            if (rc != SC_OK) return rc;
        }
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
    if ((e = s->ring.init(kRingFloats)) != cudaSuccess) return fail(e);
    s->arena.reset(cfg->hbm_budget_bytes);
    s->cfg.warp_split = s->cfg.warp_split ? 1u : 0u;
    s->grid = (uint32_t)(ctx->sms * batch_occupancy(0, 4, (int)s->cfg.warp_split, kBatchMaskWords));
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
        for (StepRecord& r : s->inflight)
            for (Request* q : r.last) { if (q->image_own) cudaFreeHost(q->image); delete q; }
        for (Request* q : s->finished) { if (q->image_own) cudaFreeHost(q->image); delete q; }
        for (Request* q : s->unread) delete q;
        s->release_all();
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
    SC_REQUIRE(j.opts.estimator <= 1u || j.opts.estimator == 3u, SC_E_INVALID,
               "estimator %u: requests take the point, isotropic or free-flight estimator", j.opts.estimator);
    SC_REQUIRE(j.opts.lambda_max > j.opts.lambda_min && j.opts.lambda_min > 0.0f, SC_E_INVALID, "band");
    SC_REQUIRE(j.opts.haze_exact == 0u, SC_E_INVALID, "requests run the fast haze samples (haze_exact 0)");
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
    int rc = s->collect(false);
    if (rc != SC_OK) return rc;
    if (s->finished.empty()) { set_error("no finished request"); return SC_E_STATE; }
    Request* q = s->finished.front();
    const size_t nf = 3ull * q->r.job.width * q->r.job.height;
    if (xyz_out) {
        SC_REQUIRE(capacity >= nf, SC_E_INVALID, "output holds %zu floats, need %zu", capacity, nf);
        std::memcpy(xyz_out, q->image, nf * sizeof(float));
    }
    s->free_image(q);
    if (!s->unread.empty()) {  // ring room came back: queue the waiting images' copies
        StepRecord rec;
        rc = s->issue_unread(rec, false);
        if (rc == SC_OK && !rec.last.empty()) {
            cudaError_t e = s->event(&rec.done);
            if (e == cudaSuccess) e = cudaEventRecord(rec.done, s->stream);
            if (e == cudaSuccess) s->inflight.push_back(std::move(rec));
            else { set_error("%s", cudaGetErrorString(e)); rc = SC_E_CUDA; }
        }
    }
    *id = q->id;
    if (width) *width = q->r.job.width;
    if (height) *height = q->r.job.height;
    if (times) { times[0] = q->t_submit; times[1] = q->t_admit; times[2] = q->t_first; times[3] = q->t_done; }
    s->finished.pop_front();
    delete q;
    return rc;
    SC_GUARD_END
}

int sc_server_peek(sc_server* s, uint64_t id, float* xyz_out, size_t capacity, uint32_t* frames_done) {
    SC_GUARD_BEGIN
    SERVER_LOCK(s);
    SC_REQUIRE(xyz_out, SC_E_INVALID, "null output");
    Request* q = nullptr;
    for (Request* a : s->active)
        if (a->id == id) q = a;
    if (!q || q->frame == 0) {
        set_error("request %llu has no frame on the device (queued, finished or unknown)", (unsigned long long)id);
        return SC_E_STATE;
    }
    const size_t nf = 3ull * q->r.job.width * q->r.job.height;
    SC_REQUIRE(capacity >= nf, SC_E_INVALID, "output holds %zu floats, need %zu", capacity, nf);
    // behind every queued frame of the request: its image after q->frame frames
    SC_CUDA(cudaMemcpyAsync(xyz_out, s->xyz_ptr(q), nf * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    SC_CUDA(cudaStreamSynchronize(s->stream));
    if (frames_done) *frames_done = q->frame;
    return s->collect(false);
    SC_GUARD_END
}

int sc_server_cancel(sc_server* s, uint64_t id) {
    SC_GUARD_BEGIN
    SERVER_LOCK(s);
    for (auto it = s->queue.begin(); it != s->queue.end(); ++it)
        if ((*it)->id == id) { delete *it; s->queue.erase(it); return SC_OK; }
    for (auto it = s->active.begin(); it != s->active.end(); ++it)
        if ((*it)->id == id) {
            // frames of it may still be queued: its range is reused only by work
            // queued behind them on the same stream, and it leaves the queued
            // steps' first-frame lists before it is deleted
            for (StepRecord& r : s->inflight) r.first.erase(std::remove(r.first.begin(), r.first.end(), *it), r.first.end());
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
    if (active) *active = (uint32_t)s->active.size() + s->retiring();  // with images still on their way
    if (finished) *finished = (uint32_t)s->finished.size();
    return SC_OK;
    SC_GUARD_END
}

}  // extern "C"
