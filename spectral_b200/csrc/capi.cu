// extern "C" entry points: context, helpers, photon film, atomic film and the
// device-pointer launches.  The objects mirror the reference crate's
// GpuContext / GpuPhotonFilm / AtomicFilm (spectral-gpu/src/{lib,vol_photons,film}.rs).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <tuple>
#include <vector>

#include "host_util.h"
#include "internal.h"

namespace sc {

static thread_local std::string g_error;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
}

int check_scene(uint32_t n_prims, uint32_t n_planes, uint32_t n_mats, const sc_primitive* prims,
                const sc_plane* planes, const sc_material* mats) {
    SC_REQUIRE(n_prims <= SC_MAX_PRIMS, SC_E_LIMIT, "scene has %u primitives (max %d)", n_prims, SC_MAX_PRIMS);
    SC_REQUIRE(n_planes <= SC_MAX_PLANES, SC_E_LIMIT, "scene has %u planes (max %d)", n_planes, SC_MAX_PLANES);
    SC_REQUIRE(n_mats <= SC_MAX_PRIMS, SC_E_LIMIT, "scene has %u materials (max %d)", n_mats, SC_MAX_PRIMS);
    SC_REQUIRE(n_prims == 0 || prims, SC_E_INVALID, "null primitive array");
    SC_REQUIRE(n_planes == 0 || planes, SC_E_INVALID, "null plane array");
    SC_REQUIRE(n_mats == 0 || mats, SC_E_INVALID, "null material array");
    for (uint32_t i = 0; i < n_prims; ++i) {
        const sc_primitive& p = prims[i];
        SC_REQUIRE(p.kind <= 1u, SC_E_INVALID, "primitive %u has kind %u (0 sphere, 1 solid)", i, p.kind);
        SC_REQUIRE(p.material < n_mats, SC_E_INVALID, "primitive %u material %u out of range", i, p.material);
        if (p.kind == 1u)
            SC_REQUIRE((uint64_t)p.plane_start + p.plane_count <= n_planes, SC_E_INVALID,
                       "primitive %u plane range [%u,+%u) exceeds %u planes", i, p.plane_start, p.plane_count, n_planes);
    }
    for (uint32_t i = 0; i < n_mats; ++i) {
        SC_REQUIRE(mats[i].kind <= 1u, SC_E_INVALID, "material %u has kind %u", i, mats[i].kind);
        SC_REQUIRE(mats[i].kind == 0u || mats[i].glass <= 3u, SC_E_INVALID, "material %u glass %u", i, mats[i].glass);
    }
    return SC_OK;
}

struct FilmGeom {
    uint32_t w, h, tiles_x, tiles_y, channels;
    size_t cells() const { return (size_t)tiles_x * tiles_y * kTilePixels * channels; }
    size_t tiles() const { return (size_t)tiles_x * tiles_y; }
};
static FilmGeom film_geom(uint32_t w, uint32_t h, uint32_t channels) {
    FilmGeom g;
    g.w = w; g.h = h; g.channels = channels;
    g.tiles_x = (w + 7u) / 8u; g.tiles_y = (h + 7u) / 8u;
    return g;
}

static void resolve_options(const sc_film_options* in, sc_film_options& o) {
    std::memset(&o, 0, sizeof o);
    if (in) o = *in;
    if (o.lambda_min == 0.0f) o.lambda_min = 380.0f;
    if (o.lambda_max == 0.0f) o.lambda_max = 730.0f;
    if (o.max_bounces == 0u) o.max_bounces = 8u;
    if (o.scale_log2 == 0u) o.scale_log2 = 32u;
}

static size_t mask_smem(uint32_t w, uint32_t h) {
    const uint32_t words = flag_words(w, h);
    return words <= kMaxSmemMaskWords ? words * sizeof(uint32_t) : 0;
}

// The launch shape of single-film traces: 256-thread CTAs, 4 per SM, the
// warp-split transport, the wavelength-ordered dispatch for spectral films
// larger than L2.  The environment variables SPECTRAL_CUDA_AGGREGATE,
// SPECTRAL_CUDA_MINB (4 or 5), SPECTRAL_CUDA_SPLIT (0: one photon per lane) and
// SPECTRAL_CUDA_ORDER (0 never, 1 large spectral films, 2 every spectral film)
// override it for measurements; every setting gives the same film bits.
static int default_shape(sc_ctx* ctx, bool spectral, int aggregate, size_t smem, LaunchShape& s,
                         uint32_t estimator = 0) {
    s.block = 256;
    s.aggregate = aggregate;
    s.minb = 4;
    if (const char* agg = std::getenv("SPECTRAL_CUDA_AGGREGATE")) s.aggregate = std::atoi(agg) ? 1 : 0;
    if (const char* mb = std::getenv("SPECTRAL_CUDA_MINB")) s.minb = std::atoi(mb) >= 5 ? 5 : 4;
    if (const char* sp = std::getenv("SPECTRAL_CUDA_SPLIT")) s.split = std::atoi(sp) ? 1 : 0;
    if (const char* od = std::getenv("SPECTRAL_CUDA_ORDER")) s.order = std::min(std::max(std::atoi(od), 0), 2);
    s.pool = ctx->pool;
    const int per_sm = estimator == 2u ? beam_occupancy_blocks(s, spectral, smem)
                                       : photon_occupancy_blocks(s, spectral, smem);
    s.grid = (uint32_t)(ctx->sms * per_sm);
    return SC_OK;
}

}  // namespace sc

using namespace sc;

// --------------------------------------------------------------------------
// photon film object
// --------------------------------------------------------------------------
struct sc_photon_film {
    sc_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    FilmGeom geom{};
    sc_film_options opts{};
    sc_camera cam{};
    sc_beam beam{};
    sc_vol_weights weights{};
    uint32_t n_photons = 0, seed = 0, spectral = 1;
    float max_dist = 0.0f;
    uint32_t n_prims = 0, n_planes = 0, n_mats = 0;
    DevBuf<sc_primitive> prims;
    DevBuf<sc_plane> planes;
    DevBuf<sc_material> mats;
    DevBuf<float> zbuf;
    DevBuf<unsigned long long> film;
    DevBuf<uint32_t> flags;
    DevBuf<float> xyz, surface, binw;
    DevBuf<uint32_t> work;
    DevBuf<uint8_t> rgb;
    DevBuf<sc_debug_photon> debug;
    LaunchShape shape{};
    uint64_t film_version = 1, xyz_version = 0;

    void bind_pool() {
        if (!ctx->pool) return;  // no pool: plain cudaMalloc buffers
        prims.bind(ctx->pool, stream); planes.bind(ctx->pool, stream); mats.bind(ctx->pool, stream);
        zbuf.bind(ctx->pool, stream); film.bind(ctx->pool, stream); flags.bind(ctx->pool, stream);
        xyz.bind(ctx->pool, stream); surface.bind(ctx->pool, stream); binw.bind(ctx->pool, stream);
        work.bind(ctx->pool, stream); rgb.bind(ctx->pool, stream); debug.bind(ctx->pool, stream);
    }

    PhotonParams params(uint32_t base, uint32_t count, uint32_t s) const {
        PhotonParams p;
        std::memset(&p, 0, sizeof p);
        p.corner = ld3(beam.corner); p.bu = ld3(beam.u); p.bv = ld3(beam.v); p.bdir = ld3(beam.dir);
        p.proj = make_proj(cam);
        p.width = geom.w; p.height = geom.h; p.tiles_x = geom.tiles_x; p.channels = geom.channels;
        p.photon_base = base; p.photon_count = count; p.seed = s; p.max_bounces = opts.max_bounces;
        p.sigma_s = weights.sigma_s; p.sigma_t = weights.sigma_t; p.g = weights.g; p.max_dist = max_dist;
        p.lambda_min = opts.lambda_min; p.lambda_range = opts.lambda_max - opts.lambda_min;
        p.bins = opts.bins; p.bin_min = opts.lambda_min;
        p.bin_inv_width = opts.bins ? (float)opts.bins / p.lambda_range : 0.0f;
        p.scale = std::ldexp(1.0f, (int)opts.scale_log2);
        p.spectral = spectral; p.estimator = opts.estimator; p.haze_exact = opts.haze_exact;
        p.zbuf = zbuf.p; p.film = film.p; p.flags = flags.p;
        p.prims = prims.p; p.planes = planes.p; p.mats = mats.p;
        p.n_prims = n_prims; p.n_planes = n_planes; p.n_mats = n_mats;
        p.cmf = ctx->cmf.p;
        return p;
    }
    int trace(uint32_t base, uint32_t end, uint32_t s) {
        if (end <= base) return SC_OK;
        DeviceGuard g(ctx->device);
        PhotonParams p = params(base, end - base, s);
        if (opts.estimator == 2u) SC_CUDA(launch_beam(p, shape, stream));
        else SC_CUDA(launch_photons(p, shape, stream));
        ++film_version;
        return SC_OK;
    }
    int ensure_xyz() {
        if (xyz_version == film_version) return SC_OK;
        ReduceParams r;
        r.film = film.p; r.flags = flags.p; r.xyz = xyz.p; r.width = geom.w; r.height = geom.h;
        r.tiles_x = geom.tiles_x; r.tiles_y = geom.tiles_y; r.channels = geom.channels; r.binw = binw.p;
        r.inv_scale = std::ldexp(1.0, -(int)opts.scale_log2);
        SC_CUDA(launch_reduce(r, false, stream));
        xyz_version = film_version;
        return SC_OK;
    }
};

extern "C" {

const char* sc_last_error(void) { return g_error.c_str(); }
const char* sc_version(void) { return "spectral_cuda 0.1 (sm_100a)"; }

int sc_load_sensor_tables(const char* path, float* out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(path && out, SC_E_INVALID, "null argument");
    FILE* f = std::fopen(path, "r");
    SC_REQUIRE(f, SC_E_INVALID, "cannot open sensor table %s", path);
    char line[512];
    int row = 0;
    while (std::fgets(line, sizeof line, f) && row < kTableN) {
        if (line[0] == '#' || line[0] == 'n' || line[0] == '\n' || line[0] == '\r') continue;
        char* p = line;
        (void)std::strtof(p, &p);
        for (int c = 0; c < 5; ++c) {
            if (*p == ',') ++p;
            out[c * kTableN + row] = std::strtof(p, &p);  // correctly rounded, like str::parse::<f32>
        }
        ++row;
    }
    std::fclose(f);
    SC_REQUIRE(row == kTableN, SC_E_INVALID, "sensor table %s has %d rows (want %d)", path, row, kTableN);
    return SC_OK;
    SC_GUARD_END
}

int sc_ctx_create(int device, const float* tables, sc_ctx** out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(out && tables, SC_E_INVALID, "null argument");
    SC_REQUIRE(device >= 0, SC_E_INVALID, "device index %d", device);
    *out = nullptr;
    int count = 0;
    const cudaError_t ce = cudaGetDeviceCount(&count);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        set_error("no CUDA device: %s", cudaGetErrorString(ce));
        return SC_E_NODEVICE;
    }
    SC_REQUIRE(device < count, SC_E_NODEVICE, "device %d not present (%d devices)", device, count);
    cudaDeviceProp prop;
    SC_CUDA(cudaGetDeviceProperties(&prop, device));
    SC_REQUIRE(prop.major == 10, SC_E_NODEVICE, "device %d is sm_%d%d; this library is built for sm_100a only",
               device, prop.major, prop.minor);
    sc_ctx* c = new sc_ctx();
    c->device = device;
    c->sms = prop.multiProcessorCount;
    c->cc_major = prop.major; c->cc_minor = prop.minor;
    std::memcpy(c->tables, tables, sizeof c->tables);
    DeviceGuard g(device);
    cudaError_t e = c->cmf.alloc(3 * kTableN);
    if (e == cudaSuccess) e = cudaMemcpy(c->cmf.p, tables, 3 * kTableN * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        set_error("context setup failed: %s", cudaGetErrorString(e));
        delete c;
        return SC_E_CUDA;
    }
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&c->pool, &props) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    } else {
        cudaGetLastError();
        c->pool = nullptr;  // no pool: photon launches run in launch order
    }
    *out = c;
    return SC_OK;
    SC_GUARD_END
}

int sc_ctx_destroy(sc_ctx* ctx) {
    SC_GUARD_BEGIN
    if (!ctx) return SC_OK;
    {
        DeviceGuard g(ctx->device);
        ctx->cmf.reset();
        ctx->binw_cache.clear();
        if (ctx->pool) {
            cudaDeviceSynchronize();  // frees still queued on streams return their blocks first
            cudaMemPoolDestroy(ctx->pool);
        }
    }
    delete ctx;
    return SC_OK;
    SC_GUARD_END
}

int sc_ctx_synchronize(sc_ctx* ctx) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx, SC_E_INVALID, "null context");
    DeviceGuard g(ctx->device);
    SC_CUDA(cudaDeviceSynchronize());
    return SC_OK;
    SC_GUARD_END
}

int sc_camera_look_at(const float origin[3], const float target[3], const float up[3], float vfov_deg, float aspect,
                      sc_camera* out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(origin && target && up && out, SC_E_INVALID, "null argument");
    // Camera::look_at (spectral-core/src/camera.rs:15-27), f32 in the same order.
    const float rads_per_deg = 3.14159265358979323846f / 180.0f;
    const float theta = vfov_deg * rads_per_deg;
    const float h = std::tan(theta / 2.0f);
    const float vh = 2.0f * h, vw = aspect * vh;
    const f3 o = ld3(origin);
    const f3 w = normalize(sub(o, ld3(target)));
    const f3 u = normalize(cross(ld3(up), w));
    const f3 v = cross(w, u);
    const f3 hor = mul(u, vw), ver = mul(v, vh);
    const f3 ll = sub(sub(sub(o, vdiv(hor, 2.0f)), vdiv(ver, 2.0f)), w);
    out->origin[0] = o.x; out->origin[1] = o.y; out->origin[2] = o.z;
    out->lower_left[0] = ll.x; out->lower_left[1] = ll.y; out->lower_left[2] = ll.z;
    out->horizontal[0] = hor.x; out->horizontal[1] = hor.y; out->horizontal[2] = hor.z;
    out->vertical[0] = ver.x; out->vertical[1] = ver.y; out->vertical[2] = ver.z;
    return SC_OK;
    SC_GUARD_END
}

int sc_camera_proj_params(const sc_camera* cam, float out[16]) {
    SC_GUARD_BEGIN
    SC_REQUIRE(cam && out, SC_E_INVALID, "null argument");
    const Proj p = make_proj(*cam);  // the basis the photon kernels project with
    const float v[16] = {p.o.x, p.o.y, p.o.z, 0.0f, p.u.x, p.u.y, p.u.z, p.vw,
                         p.v.x, p.v.y, p.v.z, p.vh, p.w.x, p.w.y, p.w.z, 0.0f};
    std::memcpy(out, v, sizeof v);
    return SC_OK;
    SC_GUARD_END
}

float sc_glass_n(uint32_t glass, float lambda_nm) { return glass_n(glass, lambda_nm); }

int sc_glass_n_many(uint32_t glass, const float* lambda_nm, size_t n, float* out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(glass <= 3u, SC_E_INVALID, "glass %u", glass);
    SC_REQUIRE((lambda_nm && out) || n == 0, SC_E_INVALID, "null argument");
    for (size_t i = 0; i < n; ++i) out[i] = glass_n(glass, lambda_nm[i]);
    return SC_OK;
    SC_GUARD_END
}

int sc_glass_n_device(sc_ctx* ctx, uint32_t glass, const float* lambda_nm_dev, size_t n, float* out_dev,
                      void* stream) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx, SC_E_INVALID, "null context");
    SC_REQUIRE(glass <= 3u, SC_E_INVALID, "glass %u", glass);
    SC_REQUIRE((lambda_nm_dev && out_dev) || n == 0, SC_E_INVALID, "null argument");
    SC_REQUIRE(n <= (size_t(1) << 31), SC_E_LIMIT, "n %zu > 2^31", n);
    if (n == 0) return SC_OK;
    DeviceGuard g(ctx->device);
    SC_CUDA(launch_glass_n(glass, lambda_nm_dev, (uint32_t)n, out_dev, static_cast<cudaStream_t>(stream)));
    return SC_OK;
    SC_GUARD_END
}

int sc_rng_draws(sc_ctx* ctx, uint32_t key, uint32_t seed, uint32_t n, uint32_t* out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && (out || n == 0), SC_E_INVALID, "null argument");
    SC_REQUIRE(n <= (1u << 20), SC_E_INVALID, "n %u > 2^20", n);
    if (n == 0) return SC_OK;
    DeviceGuard g(ctx->device);
    DevBuf<uint32_t> d;
    SC_CUDA(d.alloc(n));
    SC_CUDA(launch_rng_draws(key, seed, n, d.p, 0));
    SC_CUDA(cudaMemcpy(out, d.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return SC_OK;
    SC_GUARD_END
}

int sc_dsotm_scene(float aspect, sc_primitive* prim, sc_plane* planes, sc_material* mat, sc_beam* beam,
                   sc_camera* cam) {
    SC_GUARD_BEGIN
    SC_REQUIRE(prim && planes && mat && beam && cam, SC_E_INVALID, "null argument");
    // dsotm_scene (spectral-gpu/src/vol_photons.rs:188-222).
    const float k = 0.9f;
    const float pl[5][4] = {{-0.8660254f, 0.5f, 0.0f, -k}, {0.8660254f, 0.5f, 0.0f, -k}, {0.0f, -1.0f, 0.0f, -1.0f},
                            {0.0f, 0.0f, 1.0f, -1.0f}, {0.0f, 0.0f, -1.0f, -1.0f}};
    for (int i = 0; i < 5; ++i) {
        planes[i].normal[0] = pl[i][0]; planes[i].normal[1] = pl[i][1]; planes[i].normal[2] = pl[i][2];
        planes[i].d = pl[i][3];
    }
    std::memset(prim, 0, sizeof *prim);
    prim->plane_start = 0; prim->plane_count = 5; prim->kind = 1; prim->material = 0;
    std::memset(mat, 0, sizeof *mat);
    mat->kind = 1; mat->glass = 1;  // SF11
    const f3 bdir = normalize(mk(0.84f, 0.54f, 0.0f));
    const f3 bperp = mul(normalize(mk(-0.54f, 0.84f, 0.0f)), 0.05f);
    const float corner[3] = {-2.6f, -0.95f, -0.6f}, u[3] = {0.0f, 0.0f, 1.2f};
    for (int i = 0; i < 3; ++i) { beam->corner[i] = corner[i]; beam->u[i] = u[i]; }
    beam->v[0] = bperp.x; beam->v[1] = bperp.y; beam->v[2] = bperp.z;
    beam->dir[0] = bdir.x; beam->dir[1] = bdir.y; beam->dir[2] = bdir.z;
    const float co[3] = {0.5f, -0.5f, 12.0f}, ct[3] = {0.5f, -0.5f, 0.0f}, up[3] = {0.0f, 1.0f, 0.0f};
    return sc_camera_look_at(co, ct, up, 42.0f, aspect, cam);
    SC_GUARD_END
}

// ---------------------------- photon film ---------------------------------
int sc_photon_film_create(sc_ctx* ctx, const sc_primitive* prims, uint32_t n_prims, const sc_plane* planes,
                          uint32_t n_planes, const sc_material* mats, uint32_t n_mats, float background,
                          const sc_camera* cam, const sc_beam* beam, uint32_t width, uint32_t height,
                          uint32_t n_photons, uint32_t seed, float max_dist, const sc_vol_weights* weights,
                          const float* zbuffer, const sc_film_options* opts, sc_photon_film** out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && cam && beam && weights && out, SC_E_INVALID, "null argument");
    *out = nullptr;
    int rc = check_scene(n_prims, n_planes, n_mats, prims, planes, mats);
    if (rc != SC_OK) return rc;
    SC_REQUIRE(width > 0 && height > 0, SC_E_INVALID, "film %ux%u is empty", width, height);
    SC_REQUIRE((uint64_t)width * height <= (1ull << 28), SC_E_LIMIT, "film %ux%u too large", width, height);
    sc_film_options o;
    resolve_options(opts, o);
    SC_REQUIRE(o.bins <= SC_MAX_BINS, SC_E_LIMIT, "%u bins (max %d)", o.bins, SC_MAX_BINS);
    SC_REQUIRE(o.lambda_max > o.lambda_min, SC_E_INVALID, "empty band [%g, %g)", o.lambda_min, o.lambda_max);
    SC_REQUIRE(o.scale_log2 <= 50u, SC_E_INVALID, "scale_log2 %u > 50", o.scale_log2);
    SC_REQUIRE(o.max_bounces <= 64u, SC_E_LIMIT, "max_bounces %u > 64", o.max_bounces);
    SC_REQUIRE(o.estimator <= 3u, SC_E_INVALID, "estimator %u", o.estimator);
    SC_REQUIRE(o.haze_exact <= 1u, SC_E_INVALID, "haze_exact %u", o.haze_exact);
    SC_REQUIRE(o.estimator != 2u || (width < 65536u && height < 65536u), SC_E_LIMIT,
               "beam estimator films are below 65536 pixels per side");
    (void)background;
    sc_photon_film* f = new sc_photon_film();
    f->ctx = ctx;
    f->geom = film_geom(width, height, o.bins ? o.bins : 3u);
    f->opts = o; f->cam = *cam; f->beam = *beam; f->weights = *weights;
    f->n_photons = n_photons; f->seed = seed; f->max_dist = max_dist;
    f->n_prims = n_prims; f->n_planes = n_planes; f->n_mats = n_mats;
    DeviceGuard g(ctx->device);
    auto fail = [&](cudaError_t e) {
        set_error("photon film setup failed: %s", cudaGetErrorString(e));
        cudaStream_t st = f->stream;
        delete f;  // buffers go back on the film's stream, which is destroyed after them
        if (st) { cudaStreamSynchronize(st); cudaStreamDestroy(st); }
        return e == cudaErrorMemoryAllocation ? SC_E_NOMEM : SC_E_CUDA;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e);
    // every buffer of the film from the context's pool, on the film's stream:
    // creating and destroying films allocates nothing once the pool holds enough
    f->bind_pool();
    const size_t npx = (size_t)width * height;
    if ((e = f->prims.alloc(n_prims)) != cudaSuccess) return fail(e);
    if ((e = f->planes.alloc(n_planes)) != cudaSuccess) return fail(e);
    if ((e = f->mats.alloc(n_mats)) != cudaSuccess) return fail(e);
    if ((e = f->film.alloc(f->geom.cells())) != cudaSuccess) return fail(e);
    if ((e = f->flags.alloc(flag_words(width, height))) != cudaSuccess) return fail(e);
    if ((e = f->xyz.alloc(3 * npx)) != cudaSuccess) return fail(e);
    if ((e = f->surface.alloc(3 * npx)) != cudaSuccess) return fail(e);
    if ((e = f->work.alloc(264)) != cudaSuccess) return fail(e);
    if (n_prims && (e = cudaMemcpyAsync(f->prims.p, prims, n_prims * sizeof(sc_primitive), cudaMemcpyHostToDevice, f->stream)) != cudaSuccess) return fail(e);
    if (n_planes && (e = cudaMemcpyAsync(f->planes.p, planes, n_planes * sizeof(sc_plane), cudaMemcpyHostToDevice, f->stream)) != cudaSuccess) return fail(e);
    if (n_mats && (e = cudaMemcpyAsync(f->mats.p, mats, n_mats * sizeof(sc_material), cudaMemcpyHostToDevice, f->stream)) != cudaSuccess) return fail(e);
    if (zbuffer) {
        if ((e = f->zbuf.alloc(npx)) != cudaSuccess) return fail(e);
        if ((e = cudaMemcpyAsync(f->zbuf.p, zbuffer, npx * sizeof(float), cudaMemcpyHostToDevice, f->stream)) != cudaSuccess) return fail(e);
    }
    if (o.bins) {
        std::vector<float> w(3 * o.bins);
        bin_weights(ctx->tables, o.bins, o.lambda_min, o.lambda_max, w.data());
        if ((e = f->binw.alloc(w.size())) != cudaSuccess) return fail(e);
        if ((e = cudaMemcpyAsync(f->binw.p, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, f->stream)) != cudaSuccess) return fail(e);
    }
    if ((e = cudaMemsetAsync(f->film.p, 0, f->film.bytes(), f->stream)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(f->flags.p, 0, f->flags.bytes(), f->stream)) != cudaSuccess) return fail(e);
    if ((e = cudaMemsetAsync(f->surface.p, 0, f->surface.bytes(), f->stream)) != cudaSuccess) return fail(e);
    if ((e = cudaStreamSynchronize(f->stream)) != cudaSuccess) return fail(e);
    default_shape(ctx, o.bins != 0, 0, scene_smem_bytes(n_prims, n_planes, n_mats) + mask_smem(width, height),
                  f->shape, o.estimator);
    *out = f;
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_destroy(sc_photon_film* f) {
    SC_GUARD_BEGIN
    if (!f) return SC_OK;
    {
        DeviceGuard g(f->ctx->device);
        if (f->stream) cudaStreamSynchronize(f->stream);
        f->prims.reset(); f->planes.reset(); f->mats.reset(); f->zbuf.reset(); f->film.reset(); f->flags.reset();
        f->xyz.reset(); f->surface.reset(); f->binw.reset(); f->work.reset(); f->rgb.reset(); f->debug.reset();
        // the frees are stream-ordered: let them complete, so the next film can take the memory at once
        if (f->stream) { cudaStreamSynchronize(f->stream); cudaStreamDestroy(f->stream); }
    }
    delete f;
    return SC_OK;
    SC_GUARD_END
}

#define FILM_LOCK(f)                                        \
    SC_REQUIRE((f), SC_E_INVALID, "null photon film");      \
    std::lock_guard<std::mutex> _lk((f)->mu);               \
    DeviceGuard _dg((f)->ctx->device)

int sc_photon_film_trace_and_resolve(sc_photon_film* f, uint32_t n, uint32_t seed) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    f->n_photons = n; f->seed = seed;
    int rc = f->trace(0, n, seed);
    if (rc != SC_OK) return rc;
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_trace_chunked(sc_photon_film* f, uint32_t total, uint32_t seed) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    f->n_photons = total; f->seed = seed;
    int rc = f->trace(0, total, seed);
    if (rc != SC_OK) return rc;
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_dispatch(sc_photon_film* f, uint32_t base, uint32_t n, uint32_t seed) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    f->n_photons = n; f->seed = seed;
    return f->trace(base, n, seed);
    SC_GUARD_END
}

int sc_photon_film_trace_debug(sc_photon_film* f, uint32_t n, uint32_t seed, uint32_t debug_count,
                               sc_debug_photon* out) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(out || debug_count == 0, SC_E_INVALID, "null output");
    SC_REQUIRE(f->opts.estimator != 2u, SC_E_STATE, "trace_debug records point-estimator paths only");
    const uint32_t count = std::min(debug_count, n);
    if (debug_count) std::memset(out, 0, (size_t)debug_count * sizeof(sc_debug_photon));
    if (count == 0) return SC_OK;
    if (f->debug.n < count) SC_CUDA(f->debug.alloc(count));
    SC_CUDA(cudaMemsetAsync(f->debug.p, 0, count * sizeof(sc_debug_photon), f->stream));
    PhotonParams p = f->params(0, count, seed);
    p.debug = f->debug.p;
    SC_CUDA(launch_photon_debug(p, f->stream));
    SC_CUDA(cudaMemcpyAsync(out, f->debug.p, count * sizeof(sc_debug_photon), cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_set_spectral(sc_photon_film* f, int on) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    f->spectral = on ? 1u : 0u;
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_get_spectral(sc_photon_film* f, int* on) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(on, SC_E_INVALID, "null output");
    *on = f->spectral ? 1 : 0;
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_set_camera(sc_photon_film* f, const sc_camera* cam) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(cam, SC_E_INVALID, "null camera");
    f->cam = *cam;
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_recompute_surface(sc_photon_film* f, const sc_camera* cam) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    if (cam) f->cam = *cam;
    RimParams r;
    r.cam = f->cam; r.width = f->geom.w; r.height = f->geom.h;
    r.prims = f->prims.p; r.planes = f->planes.p; r.mats = f->mats.p;
    r.n_prims = f->n_prims; r.n_planes = f->n_planes; r.n_mats = f->n_mats;
    r.out = f->surface.p;
    SC_CUDA(launch_rim(r, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_read_surface(sc_photon_film* f, float* out) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    SC_CUDA(cudaMemcpyAsync(out, f->surface.p, f->surface.bytes(), cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_read_accum(sc_photon_film* f, float* out) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    int rc = f->ensure_xyz();
    if (rc != SC_OK) return rc;
    SC_CUDA(cudaMemcpyAsync(out, f->xyz.p, f->xyz.bytes(), cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_read_raw(sc_photon_film* f, int64_t* out) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    std::vector<int64_t> tiles(f->geom.cells());
    SC_CUDA(cudaMemcpyAsync(tiles.data(), f->film.p, f->film.bytes(), cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    const FilmGeom& g = f->geom;
    for (uint32_t py = 0; py < g.h; ++py)
        for (uint32_t px = 0; px < g.w; ++px)
            std::memcpy(out + ((size_t)py * g.w + px) * g.channels, tiles.data() + film_cell(px, py, g.tiles_x, g.channels),
                        g.channels * sizeof(int64_t));
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_clear(sc_photon_film* f) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_CUDA(cudaMemsetAsync(f->film.p, 0, f->film.bytes(), f->stream));
    SC_CUDA(cudaMemsetAsync(f->flags.p, 0, f->flags.bytes(), f->stream));
    ++f->film_version;
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_auto_expose(sc_photon_film* f, float scale, float* exposure) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(exposure, SC_E_INVALID, "null output");
    int rc = f->ensure_xyz();
    if (rc != SC_OK) return rc;
    SC_CUDA(launch_composite_max_y(f->xyz.p, f->surface.p, f->geom.w * f->geom.h, f->work.p, f->stream));
    uint32_t bits = 0;
    SC_CUDA(cudaMemcpyAsync(&bits, f->work.p, 4, cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    float max_y;
    std::memcpy(&max_y, &bits, 4);
    *exposure = std::max(scale / std::max(max_y, 1e-6f), 1.0f);
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_auto_expose_p997(sc_photon_film* f, float* exposure) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(exposure, SC_E_INVALID, "null output");
    int rc = f->ensure_xyz();
    if (rc != SC_OK) return rc;
    const uint32_t n = f->geom.w * f->geom.h;
    uint32_t k = (uint32_t)((float)n * 0.997f);
    if (k > n - 1) k = n - 1;
    SC_CUDA(launch_composite_select(f->xyz.p, f->surface.p, n, k, f->work.p, f->stream));
    uint32_t bits = 0;
    SC_CUDA(cudaMemcpyAsync(&bits, f->work.p + 258, 4, cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    float p;
    std::memcpy(&p, &bits, 4);
    *exposure = 1.0f / std::max(p, 1e-9f);
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_to_rgb8(sc_photon_film* f, float exposure, uint8_t* out) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    int rc = f->ensure_xyz();
    if (rc != SC_OK) return rc;
    const size_t n = (size_t)f->geom.w * f->geom.h;
    if (f->rgb.n < 4 * n) SC_CUDA(f->rgb.alloc(4 * n));
    SC_CUDA(launch_to_rgb8(f->xyz.p, f->surface.p, (uint32_t)n, exposure, f->rgb.p, f->stream));
    SC_CUDA(cudaMemcpyAsync(out, f->rgb.p, 3 * n, cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_gather_rgba8(sc_photon_film* f, uint64_t total_photons, float target_n, float kradius,
                                float exposure, uint8_t* out) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    SC_REQUIRE(kradius >= 0.0f && kradius <= 16.0f, SC_E_INVALID, "kradius %g outside [0, 16]", kradius);
    int rc = f->ensure_xyz();
    if (rc != SC_OK) return rc;
    const size_t n = (size_t)f->geom.w * f->geom.h;
    if (f->rgb.n < 4 * n) SC_CUDA(f->rgb.alloc(4 * n));
    const float inv_n = 1.0f / std::max((float)total_photons, 1.0f);
    SC_CUDA(launch_gather_rgba8(f->xyz.p, f->surface.p, f->geom.w, f->geom.h, inv_n * target_n, kradius, exposure,
                                f->rgb.p, f->stream));
    SC_CUDA(cudaMemcpyAsync(out, f->rgb.p, 4 * n, cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_dims(sc_photon_film* f, uint32_t* w, uint32_t* h, uint32_t* c) {
    SC_GUARD_BEGIN
    SC_REQUIRE(f, SC_E_INVALID, "null photon film");
    if (w) *w = f->geom.w;
    if (h) *h = f->geom.h;
    if (c) *c = f->geom.channels;
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_set_scene(sc_photon_film* f, const sc_primitive* prims, uint32_t n_prims,
                             const sc_plane* planes, uint32_t n_planes, const sc_material* mats, uint32_t n_mats,
                             const sc_camera* cam, const sc_beam* beam) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(cam && beam, SC_E_INVALID, "null camera or beam");
    int rc = check_scene(n_prims, n_planes, n_mats, prims, planes, mats);
    if (rc != SC_OK) return rc;
    if (f->prims.n < n_prims) SC_CUDA(f->prims.alloc(n_prims));
    if (f->planes.n < n_planes) SC_CUDA(f->planes.alloc(n_planes));
    if (f->mats.n < n_mats) SC_CUDA(f->mats.alloc(n_mats));
    if (n_prims) SC_CUDA(cudaMemcpyAsync(f->prims.p, prims, n_prims * sizeof(sc_primitive), cudaMemcpyHostToDevice, f->stream));
    if (n_planes) SC_CUDA(cudaMemcpyAsync(f->planes.p, planes, n_planes * sizeof(sc_plane), cudaMemcpyHostToDevice, f->stream));
    if (n_mats) SC_CUDA(cudaMemcpyAsync(f->mats.p, mats, n_mats * sizeof(sc_material), cudaMemcpyHostToDevice, f->stream));
    f->n_prims = n_prims; f->n_planes = n_planes; f->n_mats = n_mats;
    f->cam = *cam; f->beam = *beam;
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_device_buffers(sc_photon_film* f, void** film_dev, size_t* film_bytes, void** flags_dev,
                                  size_t* flag_bytes, void** stream) {
    SC_GUARD_BEGIN
    SC_REQUIRE(f, SC_E_INVALID, "null photon film");
    if (film_dev) *film_dev = f->film.p;
    if (film_bytes) *film_bytes = f->film.bytes();
    if (flags_dev) *flags_dev = f->flags.p;
    if (flag_bytes) *flag_bytes = f->flags.bytes();
    if (stream) *stream = f->stream;
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_mark_all_dirty(sc_photon_film* f) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_CUDA(cudaMemsetAsync(f->flags.p, 0xFF, f->flags.bytes(), f->stream));
    ++f->film_version;
    return SC_OK;
    SC_GUARD_END
}

int sc_photon_film_trace_stats(sc_photon_film* f, uint32_t base, uint32_t count, uint32_t seed, uint64_t out[4]) {
    SC_GUARD_BEGIN
    FILM_LOCK(f);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    SC_REQUIRE(f->opts.estimator != 2u, SC_E_STATE, "trace_stats counts point-estimator work only");
    DevBuf<unsigned long long> d;
    SC_CUDA(d.alloc(4));
    SC_CUDA(cudaMemsetAsync(d.p, 0, 32, f->stream));
    PhotonParams p = f->params(base, count, seed);
    SC_CUDA(launch_photon_count(p, d.p, (uint32_t)f->ctx->sms * 8u, f->stream));
    SC_CUDA(cudaMemcpyAsync(out, d.p, 32, cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}

// ---------------------------- device-pointer API ---------------------------
size_t sc_film_bytes(uint32_t w, uint32_t h, uint32_t channels) { return film_geom(w, h, channels).cells() * 8u; }
size_t sc_film_flag_bytes(uint32_t w, uint32_t h) { return (size_t)flag_words(w, h) * 4u; }

int sc_trace_photons_device(sc_ctx* ctx, const sc_trace_desc* d, uint32_t base, uint32_t count, void* film_dev,
                            uint32_t* flags_dev, void* stream) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && d && film_dev, SC_E_INVALID, "null argument");
    SC_REQUIRE(d->n_prims <= SC_MAX_PRIMS && d->n_planes <= SC_MAX_PLANES && d->n_mats <= SC_MAX_PRIMS, SC_E_LIMIT,
               "scene exceeds limits");
    SC_REQUIRE(d->width > 0 && d->height > 0, SC_E_INVALID, "empty film");
    SC_REQUIRE((uint64_t)d->width * d->height <= (1ull << 28), SC_E_LIMIT, "film %ux%u too large", d->width,
               d->height);
    sc_film_options o;
    resolve_options(&d->opts, o);
    SC_REQUIRE(o.bins <= SC_MAX_BINS && o.lambda_max > o.lambda_min && o.estimator <= 3u && o.haze_exact <= 1u,
               SC_E_INVALID, "bad film options");
    SC_REQUIRE(o.estimator != 2u || (d->width < 65536u && d->height < 65536u), SC_E_LIMIT,
               "beam estimator films are below 65536 pixels per side");
    DeviceGuard g(ctx->device);
    sc_photon_film tmp;  // parameter builder only; owns no device memory
    tmp.ctx = ctx; tmp.geom = film_geom(d->width, d->height, o.bins ? o.bins : 3u); tmp.opts = o;
    tmp.cam = d->cam; tmp.beam = d->beam; tmp.weights = d->weights; tmp.max_dist = d->max_dist;
    tmp.spectral = d->spectral;
    tmp.n_prims = d->n_prims; tmp.n_planes = d->n_planes; tmp.n_mats = d->n_mats;
    PhotonParams p = tmp.params(base, count, d->seed);
    p.prims = d->prims; p.planes = d->planes; p.mats = d->mats; p.zbuf = d->zbuffer;
    p.film = static_cast<unsigned long long*>(film_dev); p.flags = flags_dev;
    LaunchShape shape;
    default_shape(ctx, o.bins != 0, 0,
                  scene_smem_bytes(d->n_prims, d->n_planes, d->n_mats) + (flags_dev ? mask_smem(d->width, d->height) : 0),
                  shape, o.estimator);
    if (o.estimator == 2u) SC_CUDA(launch_beam(p, shape, static_cast<cudaStream_t>(stream)));
    else SC_CUDA(launch_photons(p, shape, static_cast<cudaStream_t>(stream)));
    return SC_OK;
    SC_GUARD_END
}

int sc_trace_stats_device(sc_ctx* ctx, const sc_trace_desc* d, uint32_t base, uint32_t count, uint64_t* out_dev,
                          void* stream) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && d && out_dev, SC_E_INVALID, "null argument");
    SC_REQUIRE(d->n_prims <= SC_MAX_PRIMS && d->n_planes <= SC_MAX_PLANES && d->n_mats <= SC_MAX_PRIMS, SC_E_LIMIT,
               "scene exceeds limits");
    SC_REQUIRE((uint64_t)d->width * d->height <= (1ull << 28), SC_E_LIMIT, "film %ux%u too large", d->width,
               d->height);
    sc_film_options o;
    resolve_options(&d->opts, o);
    SC_REQUIRE(o.estimator != 2u || (d->width < 65536u && d->height < 65536u), SC_E_LIMIT,
               "beam estimator films are below 65536 pixels per side");
    DeviceGuard g(ctx->device);
    sc_photon_film tmp;
    tmp.ctx = ctx; tmp.geom = film_geom(d->width, d->height, o.bins ? o.bins : 3u); tmp.opts = o;
    tmp.cam = d->cam; tmp.beam = d->beam; tmp.weights = d->weights; tmp.max_dist = d->max_dist;
    tmp.spectral = d->spectral;
    tmp.n_prims = d->n_prims; tmp.n_planes = d->n_planes; tmp.n_mats = d->n_mats;
    PhotonParams p = tmp.params(base, count, d->seed);
    p.prims = d->prims; p.planes = d->planes; p.mats = d->mats; p.zbuf = d->zbuffer;
    if (o.estimator == 2u)
        SC_CUDA(launch_beam_count(p, reinterpret_cast<unsigned long long*>(out_dev), (uint32_t)ctx->sms * 4u,
                                  static_cast<cudaStream_t>(stream)));
    else
        SC_CUDA(launch_photon_count(p, reinterpret_cast<unsigned long long*>(out_dev), (uint32_t)ctx->sms * 8u,
                                    static_cast<cudaStream_t>(stream)));
    return SC_OK;
    SC_GUARD_END
}

int sc_sensor_reduce_device(sc_ctx* ctx, uint32_t w, uint32_t h, uint32_t channels, float lambda_min,
                            float lambda_max, uint32_t scale_log2, void* film_dev, uint32_t* flags_dev, float* xyz_dev,
                            int drain, void* stream) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && film_dev && xyz_dev, SC_E_INVALID, "null argument");
    SC_REQUIRE(channels == 3u || (channels >= 1u && channels <= SC_MAX_BINS), SC_E_INVALID, "channels %u", channels);
    SC_REQUIRE(w > 0 && h > 0, SC_E_INVALID, "empty film");
    DeviceGuard g(ctx->device);
    const FilmGeom fg = film_geom(w, h, channels);
    // Bin weights are cached per (bins, band) on the context.
    const float* binw = nullptr;
    if (channels != 3u) {
        if (lambda_min == 0.0f) lambda_min = 380.0f;
        if (lambda_max == 0.0f) lambda_max = 730.0f;
        std::lock_guard<std::mutex> lk(ctx->mu);
        const auto key = std::make_tuple(channels, lambda_min, lambda_max);
        auto it = ctx->binw_cache.find(key);
        if (it == ctx->binw_cache.end()) {
            std::vector<float> wv(3 * channels);
            bin_weights(ctx->tables, channels, lambda_min, lambda_max, wv.data());
            std::unique_ptr<DevBuf<float>> buf(new DevBuf<float>());
            SC_CUDA(buf->alloc(wv.size()));
            SC_CUDA(cudaMemcpy(buf->p, wv.data(), wv.size() * sizeof(float), cudaMemcpyHostToDevice));
            it = ctx->binw_cache.emplace(key, std::move(buf)).first;
        }
        binw = it->second->p;
    }
    ReduceParams r;
    r.film = static_cast<unsigned long long*>(film_dev); r.flags = flags_dev; r.xyz = xyz_dev;
    r.width = w; r.height = h; r.tiles_x = fg.tiles_x; r.tiles_y = fg.tiles_y; r.channels = channels; r.binw = binw;
    r.inv_scale = std::ldexp(1.0, -(int)(scale_log2 ? scale_log2 : 32u));
    SC_CUDA(launch_reduce(r, drain != 0, static_cast<cudaStream_t>(stream)));
    return SC_OK;
    SC_GUARD_END
}

}  // extern "C"

// --------------------------------------------------------------------------
// atomic film (spectral-gpu/src/film.rs:40-305)
// --------------------------------------------------------------------------
struct sc_atomic_film {
    sc_ctx* ctx = nullptr;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    uint32_t w = 0, h = 0;
    DevBuf<uint32_t> film;
    DevBuf<float> accum;
    DevBuf<uint32_t> work;  // max-Y bits of auto_expose_accum
    DevBuf<uint8_t> rgb;    // to_rgb8 staging
};

extern "C" {

int sc_atomic_film_create(sc_ctx* ctx, uint32_t w, uint32_t h, sc_atomic_film** out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && out, SC_E_INVALID, "null argument");
    SC_REQUIRE(w > 0 && h > 0 && (uint64_t)w * h <= (1ull << 28), SC_E_INVALID, "film %ux%u", w, h);
    *out = nullptr;
    sc_atomic_film* f = new sc_atomic_film();
    f->ctx = ctx; f->w = w; f->h = h;
    DeviceGuard g(ctx->device);
    cudaError_t e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = f->film.alloc(3ull * w * h);
    if (e == cudaSuccess) e = f->accum.alloc(3ull * w * h);
    if (e == cudaSuccess) e = cudaMemsetAsync(f->film.p, 0, f->film.bytes(), f->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(f->accum.p, 0, f->accum.bytes(), f->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
    if (e != cudaSuccess) {
        set_error("atomic film setup failed: %s", cudaGetErrorString(e));
        if (f->stream) cudaStreamDestroy(f->stream);
        delete f;
        return e == cudaErrorMemoryAllocation ? SC_E_NOMEM : SC_E_CUDA;
    }
    *out = f;
    return SC_OK;
    SC_GUARD_END
}

int sc_atomic_film_destroy(sc_atomic_film* f) {
    SC_GUARD_BEGIN
    if (!f) return SC_OK;
    {
        DeviceGuard g(f->ctx->device);
        if (f->stream) cudaStreamSynchronize(f->stream);
        f->film.reset(); f->accum.reset();
        if (f->stream) cudaStreamDestroy(f->stream);
    }
    delete f;
    return SC_OK;
    SC_GUARD_END
}

#define AFILM_LOCK(f)                                       \
    SC_REQUIRE((f), SC_E_INVALID, "null atomic film");      \
    std::lock_guard<std::mutex> _lk((f)->mu);               \
    DeviceGuard _dg((f)->ctx->device)

int sc_atomic_film_splat(sc_atomic_film* f, uint32_t seed, uint32_t n) {
    SC_GUARD_BEGIN
    AFILM_LOCK(f);
    SC_CUDA(launch_synthetic_splat(f->film.p, f->w, f->h, seed, n, f->stream));
    return SC_OK;
    SC_GUARD_END
}
int sc_atomic_film_stream(sc_atomic_film* f, void** stream) {
    SC_GUARD_BEGIN
    SC_REQUIRE(f && stream, SC_E_INVALID, "null argument");
    *stream = f->stream;
    return SC_OK;
    SC_GUARD_END
}
int sc_atomic_film_read_raw(sc_atomic_film* f, uint32_t* out) {
    SC_GUARD_BEGIN
    AFILM_LOCK(f);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    SC_CUDA(cudaMemcpyAsync(out, f->film.p, f->film.bytes(), cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}
int sc_atomic_film_resolve(sc_atomic_film* f) {
    SC_GUARD_BEGIN
    AFILM_LOCK(f);
    SC_CUDA(launch_atomic_resolve(f->film.p, f->accum.p, f->film.n, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}
int sc_atomic_film_read_accum(sc_atomic_film* f, float* out) {
    SC_GUARD_BEGIN
    AFILM_LOCK(f);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    SC_CUDA(cudaMemcpyAsync(out, f->accum.p, f->accum.bytes(), cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}
int sc_atomic_film_auto_expose_accum(sc_atomic_film* f, float scale, float* exposure) {
    SC_GUARD_BEGIN
    AFILM_LOCK(f);
    SC_REQUIRE(exposure, SC_E_INVALID, "null output");
    if (!f->work.p) SC_CUDA(f->work.alloc(1));
    SC_CUDA(launch_composite_max_y(f->accum.p, nullptr, f->w * f->h, f->work.p, f->stream));
    uint32_t bits = 0;
    SC_CUDA(cudaMemcpyAsync(&bits, f->work.p, 4, cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    float max_y;
    std::memcpy(&max_y, &bits, 4);
    *exposure = std::max(scale / std::max(max_y, 1e-6f), 1.0f);
    return SC_OK;
    SC_GUARD_END
}
int sc_atomic_film_to_rgb8(sc_atomic_film* f, float exposure, uint8_t* out) {
    SC_GUARD_BEGIN
    AFILM_LOCK(f);
    SC_REQUIRE(out, SC_E_INVALID, "null output");
    const size_t n = (size_t)f->w * f->h;
    if (f->rgb.n < 3 * n) SC_CUDA(f->rgb.alloc(3 * n));
    SC_CUDA(launch_to_rgb8(f->accum.p, nullptr, (uint32_t)n, exposure, f->rgb.p, f->stream));
    SC_CUDA(cudaMemcpyAsync(out, f->rgb.p, 3 * n, cudaMemcpyDeviceToHost, f->stream));
    SC_CUDA(cudaStreamSynchronize(f->stream));
    return SC_OK;
    SC_GUARD_END
}
int sc_atomic_film_clear_film(sc_atomic_film* f) {
    SC_GUARD_BEGIN
    AFILM_LOCK(f);
    SC_CUDA(cudaMemsetAsync(f->film.p, 0, f->film.bytes(), f->stream));
    return SC_OK;
    SC_GUARD_END
}
int sc_atomic_film_clear_accum(sc_atomic_film* f) {
    SC_GUARD_BEGIN
    AFILM_LOCK(f);
    SC_CUDA(cudaMemsetAsync(f->accum.p, 0, f->accum.bytes(), f->stream));
    return SC_OK;
    SC_GUARD_END
}
int sc_atomic_film_check_determinism(sc_ctx* ctx, uint32_t w, uint32_t h, uint32_t seed, uint32_t n,
                                     int64_t* first_diff) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && first_diff, SC_E_INVALID, "null argument");
    sc_atomic_film *a = nullptr, *b = nullptr;
    int rc = sc_atomic_film_create(ctx, w, h, &a);
    if (rc != SC_OK) return rc;
    rc = sc_atomic_film_create(ctx, w, h, &b);
    if (rc != SC_OK) { sc_atomic_film_destroy(a); return rc; }
    std::vector<uint32_t> ra(3ull * w * h), rb(3ull * w * h);
    if ((rc = sc_atomic_film_splat(a, seed, n)) == SC_OK && (rc = sc_atomic_film_read_raw(a, ra.data())) == SC_OK &&
        (rc = sc_atomic_film_splat(b, seed, n)) == SC_OK && (rc = sc_atomic_film_read_raw(b, rb.data())) == SC_OK) {
        *first_diff = -1;
        for (size_t i = 0; i < ra.size(); ++i)
            if (ra[i] != rb[i]) { *first_diff = (int64_t)i; break; }
    }
    sc_atomic_film_destroy(a);
    sc_atomic_film_destroy(b);
    return rc;
    SC_GUARD_END
}

}  // extern "C"
