// Allocation-free render of one photon range straight to an XYZ image.
//
// For callers that cannot allocate device memory: hosts whose framework owns
// all device memory through its own pool (a raw cudaMalloc would bypass the
// pool, and cudaFree synchronises the whole device) and render loops that must
// never block on an allocation.  The caller passes the inputs (scene records
// in device memory, camera, beam, weights, film options) and the output image;
// the scratch this path needs -- the 64-bit film, its dirty-tile mask, the
// colour-matching table and the bin weights -- lives in the file-scope device
// arrays below, which every GPU that loads the library holds until the process
// exits.  The table and the bin weights reach the device as the by-value
// parameter of a small staging kernel, so no copy reads host memory after the
// call has returned.
//
// Host code must not use the arrays' names as device addresses: on the host
// they are stand-ins.  The addresses are looked up with cudaGetSymbolAddress
// once per device, with that device current, the first time the entry point
// runs on that device.
#include <mutex>

#include "host_util.h"
#include "internal.h"

namespace {

static __device__ __align__(256) unsigned long long g_noalloc_film[SC_NOALLOC_MAX_FILM_CELLS];
static __device__ __align__(256) uint32_t g_noalloc_mask[SC_NOALLOC_MAX_MASK_WORDS];
static __device__ __align__(256) float g_noalloc_tables[3 * sc::kTableN];  // xbar, ybar, zbar
static __device__ __align__(256) float g_noalloc_binw[3 * SC_MAX_BINS];

struct ScratchPtrs {
    unsigned long long* film = nullptr;
    uint32_t* mask = nullptr;
    float* tables = nullptr;
    float* binw = nullptr;
    int sms = 0;
    bool ready = false;
};

// What a call needs from the host, carried by the staging launch itself
// (3928 bytes of kernel parameter).  Device code names the arrays directly.
struct NoallocStage {
    float cmf[3 * sc::kTableN];
    float binw[3 * SC_MAX_BINS];
    uint32_t bins;
};

__global__ void noalloc_stage_kernel(const NoallocStage st) {
    for (uint32_t i = threadIdx.x; i < 3u * sc::kTableN; i += blockDim.x) g_noalloc_tables[i] = st.cmf[i];
    for (uint32_t i = threadIdx.x; i < 3u * st.bins; i += blockDim.x) g_noalloc_binw[i] = st.binw[i];
}

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
ScratchPtrs g_scratch[kMaxDevices];

// Once per device, with the device current: device addresses of the arrays.
int scratch_for_current_device(ScratchPtrs& out) {
    int dev = 0;
    SC_CUDA(cudaGetDevice(&dev));
    SC_REQUIRE(dev >= 0 && dev < kMaxDevices, SC_E_LIMIT, "device %d beyond %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lk(g_setup_mu);
    ScratchPtrs& s = g_scratch[dev];
    if (!s.ready) {
        ScratchPtrs t;
        SC_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&t.film), g_noalloc_film));
        SC_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&t.mask), g_noalloc_mask));
        SC_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&t.tables), g_noalloc_tables));
        SC_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&t.binw), g_noalloc_binw));
        SC_CUDA(cudaDeviceGetAttribute(&t.sms, cudaDevAttrMultiProcessorCount, dev));
        t.ready = true;
        s = t;
    }
    out = s;
    return SC_OK;
}

}  // namespace

extern "C" int sc_trace_xyz_noalloc(const float* tables_5x71, const sc_trace_desc* d, uint32_t photon_base,
                                    uint32_t count, float* xyz_dev, void* stream) {
    SC_GUARD_BEGIN
    using namespace sc;
    SC_REQUIRE(tables_5x71 && d && xyz_dev, SC_E_INVALID, "null argument");
    SC_REQUIRE(d->n_prims <= SC_MAX_PRIMS && d->n_planes <= SC_MAX_PLANES && d->n_mats <= SC_MAX_PRIMS, SC_E_LIMIT,
               "scene exceeds %d primitives / %d planes", SC_MAX_PRIMS, SC_MAX_PLANES);
    SC_REQUIRE((d->n_prims == 0 || d->prims) && (d->n_planes == 0 || d->planes) && (d->n_mats == 0 || d->mats),
               SC_E_INVALID, "null scene array");
    SC_REQUIRE(d->width > 0 && d->height > 0, SC_E_INVALID, "empty film");
    sc_film_options o = d->opts;
    if (o.lambda_min == 0.0f) o.lambda_min = 380.0f;
    if (o.lambda_max == 0.0f) o.lambda_max = 730.0f;
    if (o.max_bounces == 0u) o.max_bounces = 8u;
    if (o.scale_log2 == 0u) o.scale_log2 = 32u;
    SC_REQUIRE(o.bins <= SC_MAX_BINS && o.lambda_max > o.lambda_min && o.scale_log2 <= 50u && o.max_bounces <= 64u &&
                   o.haze_exact <= 1u,
               SC_E_INVALID, "bad film options");
    SC_REQUIRE(o.estimator <= 1u || o.estimator == 3u, SC_E_INVALID,
               "estimator %u: the allocation-free path takes the point (0), isotropic (1) and free-flight (3) "
               "estimators", o.estimator);
    const uint32_t channels = o.bins ? o.bins : 3u;
    const uint32_t tiles_x = (d->width + 7u) / 8u, tiles_y = (d->height + 7u) / 8u;
    const uint64_t cells = (uint64_t)tiles_x * tiles_y * kTilePixels * channels;
    const uint32_t words = flag_words(d->width, d->height);
    SC_REQUIRE(cells <= SC_NOALLOC_MAX_FILM_CELLS, SC_E_LIMIT,
               "film %ux%u with %u channels needs %llu cells; the allocation-free path holds at most %u "
               "(8x8-tile padded width * height * channels)",
               d->width, d->height, channels, (unsigned long long)cells, (unsigned)SC_NOALLOC_MAX_FILM_CELLS);
    SC_REQUIRE(words <= SC_NOALLOC_MAX_MASK_WORDS, SC_E_LIMIT, "film has too many tiles for the scratch mask");
    ScratchPtrs sp;
    int rc = scratch_for_current_device(sp);
    if (rc != SC_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // Calls share the scratch arrays: everything read before it is written is
    // reset here, on the caller's stream.  Calls that overlap on the GPU race.
    NoallocStage st;
    std::memcpy(st.cmf, tables_5x71, sizeof st.cmf);  // rows 0..2 of the sensor table
    st.bins = o.bins;
    if (o.bins) bin_weights(tables_5x71, o.bins, o.lambda_min, o.lambda_max, st.binw);
    noalloc_stage_kernel<<<1, 256, 0, s>>>(st);
    SC_CUDA(cudaGetLastError());
    SC_CUDA(cudaMemsetAsync(sp.film, 0, cells * sizeof(unsigned long long), s));
    SC_CUDA(cudaMemsetAsync(sp.mask, 0, words * sizeof(uint32_t), s));

    PhotonParams p;
    std::memset(&p, 0, sizeof p);
    p.corner = ld3(d->beam.corner); p.bu = ld3(d->beam.u); p.bv = ld3(d->beam.v); p.bdir = ld3(d->beam.dir);
    p.proj = make_proj(d->cam);
    p.width = d->width; p.height = d->height; p.tiles_x = tiles_x; p.channels = channels;
    p.photon_base = photon_base; p.photon_count = count; p.seed = d->seed; p.max_bounces = o.max_bounces;
    p.sigma_s = d->weights.sigma_s; p.sigma_t = d->weights.sigma_t; p.g = d->weights.g; p.max_dist = d->max_dist;
    p.lambda_min = o.lambda_min; p.lambda_range = o.lambda_max - o.lambda_min;
    p.bins = o.bins; p.bin_min = o.lambda_min; p.bin_inv_width = o.bins ? (float)o.bins / p.lambda_range : 0.0f;
    p.scale = std::ldexp(1.0f, (int)o.scale_log2);
    p.spectral = d->spectral; p.estimator = o.estimator; p.haze_exact = o.haze_exact;
    p.zbuf = d->zbuffer; p.film = sp.film; p.flags = sp.mask;
    p.prims = d->prims; p.planes = d->planes; p.mats = d->mats;
    p.n_prims = d->n_prims; p.n_planes = d->n_planes; p.n_mats = d->n_mats;
    p.cmf = sp.tables;  // xbar, ybar, zbar

    LaunchShape shape;
    shape.block = 256; shape.aggregate = 0; shape.minb = 4;
    shape.order = 0;  // the ordered dispatch takes stream-ordered scratch memory
    const size_t smem = scene_smem_bytes(d->n_prims, d->n_planes, d->n_mats) +
                        (words <= kMaxSmemMaskWords ? words * sizeof(uint32_t) : 0);
    shape.grid = (uint32_t)(sp.sms * photon_occupancy_blocks(shape, o.bins != 0, smem));
    SC_CUDA(launch_photons(p, shape, s));

    ReduceParams r;
    r.film = sp.film; r.flags = sp.mask; r.xyz = xyz_dev; r.width = d->width; r.height = d->height;
    r.tiles_x = tiles_x; r.tiles_y = tiles_y; r.channels = channels; r.binw = o.bins ? sp.binw : nullptr;
    r.inv_scale = std::ldexp(1.0, -(int)o.scale_log2);
    SC_CUDA(launch_reduce(r, false, s));
    return SC_OK;
    SC_GUARD_END
}
