// One scene split over GPUs: each GPU traces its range of photons into its own
// int64 film, then reduces its own band of image rows straight from every
// GPU's film (peer memory over NVLink, mapped with CUDA IPC), so no film is
// ever summed into one and no film crosses the links whole: each GPU reads
// 1/N of every film.  The bands are then gathered (XYZ rows, a few MB).  The
// sum of int64 cells is exact, so every band is bit-identical to the same rows
// of the one-GPU image.  No counterpart in the reference (single GPU).
#include <cuda.h>

#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "host_util.h"
#include "internal.h"

using namespace sc;

namespace {

// cuMemGetAddressRange through the runtime's driver entry point (no link
// against the driver library): the allocation that holds a device pointer.
using GetRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);

GetRangeFn get_range() {
    static GetRangeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<GetRangeFn>(p);
    });
    return fn;
}

// Bin-averaged CMF of (bins, band) on the device, cached on the context.
int binw_cached(sc_ctx* ctx, uint32_t channels, float lambda_min, float lambda_max, const float** out) {
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
    *out = it->second->p;
    return SC_OK;
}

}  // namespace

extern "C" {

int sc_ipc_export(sc_ctx* ctx, const void* dev_ptr, unsigned char handle[64], size_t* offset) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && dev_ptr && handle && offset, SC_E_INVALID, "null argument");
    DeviceGuard g(ctx->device);
    const GetRangeFn range = get_range();
    SC_REQUIRE(range, SC_E_CUDA, "cuMemGetAddressRange is not available");
    CUdeviceptr base = 0;
    size_t size = 0;
    SC_REQUIRE(range(&base, &size, reinterpret_cast<CUdeviceptr>(dev_ptr)) == CUDA_SUCCESS, SC_E_INVALID,
               "%p is not device memory of this context", dev_ptr);
    cudaIpcMemHandle_t h;
    SC_CUDA(cudaIpcGetMemHandle(&h, reinterpret_cast<void*>(base)));
    static_assert(sizeof h == 64, "IPC handle size");
    std::memcpy(handle, &h, sizeof h);
    *offset = (size_t)(reinterpret_cast<CUdeviceptr>(dev_ptr) - base);
    return SC_OK;
    SC_GUARD_END
}

int sc_ipc_import(sc_ctx* ctx, const unsigned char handle[64], size_t offset, void** dev_ptr) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && handle && dev_ptr, SC_E_INVALID, "null argument");
    DeviceGuard g(ctx->device);
    cudaIpcMemHandle_t h;
    std::memcpy(&h, handle, sizeof h);
    void* base = nullptr;
    SC_CUDA(cudaIpcOpenMemHandle(&base, h, cudaIpcMemLazyEnablePeerAccess));
    *dev_ptr = static_cast<unsigned char*>(base) + offset;
    return SC_OK;
    SC_GUARD_END
}

int sc_ipc_close(sc_ctx* ctx, void* dev_ptr, size_t offset) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && dev_ptr, SC_E_INVALID, "null argument");
    DeviceGuard g(ctx->device);
    SC_CUDA(cudaIpcCloseMemHandle(static_cast<unsigned char*>(dev_ptr) - offset));
    return SC_OK;
    SC_GUARD_END
}

int sc_sensor_reduce_peers(sc_ctx* ctx, uint32_t w, uint32_t h, uint32_t channels, float lambda_min,
                           float lambda_max, uint32_t scale_log2, const int64_t* const* films_dev, uint32_t n_films,
                           uint32_t row_begin, uint32_t row_end, float* xyz_dev, void* stream) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && films_dev && xyz_dev, SC_E_INVALID, "null argument");
    SC_REQUIRE(n_films >= 1 && n_films <= kMaxPeerFilms, SC_E_LIMIT, "%u films (1 to %u)", n_films, kMaxPeerFilms);
    SC_REQUIRE(channels == 3u || (channels >= 1u && channels <= SC_MAX_BINS), SC_E_INVALID, "channels %u", channels);
    SC_REQUIRE(w > 0 && h > 0 && (uint64_t)w * h <= (1ull << 28), SC_E_INVALID, "film %ux%u", w, h);
    SC_REQUIRE(row_begin <= row_end && row_end <= h && row_begin % 8u == 0u && (row_end % 8u == 0u || row_end == h),
               SC_E_INVALID, "rows [%u, %u) must start and end on 8-row tile boundaries of a %u-row film", row_begin,
               row_end, h);
    PeerFilms pf;
    std::memset(&pf, 0, sizeof pf);
    for (uint32_t f = 0; f < n_films; ++f) {
        SC_REQUIRE(films_dev[f] && (reinterpret_cast<uintptr_t>(films_dev[f]) & 15u) == 0u, SC_E_INVALID,
                   "film %u is null or not 16-byte aligned", f);
        pf.film[f] = reinterpret_cast<const unsigned long long*>(films_dev[f]);
    }
    pf.n = n_films;
    DeviceGuard g(ctx->device);
    const uint32_t tiles_x = (w + 7u) / 8u, tiles_y = (h + 7u) / 8u;
    const float* binw = nullptr;
    if (channels != 3u) {
        if (lambda_min == 0.0f) lambda_min = 380.0f;
        if (lambda_max == 0.0f) lambda_max = 730.0f;
        const int rc = binw_cached(ctx, channels, lambda_min, lambda_max, &binw);
        if (rc != SC_OK) return rc;
    }
    ReduceParams r;
    r.film = nullptr; r.flags = nullptr; r.xyz = xyz_dev;
    r.width = w; r.height = h; r.tiles_x = tiles_x; r.tiles_y = tiles_y; r.channels = channels; r.binw = binw;
    r.inv_scale = std::ldexp(1.0, -(int)(scale_log2 ? scale_log2 : 32u));
    const uint32_t t0 = (row_begin / 8u) * tiles_x, t1 = ((row_end + 7u) / 8u) * tiles_x;
    SC_CUDA(launch_reduce_peers(r, pf, t0, t1, static_cast<cudaStream_t>(stream)));
    return SC_OK;
    SC_GUARD_END
}

}  // extern "C"
