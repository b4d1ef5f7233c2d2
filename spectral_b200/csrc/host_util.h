// Host-side plumbing shared by the ABI objects: thread-local error text,
// CUDA error propagation, device guards and owned device buffers.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <tuple>

#include <cuda_runtime.h>

#include "../../include/spectral_cuda.h"

namespace sc {

void set_error(const char* fmt, ...);

#define SC_CUDA(expr)                                                                   \
    do {                                                                                \
        cudaError_t _e = (expr);                                                        \
        if (_e != cudaSuccess) {                                                        \
            ::sc::set_error("%s failed: %s", #expr, cudaGetErrorString(_e));            \
            return _e == cudaErrorMemoryAllocation ? SC_E_NOMEM : SC_E_CUDA;            \
        }                                                                               \
    } while (0)

#define SC_REQUIRE(cond, code, ...)       \
    do {                                  \
        if (!(cond)) {                    \
            ::sc::set_error(__VA_ARGS__); \
            return (code);                \
        }                                 \
    } while (0)

// Every ABI entry runs its body inside this guard so no exception escapes.
#define SC_GUARD_BEGIN try {
#define SC_GUARD_END                                                  \
    }                                                                 \
    catch (const std::bad_alloc&) {                                   \
        ::sc::set_error("host allocation failed");                    \
        return SC_E_NOMEM;                                            \
    }                                                                 \
    catch (const std::exception& ex) {                                \
        ::sc::set_error("internal error: %s", ex.what());             \
        return SC_E_INVALID;                                          \
    }                                                                 \
    catch (...) {                                                     \
        ::sc::set_error("internal error");                            \
        return SC_E_INVALID;                                          \
    }

struct DeviceGuard {
    int prev = 0;
    explicit DeviceGuard(int dev) { cudaGetDevice(&prev); if (prev != dev) cudaSetDevice(dev); }
    ~DeviceGuard() { int cur = 0; cudaGetDevice(&cur); if (cur != prev) cudaSetDevice(prev); }
};

// Device buffer.  Unbound, it holds cudaMalloc memory.  Bound to a memory pool
// and a stream (bind), it takes stream-ordered memory from the pool on that
// stream and gives it back there: a pool that keeps its memory reserved turns
// repeated create / destroy of same-sized objects into no allocation at all.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { reset(); }
    void bind(cudaMemPool_t mp, cudaStream_t s) { pool = mp; stream = s; }
    cudaError_t alloc(size_t count) {
        reset();
        if (count == 0) return cudaSuccess;
        cudaError_t e = pool ? cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), count * sizeof(T), pool, stream)
                             : cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
        if (e != cudaSuccess) { p = nullptr; return e; }
        n = count;
        return cudaSuccess;
    }
    void reset() {
        if (p) {
            if (pool) cudaFreeAsync(p, stream);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

}  // namespace sc

struct sc_ctx {
    int device = 0;
    int sms = 0;
    int cc_major = 0, cc_minor = 0;
    float tables[5 * 71];
    sc::DevBuf<float> cmf;  // 3 x 71 on the device
    // stream-ordered scratch (the wavelength-ordered photon dispatch); memory
    // freed to it stays reserved for the next launch until the context goes
    cudaMemPool_t pool = nullptr;
    std::mutex mu;
    // bin-averaged CMF weights of spectral films reduced through the
    // device-pointer API, per (bins, band); freed with the context
    std::map<std::tuple<uint32_t, float, float>, std::unique_ptr<sc::DevBuf<float>>> binw_cache;
};
