// Forward photon emitter / tracer with point-estimator haze splatting.
//
// One thread per photon, restating render_volumetric_scene_point
// (spectral-core/src/volume.rs:99-168) and its GPU mirror
// (spectral-gpu/src/shaders/volume.wgsl:542-647): emission from the beam
// aperture, hero wavelength, up to max_bounces segments, 4 uniform haze samples
// per segment connected to the camera (HG phase x transmittance / d^2), then the
// Fresnel / refract / TIR scatter at the hit.  The RNG stream is consumed in
// exactly the reference order, so paths are bit-identical to the CPU crate.
//
// Splats land in a 64-bit fixed-point film with red.global.add.u64; the film is
// tile-major (8x8 pixel tiles) and every touched tile raises a dirty flag so the
// drain/reduce pass reads only tiles that received light.
#include <map>
#include <mutex>
#include <tuple>

#include "photon_trace.cuh"

namespace sc {

namespace {

// Byte offset of the warp-split buffers: after scene records, CMF table and the
// dirty mask, rounded up to 16 bytes.
__host__ __device__ __forceinline__ size_t split_offset(const PhotonParams& p, uint32_t mask_words) {
    const size_t b = p.n_prims * sizeof(sc_primitive) + p.n_planes * sizeof(sc_plane) +
                     p.n_mats * sizeof(sc_material) + 3 * kTableN * sizeof(float) + mask_words * sizeof(uint32_t);
    return (b + 15u) & ~size_t(15);
}

// 256 threads per CTA; MINB CTAs per SM bound the registers (4: 63 registers,
// no spills; 5: 48 registers, a few spills, more warps in flight).
// FF: built with free-flight sampling (estimator 3) as well.  EXACT: haze
// samples in the CPU crate's operation order (per-photon transport only).
template <bool SPEC, int AGG, int MINB, bool SPLIT, bool FF, bool EXACT = false>
__global__ void __launch_bounds__(256, MINB) photon_kernel(const PhotonParams p, uint32_t mask_words) {
    extern __shared__ __align__(16) unsigned char smem[];
    const float* cmf;
    uint32_t* smask;
    const SceneView S = load_scene(p, smem, &cmf, &smask, mask_words);
    if (SPLIT) {  // warp-split transport: per-warp segment buffers after the scene
        // warps take chunks of the launch's photons in grid-stride order (so the
        // photons in flight stay close in launch order: the wavelength-ordered
        // dispatch relies on it), and the lanes work through a chunk with refill;
        // chunks of up to 512 photons, smaller when that leaves warps idle
        using WS = WarpSplitSmem<kWarpSegs>;
        WS* ws = reinterpret_cast<WS*>(smem + split_offset(p, mask_words));
        const uint32_t warp = threadIdx.x >> 5;
        const uint32_t warps = gridDim.x * (blockDim.x >> 5), gw = blockIdx.x * (blockDim.x >> 5) + warp;
        const uint32_t per = (uint32_t)(((uint64_t)p.photon_count + warps - 1u) / warps);
        const uint32_t chunk = min(512u, max(32u, (per + 31u) & ~31u));
        for (uint64_t base = (uint64_t)gw * chunk; base < p.photon_count; base += (uint64_t)warps * chunk) {
            const uint32_t b0 = (uint32_t)base;
            const uint32_t cnt = min(chunk, p.photon_count - b0);
            trace_warp_range<SPEC, AGG, FF, kWarpSegs>(
                p, S, cmf, cnt, [&](uint32_t k) { return p.photon_base + (p.order ? p.order[b0 + k] : b0 + k); },
                smask, ws[warp]);
        }
    } else if (EXACT) {
        const uint32_t stride = gridDim.x * blockDim.x;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.photon_count; i += stride)
            trace_photon<SPEC, AGG, false, false, FF, true>(p, S, cmf, p.photon_base + (p.order ? p.order[i] : i),
                                                             smask);
    } else {
        trace_lane_range<SPEC, AGG, FF>(p, S, cmf, blockIdx.x * blockDim.x + threadIdx.x, p.photon_count,
                                        gridDim.x * blockDim.x,
                                        [&](uint32_t i) { return p.photon_base + (p.order ? p.order[i] : i); },
                                        smask);
    }
    if (smask) {  // publish this CTA's dirty tiles
        __syncthreads();
        for (uint32_t w = threadIdx.x; w < mask_words; w += blockDim.x)
            if (smask[w]) atomicOr(p.flags + w, smask[w]);
    }
}

// Instrumented pass: same transport, no film writes; sums the per-photon work
// counters into out[0..3] = photons, segments, in-frame samples, scatters.
__global__ void __launch_bounds__(256) photon_count_kernel(const PhotonParams p, unsigned long long* out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const float* cmf;
    const SceneView S = load_scene(p, smem, &cmf);
    unsigned long long seg = 0, spl = 0, sca = 0, ph = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < p.photon_count; i += gridDim.x * blockDim.x) {
        PhotonCounts c = {0u, 0u, 0u};
        trace_photon<false, 0, false, true>(p, S, cmf, p.photon_base + i, nullptr, &c);
        seg += c.segments; spl += c.splats; sca += c.scatters; ++ph;
    }
    for (int o = 16; o > 0; o >>= 1) {
        seg += __shfl_xor_sync(0xffffffffu, seg, o);
        spl += __shfl_xor_sync(0xffffffffu, spl, o);
        sca += __shfl_xor_sync(0xffffffffu, sca, o);
        ph += __shfl_xor_sync(0xffffffffu, ph, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, ph); atomicAdd(out + 1, seg); atomicAdd(out + 2, spl); atomicAdd(out + 3, sca);
    }
}

__global__ void __launch_bounds__(256) photon_debug_kernel(const PhotonParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const float* cmf;
    const SceneView S = load_scene(p, smem, &cmf);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < p.photon_count) trace_photon<false, 0, true>(p, S, cmf, i, nullptr);
}

// Surface rim pass (spectral-gpu/src/shaders/volume.wgsl:668-703 and its CPU
// oracle cpu_surface_rim, spectral-gpu/src/vol_photons.rs:1517-1538): one camera
// primary ray per pixel, nearest hit, rim = (1 - |n.d|)^2, tinted constant XYZ.
__global__ void __launch_bounds__(256) rim_kernel(const RimParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    sc_primitive* sp = reinterpret_cast<sc_primitive*>(smem);
    sc_plane* spl = reinterpret_cast<sc_plane*>(sp + p.n_prims);
    sc_material* sm = reinterpret_cast<sc_material*>(spl + p.n_planes);
    const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (uint32_t i = tid; i < p.n_prims; i += nt) sp[i] = p.prims[i];
    for (uint32_t i = tid; i < p.n_planes; i += nt) spl[i] = p.planes[i];
    for (uint32_t i = tid; i < p.n_mats; i += nt) sm[i] = p.mats[i];
    __syncthreads();
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= p.width || py >= p.height) return;
    SceneView S;
    S.prims = sp; S.planes = spl; S.mats = sm; S.n_prims = p.n_prims;
    const float s = ((float)px + 0.5f) / (float)p.width;
    const float t = 1.0f - ((float)py + 0.5f) / (float)p.height;
    const f3 o = ld3(p.cam.origin), d = primary_dir(p.cam, s, t);
    Hit h;
    uint32_t mi;
    const size_t i = (size_t)py * p.width + px;
    float x = 0.f, y = 0.f, z = 0.f;
    if (scene_hit(S, o, d, h, mi)) {
        const float c = fminf(fmaxf(fabsf(dot(h.normal, d)), 0.0f), 1.0f);
        const float rim = (1.0f - c) * (1.0f - c);
        x = 0.015f + rim * 0.45f; y = 0.02f + rim * 0.5f; z = 0.04f + rim * 0.6f;
    }
    p.out[3 * i] = x; p.out[3 * i + 1] = y; p.out[3 * i + 2] = z;
}

__global__ void rng_draws_kernel(uint32_t key, uint32_t seed, uint32_t n, uint32_t* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    Rng r = Rng::make(key, seed);
    for (uint32_t i = 0; i < n; ++i) out[i] = r.u32();
}

// ---------------------------------------------------------------------------
// Wavelength-ordered dispatch.  Film cells are pixel-major (the bins of a pixel
// are adjacent), so photons of random wavelengths traced together touch every
// 32-byte sector of every pixel they reach, and a spectral film larger than L2
// misses on most of its atomics.  Tracing the photons of a launch in order of
// their film bin keeps the photons in flight within a few bins: about one
// sector per pixel is live at a time.  The photons and their paths are the
// same and the film is a sum of exact integers, so the image is bit-identical.
// Counting sort of the launch's photons by key (kOrderKeys groups of
// consecutive bins): per-CTA key histograms of contiguous photon chunks
// (key-major), one exclusive scan, then a scatter that stages 2048 photons at a
// time in shared memory so that each key's run is written contiguously.
constexpr uint32_t kOrderKeys = 16;
constexpr uint32_t kOrderTile = 2048;  // photons per scatter step: 8 per thread

// Sort key of photon `idx`: the group of its film bin (its third draw, as in
// the transport).
__device__ __forceinline__ uint32_t photon_key(const PhotonParams& p, uint32_t idx) {
    Rng r = Rng::make(idx, p.seed);
    r.state += 2u;  // the two aperture draws
    const float lambda = p.lambda_min + p.lambda_range * r.f32();
    const float fb = (lambda - p.bin_min) * p.bin_inv_width;
    const int bi = (int)fb;
    const uint32_t bin = fb < 0.0f ? 0u : (bi >= (int)p.bins ? p.bins - 1u : (uint32_t)bi);
    return p.bins <= kOrderKeys ? bin : bin * kOrderKeys / p.bins;
}

__global__ void __launch_bounds__(256) order_count_kernel(const PhotonParams p, uint32_t per_cta,
                                                          uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[kOrderKeys];
    const uint32_t K = min(p.bins, kOrderKeys);
    if (threadIdx.x < K) h[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t i0 = blockIdx.x * per_cta, i1 = min(i0 + per_cta, p.photon_count);
    for (uint32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) atomicAdd(&h[photon_key(p, p.photon_base + i)], 1u);
    __syncthreads();
    if (threadIdx.x < K) hist[threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// In-place exclusive scan of n counts by one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) order_scan_kernel(uint32_t* __restrict__ a, uint32_t n) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x, per = (n + 1023u) / 1024u;
    const uint32_t lo = min(t * per, n), hi = min(lo + per, n);
    uint32_t sum = 0;
    for (uint32_t i = lo; i < hi; ++i) sum += a[i];
    part[t] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < 1024u; off <<= 1) {
        const uint32_t v = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = t ? part[t - 1] : 0u;
    for (uint32_t i = lo; i < hi; ++i) {
        const uint32_t c = a[i];
        a[i] = run;
        run += c;
    }
}

// Blocks of 256 threads.
__global__ void __launch_bounds__(256) order_scatter_kernel(const PhotonParams p, uint32_t per_cta,
                                                            const uint32_t* __restrict__ offsets,
                                                            uint32_t* __restrict__ order) {
    __shared__ uint32_t cur[kOrderKeys], cnt[kOrderKeys], toff[kOrderKeys];
    __shared__ uint32_t stage[kOrderTile];
    __shared__ uint8_t skey[kOrderTile];
    const uint32_t tid = threadIdx.x, K = min(p.bins, kOrderKeys);
    if (tid < K) cur[tid] = offsets[tid * gridDim.x + blockIdx.x];
    const uint32_t i0 = blockIdx.x * per_cta, i1 = min(i0 + per_cta, p.photon_count);
    for (uint32_t t0 = i0; t0 < i1; t0 += kOrderTile) {
        if (tid < K) cnt[tid] = 0u;
        __syncthreads();
        uint32_t key[8], rank[8];
#pragma unroll
        for (uint32_t j = 0; j < 8u; ++j) {
            const uint32_t i = t0 + j * 256u + tid;
            key[j] = i < i1 ? photon_key(p, p.photon_base + i) : 0xFFu;
            rank[j] = key[j] != 0xFFu ? atomicAdd(&cnt[key[j]], 1u) : 0u;  // rank within the tile's key run
        }
        __syncthreads();
        if (tid == 0) {
            uint32_t sum = 0;
            for (uint32_t k = 0; k < K; ++k) { toff[k] = sum; sum += cnt[k]; }
        }
        __syncthreads();
#pragma unroll
        for (uint32_t j = 0; j < 8u; ++j) {
            if (key[j] != 0xFFu) {
                const uint32_t pos = toff[key[j]] + rank[j];
                stage[pos] = t0 + j * 256u + tid;
                skey[pos] = (uint8_t)key[j];
            }
        }
        __syncthreads();
        const uint32_t n = min(kOrderTile, i1 - t0);
        for (uint32_t q = tid; q < n; q += 256u) {
            const uint32_t k = skey[q];
            order[cur[k] + (q - toff[k])] = stage[q];
        }
        __syncthreads();
        if (tid < K) cur[tid] += cnt[tid];
    }
}

__global__ void glass_n_kernel(uint32_t glass, const float* __restrict__ lambda_nm, uint32_t n,
                               float* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = glass_n(glass, lambda_nm[i]);
}

}  // namespace

cudaError_t launch_glass_n(uint32_t glass, const float* lambda_nm, uint32_t n, float* out, cudaStream_t s) {
    const uint32_t need = (n + 255u) / 256u, grid = need < 148u * 16u ? need : 148u * 16u;
    glass_n_kernel<<<grid, 256, 0, s>>>(glass, lambda_nm, n, out);
    return cudaGetLastError();
}

cudaError_t launch_rng_draws(uint32_t key, uint32_t seed, uint32_t n, uint32_t* out, cudaStream_t s) {
    rng_draws_kernel<<<1, 32, 0, s>>>(key, seed, n, out);
    return cudaGetLastError();
}

size_t scene_smem_bytes(uint32_t n_prims, uint32_t n_planes, uint32_t n_mats) {
    return n_prims * sizeof(sc_primitive) + n_planes * sizeof(sc_plane) + n_mats * sizeof(sc_material) +
           3 * kTableN * sizeof(float);
}

using PhotonKernelFn = void (*)(const PhotonParams, uint32_t);

template <bool SPLIT>
static PhotonKernelFn photon_fn_t(bool spec, int agg, int minb, bool ff, bool exact) {
    // haze samples in the reference's operation order: per-photon transport,
    // plain atomics, 4 CTAs per SM
    if (exact && !SPLIT) {
        if (ff) return spec ? photon_kernel<true, 0, 4, false, true, true> : photon_kernel<false, 0, 4, false, true, true>;
        return spec ? photon_kernel<true, 0, 4, false, false, true> : photon_kernel<false, 0, 4, false, false, true>;
    }
    // free-flight launches: plain atomics, 4 CTAs per SM
    if (ff) return spec ? photon_kernel<true, 0, 4, SPLIT, true> : photon_kernel<false, 0, 4, SPLIT, true>;
    if (minb >= 5) {
        if (spec) return agg ? photon_kernel<true, 1, 5, SPLIT, false> : photon_kernel<true, 0, 5, SPLIT, false>;
        return agg ? photon_kernel<false, 1, 5, SPLIT, false> : photon_kernel<false, 0, 5, SPLIT, false>;
    }
    if (spec) return agg ? photon_kernel<true, 1, 4, SPLIT, false> : photon_kernel<true, 0, 4, SPLIT, false>;
    return agg ? photon_kernel<false, 1, 4, SPLIT, false> : photon_kernel<false, 0, 4, SPLIT, false>;
}
static PhotonKernelFn photon_fn(const LaunchShape& s, bool spec, bool ff, bool exact = false) {
    return s.split && !exact ? photon_fn_t<true>(spec, s.aggregate, s.minb, ff, false)
                             : photon_fn_t<false>(spec, s.aggregate, s.minb, ff, exact);
}
// Shared memory beyond scene + mask: one segment buffer per warp (8 warps).
static size_t split_bytes(const LaunchShape& s) {
    return s.split ? 16 + 8 * sizeof(WarpSplitSmem<kWarpSegs>) : 0;
}

void set_haze_consts(PhotonParams& p) {
    const double pi = 3.14159265358979323846;
    const double g = p.g;
    p.hz_w = (float)p.width;
    p.hz_h = (float)p.height;
    p.hz_hw = 0.5f * p.hz_w;
    p.hz_hh = 0.5f * p.hz_h;
    p.hz_sx = (float)((double)p.width / (double)p.proj.vw);
    p.hz_sy = (float)(-(double)p.height / (double)p.proj.vh);
    p.hz_k = (float)((double)p.sigma_s * (double)p.scale * 0.25 * (1.0 - g * g) / (4.0 * pi));
    p.hz_kiso = (float)((double)p.sigma_s * (double)p.scale * 0.25 / (4.0 * pi));
    p.hz_kexp = (float)(-(double)p.sigma_t * 1.4426950408889634);  // -sigma_t log2(e)
    p.hz_inv_sigma_t = p.sigma_t > 0.0f ? (float)(1.0 / (double)p.sigma_t) : 0.0f;
    p.hz_g2 = (float)(1.0 + g * g);
    p.hz_m2g = (float)(-2.0 * g);
}

int occupancy_blocks(const void* fn, int block, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, int, size_t>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_tuple(dev, fn, block, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int n = 0;
    if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, block, smem) != cudaSuccess) return 1;
    n = n > 0 ? n : 1;
    cache.emplace(key, n);
    return n;
}

int photon_occupancy_blocks(const LaunchShape& shape, bool spectral, size_t smem) {
    return occupancy_blocks(reinterpret_cast<const void*>(photon_fn(shape, spectral, false)), (int)shape.block,
                            smem + split_bytes(shape));
}

uint32_t photon_mask_words(const PhotonParams& p) {
    if (!p.flags) return 0u;
    const uint32_t tiles = p.tiles_x * ((p.height + 7u) / 8u);
    const uint32_t words = (tiles + 31u) / 32u;
    return words <= kMaxSmemMaskWords ? words : 0u;
}

// L2 bytes of the current device, read once per device.
static size_t l2_bytes() {
    static std::mutex mu;
    static std::map<int, size_t> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(dev);
    if (it != cache.end()) return it->second;
    int b = 0;
    cudaDeviceGetAttribute(&b, cudaDevAttrL2CacheSize, dev);
    cache.emplace(dev, (size_t)(b > 0 ? b : 0));
    return (size_t)(b > 0 ? b : 0);
}

// Whether a launch takes the wavelength-ordered dispatch: point / isotropic
// estimators on a spectral film larger than L2 (order 1) or on any spectral
// film (order 2), at least 2^16 photons to amortise the sort, and a memory
// pool for its scratch.
static bool ordered_dispatch(const PhotonParams& p, const LaunchShape& shape) {
    if (shape.order == 0 || !shape.pool || p.bins == 0u || p.channels != p.bins || p.order ||
        p.photon_count < (1u << 16))
        return false;
    if (shape.order >= 2) return true;
    const size_t film = (size_t)p.tiles_x * ((p.height + 7u) / 8u) * kTilePixels * p.channels * 8u;
    return film > l2_bytes();
}

static cudaError_t launch_photons_in(const PhotonParams& p, const LaunchShape& shape, cudaStream_t s);

cudaError_t launch_photons(const PhotonParams& p, const LaunchShape& shape, cudaStream_t s) {
    if (p.photon_count == 0) return cudaSuccess;
    if (!ordered_dispatch(p, shape)) return launch_photons_in(p, shape, s);
    const uint32_t grid = 148u * 4u;  // sort CTAs, each a contiguous chunk of the launch's photons
    const uint32_t per_cta = (p.photon_count + grid - 1u) / grid;
    const uint32_t keys = p.bins < kOrderKeys ? p.bins : kOrderKeys;
    const size_t words = (size_t)p.photon_count + (size_t)keys * grid;
    uint32_t* buf = nullptr;
    if (cudaMallocFromPoolAsync(reinterpret_cast<void**>(&buf), words * sizeof(uint32_t), shape.pool, s) !=
        cudaSuccess) {
        cudaGetLastError();  // no room for the sort: trace in launch order (same image)
        return launch_photons_in(p, shape, s);
    }
    uint32_t* order = buf;
    uint32_t* hist = buf + p.photon_count;
    order_count_kernel<<<grid, 256, 0, s>>>(p, per_cta, hist);
    order_scan_kernel<<<1, 1024, 0, s>>>(hist, keys * grid);
    order_scatter_kernel<<<grid, 256, 0, s>>>(p, per_cta, hist, order);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        PhotonParams q = p;
        q.order = order;
        e = launch_photons_in(q, shape, s);
    }
    const cudaError_t f = cudaFreeAsync(buf, s);
    return e != cudaSuccess ? e : f;
}

static cudaError_t launch_photons_in(const PhotonParams& p0, const LaunchShape& shape, cudaStream_t s) {
    PhotonParams p = p0;
    set_haze_consts(p);
    const bool exact = p.haze_exact != 0u;
    const uint32_t mw = photon_mask_words(p);
    const size_t smem = shape.split && !exact
                            ? split_offset(p, mw) + 8 * sizeof(WarpSplitSmem<kWarpSegs>)
                            : scene_smem_bytes(p.n_prims, p.n_planes, p.n_mats) + mw * sizeof(uint32_t);
    const bool spec = p.channels != 3u || p.bins != 0u;
    const uint32_t need = (p.photon_count + 255u) / 256u;
    const uint32_t grid = need < shape.grid ? need : shape.grid;
    const PhotonKernelFn fn = photon_fn(shape, spec, free_flight(p), exact);
    if (smem > 48 * 1024) occupancy_blocks(reinterpret_cast<const void*>(fn), 256, smem);  // raises its limit once
    fn<<<grid, 256, smem, s>>>(p, mw);
    return cudaGetLastError();
}

cudaError_t launch_photon_debug(const PhotonParams& p, cudaStream_t s) {
    if (p.photon_count == 0) return cudaSuccess;
    const size_t smem = scene_smem_bytes(p.n_prims, p.n_planes, p.n_mats);
    photon_debug_kernel<<<(p.photon_count + 255) / 256, 256, smem, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_photon_count(const PhotonParams& p0, unsigned long long* out, uint32_t grid, cudaStream_t s) {
    if (p0.photon_count == 0) return cudaSuccess;
    PhotonParams p = p0;
    set_haze_consts(p);
    const size_t smem = scene_smem_bytes(p.n_prims, p.n_planes, p.n_mats);
    const uint32_t need = (p.photon_count + 255) / 256;
    photon_count_kernel<<<need < grid ? need : grid, 256, smem, s>>>(p, out);
    return cudaGetLastError();
}

cudaError_t launch_rim(const RimParams& p, cudaStream_t s) {
    const size_t smem = p.n_prims * sizeof(sc_primitive) + p.n_planes * sizeof(sc_plane) + p.n_mats * sizeof(sc_material);
    dim3 block(16, 16), grid((p.width + 15) / 16, (p.height + 15) / 16);
    rim_kernel<<<grid, block, smem, s>>>(p);
    return cudaGetLastError();
}

}  // namespace sc
