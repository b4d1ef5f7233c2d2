// Film kernels: sensor reduction / drain, exposure, tonemap, Gaussian gather,
// and the synthetic atomic-film splat.
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>

#include "internal.h"

namespace sc {

namespace {

constexpr int kReduceThreads = 256;

// One film tile (64 pixels x C channels of int64) is staged into shared memory
// with 16-byte coalesced loads, optionally zeroed behind the load (drain), then
// reduced per pixel: XYZ film -> value / 2^scale; spectral film -> sum over bins
// of count * bin-averaged CMF (f64 accumulation, fixed order per pixel).
// Tiles whose dirty flag is clear are never read: their pixels are written as 0.
//
// Software pipeline: a CTA walks its tiles keeping the next tile's first
// 8 x 256 16-byte vectors (a whole tile up to 64 channels) in registers, so
// those loads are in flight while the current tile is reduced out of shared
// memory.
struct TileRef {
    ReduceParams p;
    uint32_t tile;
    bool valid, dirty, keep;  // keep: never drained (an accumulating film)
};

__device__ __forceinline__ TileRef tile_ref(const ReduceParams& p, uint32_t tile, bool valid, bool keep = false) {
    TileRef t;
    t.p = p;
    t.tile = tile;
    t.valid = valid;
    t.keep = keep;
    t.dirty = valid && (p.flags == nullptr || ((p.flags[tile >> 5] >> (tile & 31u)) & 1u));
    return t;
}

constexpr uint32_t kPrefetch = 8;  // 16-byte vectors per thread held across a tile

__device__ __forceinline__ void prefetch_tile(const TileRef& t, ulonglong2 (&v)[kPrefetch]) {
    if (!t.dirty) return;
    const ulonglong2* src = reinterpret_cast<const ulonglong2*>(t.p.film + (size_t)t.tile * kTilePixels * t.p.channels);
    const uint32_t n2 = kTilePixels * t.p.channels / 2u;
#pragma unroll
    for (uint32_t k = 0; k < kPrefetch; ++k) {
        const uint32_t i = threadIdx.x + k * blockDim.x;
        if (i < n2) v[k] = __ldcs(src + i);
    }
}

// Registers (and any vectors beyond them) into shared memory; zero the film
// behind the copy when draining.
__device__ __forceinline__ void stage_tile(const TileRef& t, const ulonglong2 (&v)[kPrefetch], bool drain,
                                           unsigned long long* sm) {
    if (!t.dirty) return;
    ulonglong2* src = reinterpret_cast<ulonglong2*>(t.p.film + (size_t)t.tile * kTilePixels * t.p.channels);
    ulonglong2* dst = reinterpret_cast<ulonglong2*>(sm);
    const uint32_t n2 = kTilePixels * t.p.channels / 2u;
    const ulonglong2 zero = make_ulonglong2(0ull, 0ull);
#pragma unroll
    for (uint32_t k = 0; k < kPrefetch; ++k) {
        const uint32_t i = threadIdx.x + k * blockDim.x;
        if (i < n2) {
            dst[i] = v[k];
            if (drain) __stcs(src + i, zero);
        }
    }
    for (uint32_t i = threadIdx.x + kPrefetch * blockDim.x; i < n2; i += blockDim.x) {  // > 64 channels
        dst[i] = __ldcs(src + i);
        if (drain) __stcs(src + i, zero);
    }
}

// Per-pixel reduction of a staged tile (or zeros for a clean one).
__device__ __forceinline__ void reduce_staged(const TileRef& t, bool drain, const unsigned long long* sm,
                                              double* part) {
    const ReduceParams& p = t.p;
    const uint32_t C = p.channels, tile = t.tile;
    const uint32_t tx = tile % p.tiles_x, ty = tile / p.tiles_x;
    const uint32_t tid = threadIdx.x;
    if (!t.dirty || C == 3u) {
        for (uint32_t i = tid; i < kTilePixels * 3u; i += blockDim.x) {
            const uint32_t l = i / 3u, c = i % 3u;
            const uint32_t px = tx * 8u + (l & 7u), py = ty * 8u + (l >> 3);
            if (px < p.width && py < p.height)
                p.xyz[((size_t)py * p.width + px) * 3u + c] =
                    t.dirty ? (float)((double)(long long)sm[i] * p.inv_scale) : 0.0f;
        }
    } else {
        // 4 threads per pixel, each a contiguous quarter of the bins; partials
        // are summed in quarter order so the result does not depend on timing.
        const uint32_t l = tid & 63u, q = tid >> 6;
        if (q < 4u) {
            const uint32_t b0 = q * C / 4u, b1 = (q + 1u) * C / 4u, span = b1 - b0;
            double x = 0.0, y = 0.0, z = 0.0;
            const unsigned long long* row = sm + (size_t)l * C;
            for (uint32_t j = 0; j < span; ++j) {
                const uint32_t b = b0 + (j + l) % span;  // rotate to spread banks
                const double v = (double)(long long)row[b];
                x += v * (double)p.binw[b];
                y += v * (double)p.binw[C + b];
                z += v * (double)p.binw[2u * C + b];
            }
            part[(q * 64u + l) * 3u] = x; part[(q * 64u + l) * 3u + 1u] = y; part[(q * 64u + l) * 3u + 2u] = z;
        }
        __syncthreads();
        if (tid < 64u) {
            const uint32_t px = tx * 8u + (tid & 7u), py = ty * 8u + (tid >> 3);
            if (px < p.width && py < p.height) {
                float* o = p.xyz + ((size_t)py * p.width + px) * 3u;
                for (uint32_t c = 0; c < 3u; ++c) {
                    const double s = ((part[tid * 3u + c] + part[(64u + tid) * 3u + c]) + part[(128u + tid) * 3u + c]) +
                                     part[(192u + tid) * 3u + c];
                    o[c] = (float)(s * p.inv_scale);
                }
            }
        }
    }
    if (drain && t.dirty && p.flags && tid == 0) atomicAnd(p.flags + (tile >> 5), ~(1u << (tile & 31u)));
}

// The pipelined walk over this CTA's tiles; `at(k)` gives its k-th tile.
template <bool DRAIN, class At>
__device__ __forceinline__ void reduce_walk(At at, unsigned long long* sm, double* part) {
    ulonglong2 v[kPrefetch];
    TileRef cur = at(0u);
    prefetch_tile(cur, v);
    for (uint32_t k = 0; cur.valid; ++k) {
        stage_tile(cur, v, DRAIN && !cur.keep, sm);
        __syncthreads();
        const TileRef nxt = at(k + 1u);
        prefetch_tile(nxt, v);  // in flight while this tile is reduced
        reduce_staged(cur, DRAIN && !cur.keep, sm, part);
        __syncthreads();
        cur = nxt;
    }
}

template <bool DRAIN>
__global__ void __launch_bounds__(kReduceThreads, 3) reduce_kernel(const ReduceParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    double* part = reinterpret_cast<double*>(smem);
    unsigned long long* sm = reinterpret_cast<unsigned long long*>(smem + 4 * 64 * 3 * sizeof(double));
    const uint32_t ntiles = p.tiles_x * p.tiles_y;
    reduce_walk<DRAIN>(
        [&](uint32_t k) {
            const uint32_t tile = blockIdx.x + k * gridDim.x;
            return tile_ref(p, tile < ntiles ? tile : 0u, tile < ntiles);
        },
        sm, part);
}

// The sum of several films (one per GPU of a split scene: this GPU's own and
// its peers', read over NVLink) reduced for a range of tiles.  Each tile is
// staged as the exact int64 sum of the films' cells, then reduced by the
// single-film code, so a band equals the same band of the summed film's
// image.  The films are read, not drained; every tile counts as lit.
__global__ void __launch_bounds__(kReduceThreads, 3) reduce_peers_kernel(const ReduceParams p, const PeerFilms pf,
                                                                         uint32_t tile_begin, uint32_t tile_end) {
    extern __shared__ __align__(16) unsigned char smem[];
    double* part = reinterpret_cast<double*>(smem);
    unsigned long long* sm = reinterpret_cast<unsigned long long*>(smem + 4 * 64 * 3 * sizeof(double));
    const uint32_t n2 = kTilePixels * p.channels / 2u;
    for (uint32_t tile = tile_begin + blockIdx.x; tile < tile_end; tile += gridDim.x) {
        const size_t off2 = (size_t)tile * kTilePixels * p.channels / 2u;
        for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) {
            ulonglong2 acc = make_ulonglong2(0ull, 0ull);
            for (uint32_t f = 0; f < pf.n; ++f) {
                const ulonglong2 v = __ldcs(reinterpret_cast<const ulonglong2*>(pf.film[f]) + off2 + i);
                acc.x += v.x;
                acc.y += v.y;
            }
            reinterpret_cast<ulonglong2*>(sm)[i] = acc;
        }
        __syncthreads();
        reduce_staged(tile_ref(p, tile, true), false, sm, part);
        __syncthreads();
    }
}

// Many films, step 1: one warp per dirty-mask word (32 tiles).  Clean tiles get
// zeros in the image; dirty ones go to the list (one atomic per warp), and
// when draining the word is cleared.  Words are numbered over all films
// (FilmDesc::word_begin), so a warp finds its film by a binary search.
template <bool DRAIN>
__global__ void __launch_bounds__(256) reduce_scan_kernel(const FilmDesc* __restrict__ descs, uint32_t n_films,
                                                          uint32_t total_words, DirtyTile* __restrict__ list,
                                                          uint32_t* __restrict__ count) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < total_words; w += warps) {
        uint32_t lo = 0, hi = n_films;
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (descs[mid].word_begin <= w) lo = mid; else hi = mid;
        }
        const FilmDesc& d = descs[lo];
        const uint32_t wl = w - d.word_begin;
        const uint32_t bits = d.flags[wl];
        const uint32_t tile = wl * 32u + lane;
        const bool valid = tile < d.tiles_x * d.tiles_y;
        const bool dirty = valid && ((bits >> lane) & 1u);
        const unsigned dm = __ballot_sync(0xffffffffu, dirty);
        if (dm) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(count, (uint32_t)__popc(dm));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (dirty) list[base + __popc(dm & ((1u << lane) - 1u))] = DirtyTile{lo, tile};
            if (DRAIN && !d.keep && lane == 0) d.flags[wl] = 0u;
        }
        // zeros for the clean tiles: 8 rows x 24 floats each, 6 coalesced stores per lane
        for (unsigned cm = __ballot_sync(0xffffffffu, valid && !dirty); cm; cm &= cm - 1u) {
            const uint32_t t = wl * 32u + (uint32_t)(__ffs(cm) - 1);
            const uint32_t tx = t % d.tiles_x, ty = t / d.tiles_x;
#pragma unroll
            for (uint32_t k = 0; k < 6u; ++k) {
                const uint32_t i = lane + 32u * k, row = i / 24u, col = i % 24u;
                const uint32_t px = tx * 8u + col / 3u, py = ty * 8u + row;
                if (px < d.width && py < d.height) d.xyz[((size_t)py * d.width + tx * 8u) * 3u + col] = 0.0f;
            }
        }
    }
}

// Many films, step 2: the listed dirty tiles through the pipelined walk.
template <bool DRAIN>
__global__ void __launch_bounds__(kReduceThreads, 3) reduce_list_kernel(const FilmDesc* __restrict__ descs,
                                                                     const DirtyTile* __restrict__ list,
                                                                     const uint32_t* __restrict__ count) {
    extern __shared__ __align__(16) unsigned char smem[];
    double* part = reinterpret_cast<double*>(smem);
    unsigned long long* sm = reinterpret_cast<unsigned long long*>(smem + 4 * 64 * 3 * sizeof(double));
    const uint32_t n = *count;
    reduce_walk<DRAIN>(
        [&](uint32_t k) {
            const uint32_t i = blockIdx.x + k * gridDim.x;
            ReduceParams p;
            if (i >= n) {
                p = ReduceParams{};
                return tile_ref(p, 0u, false);
            }
            const DirtyTile e = list[i];
            const FilmDesc& d = descs[e.film];
            p.film = d.film; p.flags = nullptr; p.xyz = d.xyz; p.width = d.width; p.height = d.height;
            p.tiles_x = d.tiles_x; p.tiles_y = d.tiles_y; p.channels = d.channels; p.binw = d.binw;
            p.inv_scale = d.inv_scale;
            return tile_ref(p, e.tile, true, d.keep != 0u);
        },
        sm, part);
}

__global__ void composite_max_y_kernel(const float* __restrict__ xyz, const float* __restrict__ surface,
                                       uint32_t n, uint32_t* out_bits) {
    float m = 0.0f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float y = xyz[3u * i + 1u] + (surface ? surface[3u * i + 1u] : 0.0f);
        m = fmaxf(m, y);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0f) atomicMax(out_bits, __float_as_uint(m));
}

// Radix select of the k-th smallest composited luminance (values >= 0, so the
// IEEE bit patterns order like the floats).  work: [0..255] histogram,
// [256] prefix, [257] k remaining, [258] result bits.
__global__ void select_hist_kernel(const float* __restrict__ xyz, const float* __restrict__ surface, uint32_t n,
                                   uint32_t* work, int shift) {
    __shared__ uint32_t hist[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0u;
    __syncthreads();
    const uint32_t prefix = work[256];
    const uint32_t hi_mask = shift >= 24 ? 0u : (0xFFFFFFFFu << (shift + 8));
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float y = xyz[3u * i + 1u] + (surface ? surface[3u * i + 1u] : 0.0f);
        y = fmaxf(y, 0.0f);
        const uint32_t bits = __float_as_uint(y);
        if ((bits & hi_mask) == (prefix & hi_mask)) atomicAdd(&hist[(bits >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (hist[i]) atomicAdd(&work[i], hist[i]);
}
__global__ void select_pick_kernel(uint32_t* work, int shift) {
    if (threadIdx.x != 0) return;
    uint32_t k = work[257], acc = 0;
    uint32_t b = 0;
    for (; b < 255u; ++b) {
        if (acc + work[b] > k) break;
        acc += work[b];
    }
    work[256] |= b << shift;
    work[257] = k - acc;
    for (int i = 0; i < 256; ++i) work[i] = 0u;
    if (shift == 0) work[258] = work[256];
}

__global__ void to_rgb8_kernel(const float* __restrict__ xyz, const float* __restrict__ surface, uint32_t n,
                               float exposure, uint8_t* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float c[3];
    for (int k = 0; k < 3; ++k) c[k] = xyz[3u * i + k] + (surface ? surface[3u * i + k] : 0.0f);
    // xyz_to_linear_srgb + tonemap_to_u8 (spectral-core/src/cie.rs:121-144)
    const float lin[3] = {3.2406f * c[0] - 1.5372f * c[1] - 0.4986f * c[2],
                          -0.9689f * c[0] + 1.8758f * c[1] + 0.0415f * c[2],
                          0.0557f * c[0] - 0.2040f * c[1] + 1.0570f * c[2]};
    for (int k = 0; k < 3; ++k) {
        const float v = fmaxf(lin[k] * exposure, 0.0f);
        const float mapped = v / (1.0f + v);
        float gm = mapped <= 0.0031308f ? 12.92f * mapped : 1.055f * powf(mapped, 1.0f / 2.4f) - 0.055f;
        gm = fminf(fmaxf(gm, 0.0f), 1.0f);
        const float q = gm * 255.0f + 0.5f;
        out[3u * i + k] = (uint8_t)(q >= 255.0f ? 255.0f : q);
    }
}

// Viewer reconstruction (spectral-viewer/src/main.rs:132-173): normalized
// Gaussian gather, radius kradius, sigma max(kradius/2, 0.5), scaled by k, plus
// the rim surface, XYZ -> linear sRGB, Reinhard, gamma 1/2.2, RGBA8.
__global__ void gather_kernel(const float* __restrict__ xyz, const float* __restrict__ surface, uint32_t w,
                              uint32_t h, float k, float kradius, float exposure, uint8_t* out) {
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= w || py >= h) return;
    const int radius = (int)kradius;
    const float sigma = fmaxf(kradius * 0.5f, 0.5f);
    const float inv2s2 = 1.0f / (2.0f * sigma * sigma);
    float acc[3] = {0.f, 0.f, 0.f}, wsum = 0.0f;
    for (int dy = -radius; dy <= radius; ++dy)
        for (int dx = -radius; dx <= radius; ++dx) {
            const int sx = (int)px + dx, sy = (int)py + dy;
            if (sx >= 0 && sx < (int)w && sy >= 0 && sy < (int)h) {
                const size_t si = (size_t)sy * w + sx;
                const float g = expf(-(float)(dx * dx + dy * dy) * inv2s2);
                for (int c = 0; c < 3; ++c) acc[c] = acc[c] + xyz[3 * si + c] * g;
                wsum = wsum + g;
            }
        }
    const size_t i = (size_t)py * w + px;
    const float kk = k / fmaxf(wsum, 1e-6f);
    float comp[3];
    for (int c = 0; c < 3; ++c) comp[c] = (acc[c] * kk + (surface ? surface[3 * i + c] : 0.0f)) * exposure;
    const float lin[3] = {3.2406f * comp[0] - 1.5372f * comp[1] - 0.4986f * comp[2],
                          -0.9689f * comp[0] + 1.8758f * comp[1] + 0.0415f * comp[2],
                          0.0557f * comp[0] - 0.2040f * comp[1] + 1.0570f * comp[2]};
    const float inv_gamma = (float)(1.0 / 2.2);
    for (int c = 0; c < 3; ++c) {
        const float tt = lin[c] / (1.0f + lin[c]);
        float v = powf(fmaxf(tt, 0.0f), inv_gamma);
        v = fminf(fmaxf(v, 0.0f), 1.0f);
        out[4 * i + c] = (uint8_t)(v * 255.0f + 0.5f);
    }
    out[4 * i + 3] = 255;
}

// Synthetic splat (spectral-gpu/src/shaders/vol_splat.wgsl:34-55): one thread
// per splat, a hashed pixel, XYZ in [0,2), x4096 truncated, three u32 atomics.
__global__ void synthetic_splat_kernel(uint32_t* film, uint32_t w, uint32_t h, uint32_t seed, uint32_t n) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    Rng r = Rng::make(t, seed);
    const uint32_t idx = r.u32() % (w * h);
    const float x = r.f32() * 2.0f, y = r.f32() * 2.0f, z = r.f32() * 2.0f;
    atomicAdd(film + 3u * idx, (uint32_t)(fmaxf(x, 0.0f) * 4096.0f));
    atomicAdd(film + 3u * idx + 1u, (uint32_t)(fmaxf(y, 0.0f) * 4096.0f));
    atomicAdd(film + 3u * idx + 2u, (uint32_t)(fmaxf(z, 0.0f) * 4096.0f));
}
// AtomicFilm::resolve (spectral-gpu/src/film.rs:218-224), on the device.
__global__ void atomic_resolve_kernel(uint32_t* film, float* accum, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t v = film[i];
        film[i] = 0u;
        accum[i] += (float)v / 4096.0f;
    }
}

size_t reduce_smem(uint32_t channels) {
    return 4 * 64 * 3 * sizeof(double) + (size_t)kTilePixels * channels * sizeof(unsigned long long);
}

}  // namespace

// Resident CTAs of a reduce kernel on the current device for `smem` bytes of
// dynamic shared memory, worked out once per (device, kernel, size) (raising
// the kernel's shared-memory limit on the way) and then served from a table.
static uint32_t reduce_grid(const void* fn, int which, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, size_t>, uint32_t> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_tuple(dev, which, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kReduceThreads, smem);
    const uint32_t grid = (uint32_t)sms * (uint32_t)(per_sm > 0 ? per_sm : 1);
    cache.emplace(key, grid);
    return grid;
}

cudaError_t launch_reduce(const ReduceParams& p, bool drain, cudaStream_t s) {
    const size_t smem = reduce_smem(p.channels);
    const uint32_t ntiles = p.tiles_x * p.tiles_y;
    const void* fn = drain ? reinterpret_cast<const void*>(&reduce_kernel<true>)
                           : reinterpret_cast<const void*>(&reduce_kernel<false>);
    uint32_t grid = reduce_grid(fn, drain ? 1 : 0, smem);
    if (grid > ntiles) grid = ntiles;
    if (grid == 0) return cudaSuccess;
    if (drain) reduce_kernel<true><<<grid, kReduceThreads, smem, s>>>(p);
    else reduce_kernel<false><<<grid, kReduceThreads, smem, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_reduce_peers(const ReduceParams& p, const PeerFilms& films, uint32_t tile_begin, uint32_t tile_end,
                                cudaStream_t s) {
    if (tile_end <= tile_begin || films.n == 0) return cudaSuccess;
    const size_t smem = reduce_smem(p.channels);
    uint32_t grid = reduce_grid(reinterpret_cast<const void*>(&reduce_peers_kernel), 2, smem);
    if (grid > tile_end - tile_begin) grid = tile_end - tile_begin;
    reduce_peers_kernel<<<grid, kReduceThreads, smem, s>>>(p, films, tile_begin, tile_end);
    return cudaGetLastError();
}

cudaError_t launch_reduce_many(const FilmDesc* descs, uint32_t n_films, uint32_t total_words, bool drain,
                               uint32_t max_channels, DirtyTile* list, uint32_t* count, cudaStream_t s) {
    if (total_words == 0 || n_films == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t need = (total_words + 7u) / 8u, cap = (uint32_t)sms * 8u;
    const uint32_t sgrid = need < cap ? need : cap;
    if (drain) reduce_scan_kernel<true><<<sgrid, 256, 0, s>>>(descs, n_films, total_words, list, count);
    else reduce_scan_kernel<false><<<sgrid, 256, 0, s>>>(descs, n_films, total_words, list, count);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t smem = reduce_smem(max_channels);
    const void* fn = drain ? reinterpret_cast<const void*>(&reduce_list_kernel<true>)
                           : reinterpret_cast<const void*>(&reduce_list_kernel<false>);
    const uint32_t grid = reduce_grid(fn, drain ? 3 : 2, smem);
    if (drain) reduce_list_kernel<true><<<grid, kReduceThreads, smem, s>>>(descs, list, count);
    else reduce_list_kernel<false><<<grid, kReduceThreads, smem, s>>>(descs, list, count);
    return cudaGetLastError();
}

cudaError_t launch_composite_max_y(const float* xyz, const float* surface, uint32_t n, uint32_t* out_bits,
                                   cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out_bits, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    uint32_t grid = (n + 255) / 256;
    if (grid > 1184) grid = 1184;
    if (grid == 0) grid = 1;
    composite_max_y_kernel<<<grid, 256, 0, s>>>(xyz, surface, n, out_bits);
    return cudaGetLastError();
}

cudaError_t launch_composite_select(const float* xyz, const float* surface, uint32_t n, uint32_t k, uint32_t* work,
                                    cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(work, 0, 259 * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(work + 257, &k, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    uint32_t grid = (n + 255) / 256;
    if (grid > 1184) grid = 1184;
    if (grid == 0) grid = 1;
    for (int shift = 24; shift >= 0; shift -= 8) {
        select_hist_kernel<<<grid, 256, 0, s>>>(xyz, surface, n, work, shift);
        select_pick_kernel<<<1, 32, 0, s>>>(work, shift);
    }
    return cudaGetLastError();
}

cudaError_t launch_to_rgb8(const float* xyz, const float* surface, uint32_t n, float exposure, uint8_t* out,
                           cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    to_rgb8_kernel<<<(n + 255) / 256, 256, 0, s>>>(xyz, surface, n, exposure, out);
    return cudaGetLastError();
}

cudaError_t launch_gather_rgba8(const float* xyz, const float* surface, uint32_t w, uint32_t h, float k,
                                float kradius, float exposure, uint8_t* out, cudaStream_t s) {
    dim3 block(16, 16), grid((w + 15) / 16, (h + 15) / 16);
    gather_kernel<<<grid, block, 0, s>>>(xyz, surface, w, h, k, kradius, exposure, out);
    return cudaGetLastError();
}

cudaError_t launch_synthetic_splat(uint32_t* film, uint32_t w, uint32_t h, uint32_t seed, uint32_t n,
                                   cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    synthetic_splat_kernel<<<(n + 255) / 256, 256, 0, s>>>(film, w, h, seed, n);
    return cudaGetLastError();
}

cudaError_t launch_atomic_resolve(uint32_t* film, float* accum, size_t n, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    size_t grid = (n + 255) / 256;
    if (grid > 4096) grid = 4096;
    atomic_resolve_kernel<<<(unsigned)grid, 256, 0, s>>>(film, accum, n);
    return cudaGetLastError();
}

// Bin-averaged colour matching: for bin b of [lambda_min, lambda_max), the mean
// of the clamped table lerp over 16 sub-bin midpoints (what a photon drawn
// uniformly inside the bin would deposit on average).
void bin_weights(const float* tables, uint32_t bins, float lambda_min, float lambda_max, float* out) {
    const double width = ((double)lambda_max - (double)lambda_min) / (double)bins;
    for (uint32_t b = 0; b < bins; ++b) {
        double acc[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < 16; ++j) {
            const float nm = (float)((double)lambda_min + width * ((double)b + ((double)j + 0.5) / 16.0));
            for (int c = 0; c < 3; ++c) acc[c] += (double)tab_sample(tables + c * kTableN, nm);
        }
        for (int c = 0; c < 3; ++c) out[c * bins + b] = (float)(acc[c] / 16.0);
    }
}

Proj make_proj(const sc_camera& c) { return proj_make(c); }

}  // namespace sc
