// Batched uneven workload: many independent scenes (different photon budgets,
// film sizes and spectral bins) traced by ONE persistent launch, followed by one
// persistent drain/sensor-reduce over every film, captured in a CUDA graph.
//
// Work distribution: the host cuts every job into chunks of `chunk` photons and
// orders them largest job first; warps steal chunks from a global counter (one
// atomic per chunk).  A warp keeps its current job's parameters, scene records
// and a private dirty-tile mask in shared memory and only restages them when it
// moves to another job.  Photon i of a job is keyed by its index inside that
// job, so a batched film is bit-identical to the film of a plain per-scene launch.
#include "batch.h"

namespace sc {

namespace {

constexpr size_t kCmfBytes16 = (3 * kTableN * sizeof(float) + 15) / 16 * 16;  // warp slots start 16-aligned

struct alignas(16) WarpSlot {
    PhotonParams p;
    sc_primitive prims[kBatchPrims];
    sc_plane planes[kBatchPlanes];
    sc_material mats[kBatchPrims];
};

__device__ __forceinline__ void flush_mask(uint32_t* mask, uint32_t words, uint32_t* flags, uint32_t lane) {
    for (uint32_t w = lane; w < words; w += 32u) {
        const uint32_t v = mask[w];
        if (v) { atomicOr(flags + w, v); mask[w] = 0u; }
    }
    __syncwarp();
}

// FF: built with free-flight sampling (estimator 3) as well; jobs choose per job.
template <int AGG, int MINB, bool SPLIT, bool FF>
__global__ void __launch_bounds__(256, MINB) batch_kernel(const BatchJobDev* __restrict__ jobs,
                                                          const WorkItem* __restrict__ items, uint32_t n_items,
                                                          uint32_t* counter, const float* __restrict__ cmf_g,
                                                          uint32_t mask_words_max) {
    extern __shared__ __align__(16) unsigned char smem[];
    float* cmf = reinterpret_cast<float*>(smem);
    WarpSlot* slots = reinterpret_cast<WarpSlot*>(smem + kCmfBytes16);
    uint32_t* masks = reinterpret_cast<uint32_t*>(slots + blockDim.x / 32);
    using WS = WarpSplitSmem<kBatchWarpSegs>;
    WS* split = reinterpret_cast<WS*>(masks + (blockDim.x / 32) * mask_words_max);
    for (uint32_t i = threadIdx.x; i < 3u * kTableN; i += blockDim.x) cmf[i] = cmf_g[i];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    uint32_t* mask = masks + warp * mask_words_max;
    for (uint32_t i = threadIdx.x; i < (blockDim.x / 32) * mask_words_max; i += blockDim.x) masks[i] = 0u;
    __syncthreads();
    WarpSlot& slot = slots[warp];
    uint32_t cur = 0xFFFFFFFFu, cur_words = 0;
    uint32_t* cur_flags = nullptr;
    for (;;) {
        uint32_t it = 0;
        if (lane == 0) it = atomicAdd(counter, 1u);
        it = __shfl_sync(0xffffffffu, it, 0);
        if (it >= n_items) break;
        const WorkItem item = items[it];
        if (item.job != cur) {
            if (cur_words) flush_mask(mask, cur_words, cur_flags, lane);
            const BatchJobDev& J = jobs[item.job];
            // stage the job (params + scene records) into this warp's slot
            const uint4* src = reinterpret_cast<const uint4*>(&J.slot_image);
            uint4* dst = reinterpret_cast<uint4*>(&slot);
            for (uint32_t w = lane; w < sizeof(WarpSlot) / 16; w += 32u) dst[w] = src[w];
            cur = item.job;
            cur_words = J.mask_words <= mask_words_max ? J.mask_words : 0u;
            cur_flags = J.flags;
            __syncwarp();
        }
        SceneView S;
        S.prims = slot.prims; S.planes = slot.planes; S.mats = slot.mats; S.n_prims = slot.p.n_prims;
        if (SPLIT) {
            const uint32_t first = item.begin;
            trace_warp_range<true, AGG, FF, kBatchWarpSegs>(slot.p, S, cmf, item.count,
                                                            [first](uint32_t k) { return first + k; },
                                                            cur_words ? mask : nullptr, split[warp]);
        } else {
            const uint32_t first = item.begin;
            trace_lane_range<true, AGG, FF>(slot.p, S, cmf, lane, item.count, 32u,
                                            [first](uint32_t k) { return first + k; }, cur_words ? mask : nullptr);
        }
        __syncwarp();
    }
    if (cur_words) flush_mask(mask, cur_words, cur_flags, lane);
}

using BatchFn = void (*)(const BatchJobDev*, const WorkItem*, uint32_t, uint32_t*, const float*, uint32_t);

template <bool SPLIT>
BatchFn batch_fn_t(int agg, int minb, bool ff) {
    if (ff) return batch_kernel<0, 4, SPLIT, true>;  // batches with free-flight jobs: plain atomics, 4 CTAs per SM
    if (minb >= 5) return agg ? batch_kernel<1, 5, SPLIT, false> : batch_kernel<0, 5, SPLIT, false>;
    return agg ? batch_kernel<1, 4, SPLIT, false> : batch_kernel<0, 4, SPLIT, false>;
}
BatchFn batch_fn(int agg, int minb, int split, bool ff) {
    return split ? batch_fn_t<true>(agg, minb, ff) : batch_fn_t<false>(agg, minb, ff);
}

}  // namespace

static_assert(sizeof(WarpSlot) % 16 == 0, "warp slot must be a multiple of 16 bytes");
static_assert(sizeof(WarpSlot) == sizeof(BatchSlotImage), "slot image layout");

size_t batch_smem(uint32_t mask_words_max, int split, uint32_t block) {
    const size_t warps = block / 32u;
    return kCmfBytes16 + warps * sizeof(WarpSlot) + warps * mask_words_max * sizeof(uint32_t) +
           (split ? warps * sizeof(WarpSplitSmem<kBatchWarpSegs>) : 0);
}

int batch_occupancy(int agg, int minb, int split, uint32_t mask_words_max, uint32_t block, bool ff) {
    int n = 0;
    const void* fn = reinterpret_cast<const void*>(batch_fn(agg, minb, split, ff));
    const size_t smem = batch_smem(mask_words_max, split, block);
    if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, (int)block, smem) != cudaSuccess) return 1;
    return n > 0 ? n : 1;
}

cudaError_t launch_batch(const BatchJobDev* jobs, const WorkItem* items, uint32_t n_items, uint32_t* counter,
                         const float* cmf, uint32_t mask_words_max, int agg, int minb, int split, uint32_t grid,
                         cudaStream_t s, uint32_t block, bool ff) {
    // the shared-memory attribute was raised by batch_occupancy before any capture
    const size_t smem = batch_smem(mask_words_max, split, block);
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    batch_fn(agg, minb, split, ff)<<<grid, block, smem, s>>>(jobs, items, n_items, counter, cmf, mask_words_max);
    return cudaGetLastError();
}

}  // namespace sc
