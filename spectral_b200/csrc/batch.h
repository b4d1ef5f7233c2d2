// Batched uneven workload: device structures shared by batch.cu (kernel) and
// batch_api.cu (host object).
#pragma once
#include "photon_trace.cuh"

namespace sc {

constexpr uint32_t kBatchPrims = 4;
constexpr uint32_t kBatchPlanes = 16;
// Per-warp dirty masks up to this many words live in shared memory (a 1024x1024
// film has 16384 tiles = 512 words); larger films mark their tiles with red.or.
constexpr uint32_t kBatchMaskWords = 512;

// What one warp stages for its current job (byte image copied as 16-byte words).
struct alignas(16) BatchSlotImage {
    PhotonParams p;
    sc_primitive prims[kBatchPrims];
    sc_plane planes[kBatchPlanes];
    sc_material mats[kBatchPrims];
};

struct alignas(16) BatchJobDev {
    BatchSlotImage slot_image;
    uint32_t* flags;
    uint32_t mask_words;
};

struct WorkItem { uint32_t job, begin, count; };

// `block`: threads per CTA, 128 or 256 (one shared-memory job slot per warp).
// `ff`: some job uses free-flight sampling (the kernel built with it).
size_t batch_smem(uint32_t mask_words_max, int split, uint32_t block = 256);
int batch_occupancy(int agg, int minb, int split, uint32_t mask_words_max, uint32_t block = 256, bool ff = false);
cudaError_t launch_batch(const BatchJobDev* jobs, const WorkItem* items, uint32_t n_items, uint32_t* counter,
                         const float* cmf, uint32_t mask_words_max, int agg, int minb, int split, uint32_t grid,
                         cudaStream_t s, uint32_t block = 256, bool ff = false);

}  // namespace sc
