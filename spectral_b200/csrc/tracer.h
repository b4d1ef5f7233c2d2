// Wavefront camera tracer: device structures shared by tracer.cu and the host
// object in tracer_api.cu.
#pragma once
#include "internal.h"

namespace sc {

// Everything a wave needs, kept in device memory so a captured graph stays
// valid when the camera or scene changes.
struct TracerParams {
    sc_camera cam;
    uint32_t width, height, seed, illuminant;
    float background, horizon;
    uint32_t has_horizon, max_depth, rr_start;
    uint32_t spectral;  // 1: n at the hero wavelength; 0: n(550 nm) for every path (trace.wgsl:477-480)
    f3 em_center;
    float em_radius, em_scale;
    const sc_primitive* prims; const sc_plane* planes; const sc_material* mats;
    uint32_t n_prims, n_planes, n_mats;
    const float* tables;  // device 5 x 71 sensor table
    // per primitive: a sphere (centre, radius^2) holding a bounded convex
    // solid, radius^2 = +inf where there is none (spheres, unbounded solids)
    const float4* bounds;
};

// Structure-of-arrays ray / path queue.
struct RayQueue {
    float *ox, *oy, *oz, *dx, *dy, *dz, *tp, *u;
    uint32_t *rng, *id, *flags;  // flags: valid lanes (bits 0-7), depth (bits 8-15)
};
struct TracerLaunch {
    RayQueue qa, qb;        // rays of the bounce being shaded / of the next one
    uint32_t* counts;       // max_depth + 1 queue lengths, then the tail's claim counter
    float* result;          // 3 per path of the wave
    float* sum;             // 3 * w * h running sum
    const uint32_t* d_base; // sample index of the first sample of this accumulate
    unsigned long long* segments;  // running count of traced segments
    uint32_t spp, max_depth, n_planes, grid;
    uint32_t wave_bounces;  // compacted wavefront bounces before the tail
};

// out[i] = sum[i] / count for the n floats of the running sums.
cudaError_t launch_tracer_mean(const float* sum, float* out, size_t n, float count, int sms, cudaStream_t st);
size_t tracer_dyn_smem(uint32_t n_planes);
int tracer_grid(int sms);
cudaError_t launch_tracer_wave(const TracerParams* d_params, const TracerLaunch& L, uint32_t first_pixel,
                               uint32_t n_pixels, cudaStream_t st);

}  // namespace sc
