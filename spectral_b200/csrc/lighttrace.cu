// Screen-caustic forward light tracer and the scene z-buffer.
//
// Light tracer: one thread per photon restating lighttrace::trace /
// trace_photon / Screen::splat (spectral-core/src/lighttrace.rs:75-166): the
// photon leaves the beam aperture with a wavelength drawn from the band, and at
// every bounce the nearer of the scene hit and the screen rectangle wins; a
// photon that reaches the screen deposits cmf(lambda) * power bilinearly into
// the four surrounding texels of a 64-bit fixed-point XYZ screen film.
//
// Z-buffer: the euclidean distance to the nearest surface along each pixel's
// primary ray, INF where nothing is hit (the z-buffer pass of
// spectral-core/examples/prism_on_plane.rs:125-160), as input to the haze film.
#include "host_util.h"
#include "internal.h"

namespace sc {

namespace {

// Screen rectangle with its normal and the squared edge lengths.
struct ScreenView {
    f3 corner, u, v, normal;
    float uu, vv;
};

ScreenView make_screen(const sc_screen& s) {
    ScreenView v;
    v.corner = ld3(s.corner); v.u = ld3(s.u); v.v = ld3(s.v);
    v.normal = normalize(cross(v.u, v.v));  // Screen::new (lighttrace.rs:27-34)
    v.uu = dot(v.u, v.u); v.vv = dot(v.v, v.v);
    return v;
}

// Screen::screen_coords (lighttrace.rs:42-62): ray parameter of the rectangle
// hit, +INF on a miss; (s, r) in [0,1) on a hit.
__device__ __forceinline__ float screen_coords(const ScreenView& S, f3 o, f3 d, float& s, float& r) {
    const float inf = __int_as_float(0x7f800000);
    const float denom = dot(d, S.normal);
    if (fabsf(denom) < 1e-8f) return inf;
    const float t = dot(sub(S.corner, o), S.normal) / denom;
    if (t <= 1e-4f) return inf;
    const f3 rel = sub(add(o, mul(d, t)), S.corner);
    const float ss = dot(rel, S.u) / S.uu;
    const float rv = dot(rel, S.v) / S.vv;
    if (!(ss >= 0.0f && ss < 1.0f && rv >= 0.0f && rv < 1.0f)) return inf;
    s = ss;
    r = rv;
    return t;
}

struct LightParams {
    f3 corner, bu, bv, bdir;
    ScreenView scr;
    uint32_t width, height, seed, max_bounces, photon_count, spectral;
    float lambda_min, lambda_range, scale;
    const sc_primitive* prims; const sc_plane* planes; const sc_material* mats;
    uint32_t n_prims, n_planes, n_mats;
    const float* cmf;
    unsigned long long* film;  // row-major [h][w][3]
};

__global__ void __launch_bounds__(256) lighttrace_kernel(const LightParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    sc_primitive* sp = reinterpret_cast<sc_primitive*>(smem);
    sc_plane* spl = reinterpret_cast<sc_plane*>(sp + p.n_prims);
    sc_material* sm = reinterpret_cast<sc_material*>(spl + p.n_planes);
    float* cmf = reinterpret_cast<float*>(sm + p.n_mats);
    for (uint32_t i = threadIdx.x; i < p.n_prims; i += blockDim.x) sp[i] = p.prims[i];
    for (uint32_t i = threadIdx.x; i < p.n_planes; i += blockDim.x) spl[i] = p.planes[i];
    for (uint32_t i = threadIdx.x; i < p.n_mats; i += blockDim.x) sm[i] = p.mats[i];
    for (uint32_t i = threadIdx.x; i < 3u * kTableN; i += blockDim.x) cmf[i] = p.cmf[i];
    __syncthreads();
    SceneView S;
    S.prims = sp; S.planes = spl; S.mats = sm; S.n_prims = p.n_prims;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < p.photon_count; idx += gridDim.x * blockDim.x) {
        Rng r = Rng::make(idx, p.seed);
        const float r1 = r.f32();
        const float r2 = r.f32();
        f3 o = add(add(p.corner, mul(p.bu, r1)), mul(p.bv, r2));
        const float lambda = p.lambda_min + p.lambda_range * r.f32();
        f3 d = p.bdir;
        float power = 1.0f;
        bool landed = false;
        float ls = 0.0f, lr = 0.0f;
        for (uint32_t b = 0; b < p.max_bounces; ++b) {
            Hit h;
            uint32_t mi = 0;
            const bool any = scene_hit(S, o, d, h, mi);
            const float scene_t = any ? h.t : __int_as_float(0x7f800000);
            float ss = 0.0f, rr = 0.0f;
            const float screen_t = screen_coords(p.scr, o, d, ss, rr);
            if (screen_t < scene_t) { landed = true; ls = ss; lr = rr; break; }
            if (!any) break;
            const sc_material& m = S.mats[mi];
            const float nh = m.kind == 1u ? glass_n(m.glass, p.spectral ? lambda : 550.0f) : 1.0f;
            f3 nd;
            float w;
            scatter(m, d, h, nh, r, nd, w);
            power *= w;
            o = h.point;
            d = nd;
        }
        if (!landed) continue;
        // Screen::splat with texel_bilinear (lighttrace.rs:67-91)
        const float cx = tab_sample(cmf, lambda), cy = tab_sample(cmf + kTableN, lambda),
                    cz = tab_sample(cmf + 2 * kTableN, lambda);
        const float fx = fminf(fmaxf(ls * (float)p.width - 0.5f, 0.0f), (float)p.width - 1.0f);
        const float fy = fminf(fmaxf((1.0f - lr) * (float)p.height - 0.5f, 0.0f), (float)p.height - 1.0f);
        const uint32_t x0 = (uint32_t)floorf(fx), y0 = (uint32_t)floorf(fy);
        const uint32_t x1 = min(x0 + 1u, p.width - 1u), y1 = min(y0 + 1u, p.height - 1u);
        const float dx = fx - (float)x0, dy = fy - (float)y0;
        const uint32_t xs[4] = {x0, x1, x0, x1}, ys[4] = {y0, y0, y1, y1};
        const float ws[4] = {(1.0f - dx) * (1.0f - dy), dx * (1.0f - dy), (1.0f - dx) * dy, dx * dy};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            unsigned long long* c = p.film + ((size_t)ys[q] * p.width + xs[q]) * 3u;
            const unsigned long long vx = to_fixed(cx * power * ws[q], p.scale);
            const unsigned long long vy = to_fixed(cy * power * ws[q], p.scale);
            const unsigned long long vz = to_fixed(cz * power * ws[q], p.scale);
            if (vx) atomicAdd(c, vx);
            if (vy) atomicAdd(c + 1, vy);
            if (vz) atomicAdd(c + 2, vz);
        }
    }
}

__global__ void film_to_f32_kernel(const unsigned long long* film, float* out, size_t n, double inv_scale) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (float)((double)(long long)film[i] * inv_scale);
}

__global__ void __launch_bounds__(256) zbuffer_kernel(sc_camera cam, uint32_t w, uint32_t h,
                                                      const sc_primitive* prims, const sc_plane* planes,
                                                      const sc_material* mats, uint32_t n_prims, uint32_t n_planes,
                                                      uint32_t n_mats, ScreenView floor, int has_floor,
                                                      float* out) {
    extern __shared__ __align__(16) unsigned char smem[];
    sc_primitive* sp = reinterpret_cast<sc_primitive*>(smem);
    sc_plane* spl = reinterpret_cast<sc_plane*>(sp + n_prims);
    sc_material* sm = reinterpret_cast<sc_material*>(spl + n_planes);
    const uint32_t tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (uint32_t i = tid; i < n_prims; i += nt) sp[i] = prims[i];
    for (uint32_t i = tid; i < n_planes; i += nt) spl[i] = planes[i];
    for (uint32_t i = tid; i < n_mats; i += nt) sm[i] = mats[i];
    __syncthreads();
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
    if (px >= w || py >= h) return;
    SceneView S;
    S.prims = sp; S.planes = spl; S.mats = sm; S.n_prims = n_prims;
    const float s = ((float)px + 0.5f) / (float)w;
    const float t = 1.0f - ((float)py + 0.5f) / (float)h;
    Hit hit;
    uint32_t mi;
    const f3 o = ld3(cam.origin), d = primary_dir(cam, s, t);
    const float t_scene = scene_hit(S, o, d, hit, mi) ? hit.t : __int_as_float(0x7f800000);
    float fs, fr, t_floor = __int_as_float(0x7f800000);
    if (has_floor) t_floor = screen_coords(floor, o, d, fs, fr);
    out[(size_t)py * w + px] = t_scene < t_floor ? t_scene : t_floor;
}

int upload_scene(const sc_primitive* prims, uint32_t np, const sc_plane* planes, uint32_t npl,
                 const sc_material* mats, uint32_t nm, DevBuf<sc_primitive>& dp, DevBuf<sc_plane>& dpl,
                 DevBuf<sc_material>& dm) {
    const int rc = check_scene(np, npl, nm, prims, planes, mats);
    if (rc != SC_OK) return rc;
    SC_CUDA(dp.alloc(np ? np : 1));
    SC_CUDA(dpl.alloc(npl ? npl : 1));
    SC_CUDA(dm.alloc(nm ? nm : 1));
    if (np) SC_CUDA(cudaMemcpy(dp.p, prims, np * sizeof(sc_primitive), cudaMemcpyHostToDevice));
    if (npl) SC_CUDA(cudaMemcpy(dpl.p, planes, npl * sizeof(sc_plane), cudaMemcpyHostToDevice));
    if (nm) SC_CUDA(cudaMemcpy(dm.p, mats, nm * sizeof(sc_material), cudaMemcpyHostToDevice));
    return SC_OK;
}

}  // namespace

}  // namespace sc

using namespace sc;

extern "C" {

int sc_lighttrace(sc_ctx* ctx, const sc_primitive* prims, uint32_t n_prims, const sc_plane* planes, uint32_t n_planes,
                  const sc_material* mats, uint32_t n_mats, const sc_screen* screen, uint32_t width, uint32_t height,
                  const sc_beam* beam, uint32_t n_photons, uint32_t seed, const sc_film_options* opts,
                  float* out_sum) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && screen && beam && out_sum, SC_E_INVALID, "null argument");
    SC_REQUIRE(width > 0 && height > 0 && (uint64_t)width * height <= (1ull << 28), SC_E_INVALID, "screen %ux%u",
               width, height);
    sc_film_options o{};
    if (opts) o = *opts;
    if (o.lambda_min == 0.0f) o.lambda_min = 380.0f;
    if (o.lambda_max == 0.0f) o.lambda_max = 730.0f;
    if (o.max_bounces == 0u) o.max_bounces = 8u;
    if (o.scale_log2 == 0u) o.scale_log2 = 32u;
    SC_REQUIRE(o.lambda_max > o.lambda_min && o.scale_log2 <= 50u && o.max_bounces <= 64u, SC_E_INVALID,
               "bad options");
    DeviceGuard g(ctx->device);
    DevBuf<sc_primitive> dp;
    DevBuf<sc_plane> dpl;
    DevBuf<sc_material> dm;
    int rc = upload_scene(prims, n_prims, planes, n_planes, mats, n_mats, dp, dpl, dm);
    if (rc != SC_OK) return rc;
    const size_t n = 3ull * width * height;
    DevBuf<unsigned long long> film;
    DevBuf<float> out;
    SC_CUDA(film.alloc(n));
    SC_CUDA(out.alloc(n));
    SC_CUDA(cudaMemset(film.p, 0, film.bytes()));
    LightParams p;
    std::memset(&p, 0, sizeof p);
    p.corner = ld3(beam->corner); p.bu = ld3(beam->u); p.bv = ld3(beam->v); p.bdir = ld3(beam->dir);
    p.scr = make_screen(*screen);
    p.width = width; p.height = height; p.seed = seed; p.max_bounces = o.max_bounces; p.photon_count = n_photons;
    p.spectral = 1; p.lambda_min = o.lambda_min; p.lambda_range = o.lambda_max - o.lambda_min;
    p.scale = std::ldexp(1.0f, (int)o.scale_log2);
    p.prims = dp.p; p.planes = dpl.p; p.mats = dm.p; p.n_prims = n_prims; p.n_planes = n_planes; p.n_mats = n_mats;
    p.cmf = ctx->cmf.p;
    p.film = film.p;
    if (n_photons) {
        const size_t smem = n_prims * sizeof(sc_primitive) + n_planes * sizeof(sc_plane) +
                            n_mats * sizeof(sc_material) + 3 * kTableN * sizeof(float);
        uint32_t grid = (n_photons + 255u) / 256u;
        const uint32_t cap = (uint32_t)ctx->sms * 8u;
        lighttrace_kernel<<<grid < cap ? grid : cap, 256, smem>>>(p);
        SC_CUDA(cudaGetLastError());
    }
    film_to_f32_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256>>>(film.p, out.p, n,
                                                                                   std::ldexp(1.0, -(int)o.scale_log2));
    SC_CUDA(cudaGetLastError());
    SC_CUDA(cudaMemcpy(out_sum, out.p, n * sizeof(float), cudaMemcpyDeviceToHost));
    return SC_OK;
    SC_GUARD_END
}

int sc_scene_zbuffer(sc_ctx* ctx, const sc_primitive* prims, uint32_t n_prims, const sc_plane* planes,
                     uint32_t n_planes, const sc_material* mats, uint32_t n_mats, const sc_screen* floor,
                     const sc_camera* cam, uint32_t width, uint32_t height, float* out) {
    SC_GUARD_BEGIN
    SC_REQUIRE(ctx && cam && out, SC_E_INVALID, "null argument");
    SC_REQUIRE(width > 0 && height > 0 && (uint64_t)width * height <= (1ull << 28), SC_E_INVALID, "image %ux%u",
               width, height);
    DeviceGuard g(ctx->device);
    DevBuf<sc_primitive> dp;
    DevBuf<sc_plane> dpl;
    DevBuf<sc_material> dm;
    int rc = upload_scene(prims, n_prims, planes, n_planes, mats, n_mats, dp, dpl, dm);
    if (rc != SC_OK) return rc;
    DevBuf<float> z;
    SC_CUDA(z.alloc((size_t)width * height));
    const size_t smem = n_prims * sizeof(sc_primitive) + n_planes * sizeof(sc_plane) + n_mats * sizeof(sc_material);
    dim3 block(16, 16), grid((width + 15) / 16, (height + 15) / 16);
    ScreenView fv;
    std::memset(&fv, 0, sizeof fv);
    if (floor) fv = make_screen(*floor);
    zbuffer_kernel<<<grid, block, smem>>>(*cam, width, height, dp.p, dpl.p, dm.p, n_prims, n_planes, n_mats, fv,
                                          floor ? 1 : 0, z.p);
    SC_CUDA(cudaGetLastError());
    SC_CUDA(cudaMemcpy(out, z.p, z.bytes(), cudaMemcpyDeviceToHost));
    return SC_OK;
    SC_GUARD_END
}

}  // extern "C"
