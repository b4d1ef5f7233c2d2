// CPU check of sc::solid_bound (spectral_b200/csrc/solid_bound.h), built and run
// by tests/test_solid_bounds.py.  Prints one line per failed case and "ok".
#include <cstdio>
#include <random>

#include "solid_bound.h"

static int failures = 0;

static void expect(bool cond, const char* what) {
    if (!cond) {
        std::printf("FAIL %s\n", what);
        ++failures;
    }
}

static bool unbounded(const float b[4]) { return !(b[3] < std::numeric_limits<float>::infinity()); }

// Every point of the solid that a dense sample of the cube [lo, hi]^3 around
// the sphere's centre (offsets) finds lies in the sphere.
static bool contains_samples(const std::vector<sc_plane>& pl, const float b[4], double lo, double hi, std::mt19937& rng,
                             int n, bool around_centre = false) {
    std::uniform_real_distribution<double> u(lo, hi);
    for (int k = 0; k < n; ++k) {
        double x[3] = {u(rng), u(rng), u(rng)};
        if (around_centre)
            for (int q = 0; q < 3; ++q) x[q] += b[q];
        bool inside = true;
        for (const sc_plane& p : pl)
            inside = inside && p.normal[0] * x[0] + p.normal[1] * x[1] + p.normal[2] * x[2] + p.d <= 0.0;
        if (!inside) continue;
        const double dx = x[0] - b[0], dy = x[1] - b[1], dz = x[2] - b[2];
        if (dx * dx + dy * dy + dz * dz > (double)b[3]) return false;
    }
    return true;
}

int main() {
    std::mt19937 rng(12345);
    float b[4];
    // unit cube [-1, 1]^3: centre 0, radius sqrt(3) * 1.01 + 1e-3
    std::vector<sc_plane> cube = {{{1, 0, 0}, -1}, {{-1, 0, 0}, -1}, {{0, 1, 0}, -1},
                                  {{0, -1, 0}, -1}, {{0, 0, 1}, -1}, {{0, 0, -1}, -1}};
    sc::solid_bound(cube.data(), 6, b);
    const double r = std::sqrt(3.0) * 1.01 + 1e-3;
    expect(std::fabs(b[0]) < 1e-6 && std::fabs(b[1]) < 1e-6 && std::fabs(b[2]) < 1e-6, "cube centre");
    expect(std::fabs(std::sqrt((double)b[3]) - r) < 1e-5, "cube radius");
    // the cube without its top: unbounded
    sc::solid_bound(cube.data(), 5, b);
    expect(unbounded(b), "open box is unbounded");
    // fewer than 4 planes, a half-space, a slab: unbounded
    sc::solid_bound(cube.data(), 1, b);
    expect(unbounded(b), "half-space is unbounded");
    std::vector<sc_plane> slab = {{{0, 0, 1}, -1}, {{0, 0, -1}, -1}, {{0, 0, 1}, -2}, {{0, 0, -1}, -2}};
    sc::solid_bound(slab.data(), 4, b);
    expect(unbounded(b), "parallel planes are unbounded");
    // a triangular prism without caps is unbounded along its axis; with caps bounded
    const double s3 = std::sqrt(3.0) / 2.0;
    std::vector<sc_plane> prism = {{{0, -1, 0}, -1}, {{(float)s3, 0.5f, 0}, -1}, {{(float)-s3, 0.5f, 0}, -1},
                                   {{0, 0, 1}, -0.5f}, {{0, 0, -1}, -0.5f}};
    sc::solid_bound(prism.data(), 4, b);
    expect(unbounded(b), "prism with one cap is unbounded");
    sc::solid_bound(prism.data(), 5, b);
    expect(!unbounded(b) && contains_samples(prism, b, -3, 3, rng, 200000), "capped prism inside its sphere");
    // a tetrahedron (vertices 0, e_x, e_y, e_z)
    std::vector<sc_plane> tet = {{{0, 0, -1}, 0}, {{0, -1, 0}, 0}, {{-1, 0, 0}, 0},
                                 {{0.57735027f, 0.57735027f, 0.57735027f}, -0.57735027f}};
    sc::solid_bound(tet.data(), 4, b);
    expect(!unbounded(b) && std::fabs(b[0] - 0.25f) < 1e-5 && contains_samples(tet, b, -0.5, 1.5, rng, 200000),
           "tetrahedron");
    // random polytopes: half-spaces tangent to a sphere of radius 0.5 around a
    // random centre; bounded ones hold every sampled interior point
    std::normal_distribution<double> g(0.0, 1.0);
    std::uniform_real_distribution<double> uc(-2.0, 2.0);
    int bounded_seen = 0, unbounded_seen = 0;
    for (int trial = 0; trial < 300; ++trial) {
        const int k = 4 + trial % 12;
        const double c[3] = {uc(rng), uc(rng), uc(rng)};
        const bool hemi = trial % 5 == 0;  // every normal with n_z > 0: unbounded towards -z
        std::vector<sc_plane> pl;
        for (int i = 0; i < k; ++i) {
            double n[3] = {g(rng), g(rng), g(rng)};
            const double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            for (double& v : n) v /= l;
            if (hemi && n[2] < 0) n[2] = -n[2];
            const float nf[3] = {(float)n[0], (float)n[1], (float)n[2]};
            pl.push_back({{nf[0], nf[1], nf[2]}, (float)(-0.5 - (nf[0] * c[0] + nf[1] * c[1] + nf[2] * c[2]))});
        }
        sc::solid_bound(pl.data(), (uint32_t)pl.size(), b);
        if (hemi) {
            expect(unbounded(b), "normals in one hemisphere: unbounded");
            ++unbounded_seen;
            continue;
        }
        if (unbounded(b)) { ++unbounded_seen; continue; }  // never wrong, only less culling
        ++bounded_seen;
        char what[64];
        std::snprintf(what, sizeof what, "random polytope %d inside its sphere", trial);
        const double reach = 3.0 * std::sqrt((double)b[3]);  // a missed vertex would leave points out here
        expect(contains_samples(pl, b, -reach, reach, rng, 50000, true), what);
    }
    expect(bounded_seen > 100, "enough bounded random polytopes");
    std::printf("bounded %d unbounded %d\n", bounded_seen, unbounded_seen);
    if (failures == 0) std::printf("ok\n");
    return failures == 0 ? 0 : 1;
}
