// Host-side bounding sphere of a convex solid (the camera tracer uses it to
// skip the plane tests of solids a ray cannot hit).  Header-only so that a CPU
// test can compile it on its own.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

#include "spectral_cuda.h"

namespace sc {

// A sphere holding the convex solid {x : n_i . x + d_i <= 0} of `n` planes, as
// (centre, radius^2), or radius^2 = +inf when the solid is unbounded (or has
// fewer than 4 planes).  Unbounded: some direction u = +-(n_i x n_j) has
// n_k . u <= 1e-6 |n_k| |u| for every k (an edge direction of the recession
// cone, which a bounded solid does not have; the tolerance errs towards
// "unbounded").  Otherwise the solid is the hull of its vertices (the
// intersections of three planes that lie inside all, with a loose tolerance
// that can only add points), and the sphere around their centroid through the
// farthest one is inflated by 1 % + 1e-3.
inline void solid_bound(const sc_plane* pl, uint32_t n, float out[4]) {
    out[0] = out[1] = out[2] = 0.0f;
    out[3] = std::numeric_limits<float>::infinity();
    if (n < 4) return;
    auto nv = [&](uint32_t i, int c) { return (double)pl[i].normal[c]; };
    auto norm3 = [](const double v[3]) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); };
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = i + 1; j < n; ++j) {
            const double u[3] = {nv(i, 1) * nv(j, 2) - nv(i, 2) * nv(j, 1), nv(i, 2) * nv(j, 0) - nv(i, 0) * nv(j, 2),
                                 nv(i, 0) * nv(j, 1) - nv(i, 1) * nv(j, 0)};
            const double lu = norm3(u);
            const double ni[3] = {nv(i, 0), nv(i, 1), nv(i, 2)}, nj[3] = {nv(j, 0), nv(j, 1), nv(j, 2)};
            if (!(lu > 1e-9 * norm3(ni) * norm3(nj))) continue;  // parallel planes: no edge direction
            for (int sgn = -1; sgn <= 1; sgn += 2) {
                bool recedes = true;
                for (uint32_t k = 0; k < n && recedes; ++k) {
                    const double nk[3] = {nv(k, 0), nv(k, 1), nv(k, 2)};
                    const double dotku = sgn * (nk[0] * u[0] + nk[1] * u[1] + nk[2] * u[2]);
                    recedes = dotku <= 1e-6 * norm3(nk) * lu;
                }
                if (recedes) return;
            }
        }
    std::vector<std::array<double, 3>> verts;
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = i + 1; j < n; ++j)
            for (uint32_t k = j + 1; k < n; ++k) {
                const double a[3][3] = {{nv(i, 0), nv(i, 1), nv(i, 2)}, {nv(j, 0), nv(j, 1), nv(j, 2)},
                                        {nv(k, 0), nv(k, 1), nv(k, 2)}};
                const double b[3] = {-(double)pl[i].d, -(double)pl[j].d, -(double)pl[k].d};
                const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                                   a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                                   a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
                if (std::fabs(det) < 1e-12) continue;
                double x[3];
                for (int c = 0; c < 3; ++c) {  // Cramer's rule
                    double m[3][3];
                    for (int r = 0; r < 3; ++r)
                        for (int q = 0; q < 3; ++q) m[r][q] = q == c ? b[r] : a[r][q];
                    x[c] = (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                            m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                            m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0])) / det;
                }
                bool inside = true;
                for (uint32_t m = 0; m < n && inside; ++m)
                    inside = nv(m, 0) * x[0] + nv(m, 1) * x[1] + nv(m, 2) * x[2] + pl[m].d <=
                             1e-4 * (1.0 + norm3(x));
                if (inside) verts.push_back({x[0], x[1], x[2]});
            }
    if (verts.empty()) return;
    double c[3] = {0, 0, 0};
    for (const auto& v : verts)
        for (int q = 0; q < 3; ++q) c[q] += v[q] / (double)verts.size();
    double r2 = 0.0;
    for (const auto& v : verts)
        r2 = std::max(r2, (v[0] - c[0]) * (v[0] - c[0]) + (v[1] - c[1]) * (v[1] - c[1]) + (v[2] - c[2]) * (v[2] - c[2]));
    const double r = std::sqrt(r2) * 1.01 + 1e-3;
    out[0] = (float)c[0]; out[1] = (float)c[1]; out[2] = (float)c[2];
    out[3] = (float)(r * r);
}

}  // namespace sc
