// Host-side sky-bin bookkeeping and the traced direction table.
//
// Both follow the reference host code value for value, because the shadow
// bits and neighbor ids must be bit-identical:
//   * sky bins: src/sky_bins.cpp:9-52 (5 deg x 5 deg bins, 1e-8 nudge, dense
//     index of sun-visited upper bins, per-hour dense index, alt >= 1 gate);
//   * directions: include/cuda/viewshed_stage.cuh:64-80 (bin centres, i-major
//     over 72 azimuths, j-minor over 18 upper then 18 lower elevations,
//     float cosf/sinf, normalised).
// Compiled with -ffp-contract=off so no product is fused on the host.
//
// Each upper direction also names the early-exit table of its cone (cone.cu):
// its quadrant and the two consecutive vectors of the Farey set of order
// kConeOrder between which its unsigned step vector (1/dX, 1/dY) lies.
#include "sky.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <tuple>

namespace sgb {

namespace {
constexpr float kDegToRad = 0.0174532925f;   // include/pipeline_math_constants.h:15

// Primitive vectors (p, q), 0 <= p, q <= n, by angle from (1, 0) to (0, 1);
// consecutive ones have determinant 1.
std::vector<std::pair<int, int>> farey_vectors(int n)
{
    std::vector<std::pair<int, int>> v;
    for (int p = 0; p <= n; ++p)
        for (int q = 0; q <= n; ++q)
            if ((p || q) && std::gcd(p, q) == 1) v.emplace_back(p, q);
    std::sort(v.begin(), v.end(), [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
        return (long long)a.first * b.second - (long long)a.second * b.first > 0;
    });
    return v;
}

// Index of the cone (F[k], F[k + 1]) holding the direction (dY, dX), which
// is proportional to (1/dX, 1/dY).  The cross products of small integers
// with floats are exact in double and so are their signs.
int cone_of(const std::vector<std::pair<int, int>>& F, float dX, float dY)
{
    for (size_t k = 0; k + 1 < F.size(); ++k) {
        const double a = (double)F[k].first * dX - (double)F[k].second * dY;             // det(F[k], v)
        const double b = (double)dY * F[k + 1].second - (double)dX * F[k + 1].first;     // det(v, F[k+1])
        if (a >= 0.0 && b >= 0.0) return (int)k;
    }
    return -1;
}
}

SkyTables make_sky_tables(const float* sun_az_alt, float h_res, float v_res)
{
    SkyTables t;
    t.hsize = (int)std::ceil(360.0f / h_res);
    t.vsize = (int)std::ceil(90.0f / v_res);
    t.vsize_full = 2 * t.vsize;
    t.nudged.resize(2 * (size_t)kHoursPerYear);
    std::vector<unsigned char> used((size_t)t.hsize * t.vsize, 0);
    for (int k = 0; k < kHoursPerYear; ++k) {
        const float az = sun_az_alt[2 * k] - 1e-8f;
        const float alt = sun_az_alt[2 * k + 1] - 1e-8f;
        t.nudged[2 * k] = az;
        t.nudged[2 * k + 1] = alt;
        if (alt < 1.0f) continue;
        const unsigned bi = (unsigned)(az / h_res);
        const unsigned bj = (unsigned)(alt / v_res);
        if (bi < (unsigned)t.hsize && bj < (unsigned)t.vsize) used[bi * t.vsize + bj] = 1;
    }
    t.full_to_dense.assign((size_t)t.hsize * t.vsize, -1);
    t.active = 0;
    for (int i = 0; i < t.hsize; ++i)
        for (int j = 0; j < t.vsize; ++j)
            if (used[(size_t)i * t.vsize + j]) t.full_to_dense[(size_t)i * t.vsize + j] = t.active++;
    t.words32 = (t.active + 31) / 32;
    t.sun_dense.resize(kHoursPerYear);
    for (int k = 0; k < kHoursPerYear; ++k) {
        const float az = t.nudged[2 * k], alt = t.nudged[2 * k + 1];
        if (alt < 1.0f) { t.sun_dense[k] = -1; continue; }
        t.hour_index.push_back(k);   // daylight gate of gpu_irradiance_uncompressed.cu:117
        const unsigned bi = (unsigned)(az / h_res);
        const unsigned bj = (unsigned)(alt / v_res);
        t.sun_dense[k] = (bi < (unsigned)t.hsize && bj < (unsigned)t.vsize)
                             ? t.full_to_dense[bi * t.vsize + bj] : -1;
    }

    const int D = t.hsize * t.vsize_full;
    t.dirs.resize(D);
    for (unsigned i = 0; i < (unsigned)t.hsize; ++i) {
        for (unsigned j = 0; j < (unsigned)t.vsize_full; ++j) {
            float cx, cy, cz;
            int upper, dense = -1;
            if (j < (unsigned)t.vsize) {
                const float e = (j + 0.5f) * v_res;
                cx = cosf(e * kDegToRad) * sinf(((i + 0.5f) * h_res) * kDegToRad);
                cy = -cosf(e * kDegToRad) * cosf(((i + 0.5f) * h_res) * kDegToRad);
                cz = sinf(e * kDegToRad);
                upper = 1;
                dense = t.full_to_dense[i * (unsigned)t.vsize + j];
            } else {
                const float e = (j - (unsigned)t.vsize + 0.5f) * v_res;
                cx = cosf(e * kDegToRad) * sinf(((i + 0.5f) * h_res) * kDegToRad);
                cy = -cosf(e * kDegToRad) * cosf(((i + 0.5f) * h_res) * kDegToRad);
                cz = -sinf(e * kDegToRad);
                upper = 0;
            }
            const float len = sqrtf(cx * cx + cy * cy + cz * cz);
            if (len > 0.0f) { cx /= len; cy /= len; cz /= len; }
            DirEntry& d = t.dirs[(size_t)i * t.vsize_full + j];
            d.cx = cx; d.cy = cy; d.cz = cz;
            d.ax = fmaxf(fabsf(cx), 1e-8f);
            d.ay = fmaxf(fabsf(cy), 1e-8f);
            d.dX = 1.0f / d.ax;
            d.dY = 1.0f / d.ay;
            d.meta = ((dense + 1) & 0xFFFF) | (upper << 16);
        }
    }

    // Every upper direction gets a table, or none does (the tracer then uses
    // one table whose bound is maxz for all of them).
    const std::vector<std::pair<int, int>> F = farey_vectors(kConeOrder);
    bool ok = true;
    for (size_t k = 0; k + 1 < F.size(); ++k)
        ok = ok && (long long)F[k].first * F[k + 1].second - (long long)F[k].second * F[k + 1].first == 1;
    std::map<std::tuple<int, int, int>, int> table_of;
    std::vector<int> table(t.dirs.size(), 0);
    for (size_t i = 0; ok && i < t.dirs.size(); ++i) {
        const DirEntry& d = t.dirs[i];
        if (!((d.meta >> 16) & 1)) continue;
        const int sx = d.cx >= 0.0f ? 1 : -1, sy = d.cy >= 0.0f ? 1 : -1;
        const int k = cone_of(F, d.dX, d.dY);
        if (k < 0) { ok = false; break; }   // not reached: the cones cover the quadrant
        const auto key = std::make_tuple(sx, sy, k);
        auto it = table_of.find(key);
        if (it == table_of.end()) {
            if ((int)t.cones.size() >= kMaxConeTables) { ok = false; break; }
            it = table_of.emplace(key, (int)t.cones.size()).first;
            t.cones.push_back({sx, sy, F[k].first, F[k].second, F[k + 1].first, F[k + 1].second});
        }
        table[i] = it->second;
    }
    if (!ok) t.cones.clear();
    else
        for (size_t i = 0; i < t.dirs.size(); ++i) t.dirs[i].meta |= table[i] << 17;
    return t;
}

}  // namespace sgb
