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
#include "sky.h"

#include <cmath>

namespace sgb {

namespace {
constexpr float kDegToRad = 0.0174532925f;   // include/pipeline_math_constants.h:15
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
    return t;
}

}  // namespace sgb
