// Test infrastructure: extern "C" entry points over the reference's own host
// code (ba-RLE encoder, sky bins, voxelization), compiled from the reference
// sources where they lie.  Used only to pin the oracle's restatement and to
// generate golden fixtures; never linked into the product.
#include <cstring>
#include <vector>

#include "barle_compression.h"
#include "sky_bins.h"
#include "sun_position.h"
#include "voxelization.h"

extern "C" {

// src/barle_compression.cpp:156-187 for one zero-terminated list.
int ref_barle_compress(const int* raw, int max_neighbors, unsigned char* out, int cap)
{
    int raw_bytes = 0;
    std::vector<solar_gpu::barle::Byte> v =
        solar_gpu::barle::compress_voxel_neighbors(raw, max_neighbors, raw_bytes);
    if ((int)v.size() > cap) return -1;
    if (!v.empty()) std::memcpy(out, v.data(), v.size());
    return (int)v.size();
}

// src/sky_bins.cpp:9-52 with the default 5 deg / 5 deg bins.
int ref_sky_bins(const float* sun_az_alt, int* full_to_dense, int* sun_dense_idx,
                 float* nudged, int* meta)
{
    std::vector<solar_gpu::SunSample> sun(solar_gpu::kHoursPerYear);
    for (int k = 0; k < solar_gpu::kHoursPerYear; ++k)
        sun[k] = solar_gpu::SunSample(sun_az_alt[2 * k], sun_az_alt[2 * k + 1]);
    solar_gpu::SkyBins b = solar_gpu::compute_sky_bins(sun);
    for (size_t i = 0; i < b.full_to_dense.size(); ++i) full_to_dense[i] = b.full_to_dense[i];
    for (int k = 0; k < solar_gpu::kHoursPerYear; ++k) {
        sun_dense_idx[k] = b.sun_dense_idx[k];
        nudged[2 * k] = std::get<0>(b.sun_azm_alt[k]);
        nudged[2 * k + 1] = std::get<1>(b.sun_azm_alt[k]);
    }
    meta[0] = (int)b.h_hsize;
    meta[1] = (int)b.h_vsize;
    meta[2] = (int)b.h_vsize_full;
    meta[3] = (int)b.active_bin_count;
    meta[4] = (int)b.hgrid_size_s;
    return 0;
}

// src/voxelization.cpp:10-64.  Returns the wall count (or -1 if cap is short).
int ref_detect_walls(const float* heights, int W, int H, float voxel_size,
                     int* parent, float* z, float* aspect, int cap)
{
    solar_gpu::HeightGrid g;
    g.width = W;
    g.height = H;
    g.scaleX = g.scaleY = voxel_size;
    g.heights.assign(heights, heights + (size_t)W * H);
    std::vector<solar_gpu::WallVoxel> w = solar_gpu::detect_wall_voxels(g, voxel_size);
    if ((int)w.size() > cap) return -1;
    for (size_t i = 0; i < w.size(); ++i) {
        parent[i] = w[i].parentIdx;
        z[i] = w[i].z;
        aspect[i] = w[i].aspect;
    }
    return (int)w.size();
}

// src/voxelization.cpp:66-97.
void ref_top_slope_aspect(const float* heights, int W, int H, float scale, float* slope, float* aspect)
{
    solar_gpu::HeightGrid g;
    g.width = W;
    g.height = H;
    g.scaleX = g.scaleY = scale;
    g.heights.assign(heights, heights + (size_t)W * H);
    solar_gpu::SlopeAspect sa = solar_gpu::compute_top_slope_aspect(g);
    std::memcpy(slope, sa.slope.data(), sizeof(float) * (size_t)W * H);
    std::memcpy(aspect, sa.aspect.data(), sizeof(float) * (size_t)W * H);
}

// include/sun_position.h:24-40: hourly (azimuth, altitude) for 2026.
int ref_sun_positions(float lon, float lat, int tz, float* out, int cap)
{
    std::vector<solar_gpu::SunSample> v;
    solar_gpu::SunPositionCalculator calc(lon, lat, tz);
    calc.calc(v);
    if ((int)v.size() > cap) return -1;
    for (size_t k = 0; k < v.size(); ++k) {
        out[2 * k] = std::get<0>(v[k]);
        out[2 * k + 1] = std::get<1>(v[k]);
    }
    return (int)v.size();
}

}  // extern "C"
