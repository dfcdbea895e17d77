// The reference's own C++ entry points (include/solar_gpu_api.h:37-54),
// exported with identical signatures so the reference CLI (src/main.cpp)
// links against libsolargpu_b200.so unchanged.  They repack the
// std::vector<std::tuple<float, float>> sun series into a flat array and
// forward to the C ABI (include/solargpu_b200.h).  Unlike the reference,
// a failure returns a nonzero code instead of exiting the process.
#include <tuple>
#include <vector>

#include "solargpu_b200.h"

namespace solar_gpu {

using SunSample = std::tuple<float, float>;   // include/sun_position.h:15

namespace {

std::vector<float> flatten(const std::vector<SunSample>& sun)
{
    std::vector<float> flat(2 * sun.size());
    for (size_t k = 0; k < sun.size(); ++k) {
        flat[2 * k] = std::get<0>(sun[k]);
        flat[2 * k + 1] = std::get<1>(sun[k]);
    }
    return flat;
}

}  // namespace

int uncompressed_gpu_irradiance(const float* grid_data, int grid_width, int grid_height,
    int num_total_voxels, int num_top_voxels,
    const int* pixel_parent, const float* wall_z, float max_height,
    const std::vector<SunSample>& sun_positions,
    const std::vector<float>& direct_irradiance, const std::vector<float>& diffuse_irradiance,
    const float* slopes, const float* aspects, float* irradiance_out)
{
    const std::vector<float> sun = flatten(sun_positions);
    return solar_gpu_uncompressed_gpu_irradiance(grid_data, grid_width, grid_height, num_total_voxels,
        num_top_voxels, pixel_parent, wall_z, max_height, sun.data(), (int)sun_positions.size(),
        direct_irradiance.data(), (int)direct_irradiance.size(), diffuse_irradiance.data(),
        (int)diffuse_irradiance.size(), slopes, aspects, irradiance_out);
}

int compressed_gpu_irradiance(const float* grid_data, int grid_width, int grid_height,
    int num_total_voxels, int num_top_voxels,
    const int* pixel_parent, const float* wall_z, float max_height,
    const std::vector<SunSample>& sun_positions,
    const std::vector<float>& direct_irradiance, const std::vector<float>& diffuse_irradiance,
    const float* slopes, const float* aspects, float* irradiance_out)
{
    const std::vector<float> sun = flatten(sun_positions);
    return solar_gpu_compressed_gpu_irradiance(grid_data, grid_width, grid_height, num_total_voxels,
        num_top_voxels, pixel_parent, wall_z, max_height, sun.data(), (int)sun_positions.size(),
        direct_irradiance.data(), (int)direct_irradiance.size(), diffuse_irradiance.data(),
        (int)diffuse_irradiance.size(), slopes, aspects, irradiance_out);
}

}  // namespace solar_gpu
