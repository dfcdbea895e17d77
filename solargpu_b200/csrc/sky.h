// Host-side sky bins and traced direction table (see sky.cpp).
#pragma once

#include <vector>

#include "sgb_internal.cuh"

namespace sgb {

struct SkyTables {
    int hsize = 0, vsize = 0, vsize_full = 0;
    int active = 0;                 // sun-visited upper bins
    int words32 = 0;                // shadow words per voxel
    std::vector<int> full_to_dense; // [hsize * vsize]
    std::vector<int> sun_dense;     // [8760]
    std::vector<float> nudged;      // [8760 * 2]
    std::vector<int> hour_index;    // daylight hours (nudged altitude >= 1 deg), ascending
    std::vector<DirEntry> dirs;     // [hsize * vsize_full]
    std::vector<ConeSpec> cones;    // early-exit tables named by the upper directions' meta
};

SkyTables make_sky_tables(const float* sun_az_alt, float h_res = 5.0f, float v_res = 5.0f);

}  // namespace sgb
