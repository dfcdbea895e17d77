// Test infrastructure: a C++ caller of the two drop-in entry points, compiled
// against the reference's own public header (include/solar_gpu_api.h and
// include/sun_position.h, from where they lie) and linked against
// libsolargpu_b200.so -- the way the reference CLI (src/main.cpp:134-143)
// would link against this library.  It exercises the exported C++ symbols
// (namespace solar_gpu, std::vector<std::tuple<float, float>> sun series).
//
//   cxx_caller <in.bin> <out.bin>
//
// in.bin (little endian): int32 W, H, num_total, num_top; float32 max_height;
// float32 grid[W*H]; int32 pixel_parent[num_total]; float32 wall_z[num_total -
// num_top]; float32 sun[8760][2]; float32 direct[8760]; float32 diffuse[8760];
// float32 slopes[num_total]; float32 aspects[num_total].
// out.bin: int32 rc_uncompressed, rc_compressed; float32 uncompressed[num_total];
// float32 compressed[num_total].
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "solar_gpu_api.h"

namespace {

template <typename T>
bool read_n(FILE* f, T* p, size_t n)
{
    return std::fread(p, sizeof(T), n, f) == n;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    int hdr[4];
    float maxz = 0.0f;
    if (!read_n(f, hdr, 4) || !read_n(f, &maxz, 1)) return 4;
    const int W = hdr[0], H = hdr[1], N = hdr[2], T = hdr[3];
    const int hours = 8760;
    std::vector<float> grid((size_t)W * H), wall((size_t)(N - T)), sun(2 * hours), direct(hours), diffuse(hours),
        slopes(N), aspects(N);
    std::vector<int> parent(N);
    bool ok = read_n(f, grid.data(), grid.size()) && read_n(f, parent.data(), parent.size()) &&
              read_n(f, wall.data(), wall.size()) && read_n(f, sun.data(), sun.size()) &&
              read_n(f, direct.data(), direct.size()) && read_n(f, diffuse.data(), diffuse.size()) &&
              read_n(f, slopes.data(), slopes.size()) && read_n(f, aspects.data(), aspects.size());
    std::fclose(f);
    if (!ok) return 5;

    // the caller-side containers of src/main.cpp:99-127
    std::vector<solar_gpu::SunSample> sun_positions(hours);
    for (int k = 0; k < hours; ++k) sun_positions[k] = solar_gpu::SunSample(sun[2 * k], sun[2 * k + 1]);
    std::vector<float> out_unc(N, 0.0f), out_com(N, 0.0f);
    const float* wz = N > T ? wall.data() : nullptr;
    const int rc_unc = solar_gpu::uncompressed_gpu_irradiance(grid.data(), W, H, N, T, parent.data(), wz, maxz,
                                                              sun_positions, direct, diffuse, slopes.data(),
                                                              aspects.data(), out_unc.data());
    const int rc_com = solar_gpu::compressed_gpu_irradiance(grid.data(), W, H, N, T, parent.data(), wz, maxz,
                                                            sun_positions, direct, diffuse, slopes.data(),
                                                            aspects.data(), out_com.data());
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 6;
    const int rcs[2] = {rc_unc, rc_com};
    std::fwrite(rcs, sizeof(int), 2, o);
    std::fwrite(out_unc.data(), sizeof(float), out_unc.size(), o);
    std::fwrite(out_com.data(), sizeof(float), out_com.size(), o);
    std::fclose(o);
    return 0;
}
