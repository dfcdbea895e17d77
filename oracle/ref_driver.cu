// Test infrastructure: a driver for the reference CUDA pipeline, compiled
// together with the reference's own .cu/.cpp sources (unmodified, from where
// they lie) into oracle/_ref/libsolarref.so.  It replaces the reference CLI
// (which needs libtiff) with in-memory inputs and exposes:
//   * ref_uncompressed / ref_compressed: the stock public API
//     (include/solar_gpu_api.h:37-54), called exactly as src/main.cpp:134-143
//     calls it;
//   * ref_stage1: the reference's own out-of-core viewshed stage
//     (include/cuda/viewshed_stage.cuh:37-125) with the two stock chunk
//     consumers (CSR: gpu_irradiance_uncompressed.cu:84-94; ba-RLE:
//     gpu_irradiance_compressed.cu:245-257) to dump neighbor lists, ba-RLE
//     streams and the shadow bitmap for parity checks.
// Never linked into the product.
#include <cstdlib>
#include <cstring>
#include <vector>

#include "solar_gpu_api.h"
#include "barle_compression.h"
#include "cuda_utils.cuh"
#include "sky_bins.h"
#include "voxel_types.h"
#include "cuda/device_globals.cuh"
#include "cuda/viewshed_stage.cuh"

using namespace solar_gpu;

extern "C" {

struct RefStage1 {
    long long num_total;
    long long nnz;
    int* csr_off;          // [num_total + 1]
    int* csr_ids;          // [nnz], 1-based cell ids in first-occurrence order
    long long barle_bytes;
    int* barle_off;        // [num_total + 1]
    unsigned char* barle;  // [barle_bytes]
    int svf_words8;        // hgrid_size_s
    unsigned char* svf;    // [svf_words8][num_total], word-major / voxel-minor
};

static std::vector<SunSample> to_samples(const float* sun)
{
    std::vector<SunSample> s(kHoursPerYear);
    for (int k = 0; k < kHoursPerYear; ++k) s[k] = SunSample(sun[2 * k], sun[2 * k + 1]);
    return s;
}

int ref_stage1(const float* grid, int W, int H, int num_total, int num_top,
               const int* pix_parent, const float* wall_z, float maxz,
               const float* sun, RefStage1* out)
{
    std::memset(out, 0, sizeof(*out));
    cudaSetDevice(0);
    SkyBins bins = compute_sky_bins(to_samples(sun));
    std::vector<float> zeros(kHoursPerYear, 0.0f);
    upload_pipeline_constants(W, H, num_top, num_total, maxz, bins, zeros, zeros);
    const int num_walls = num_total - num_top;
    float* grid_d = nullptr; int* pp_d = nullptr; float* wz_d = nullptr;
    cudaSafeCall(cudaMalloc((void**)&grid_d, (size_t)W * H * sizeof(float)));
    cudaSafeCall(cudaMalloc((void**)&pp_d, (size_t)num_total * sizeof(int)));
    cudaSafeCall(cudaMemcpy(grid_d, grid, (size_t)W * H * sizeof(float), cudaMemcpyHostToDevice));
    cudaSafeCall(cudaMemcpy(pp_d, pix_parent, (size_t)num_total * sizeof(int), cudaMemcpyHostToDevice));
    if (num_walls > 0) {
        cudaSafeCall(cudaMalloc((void**)&wz_d, (size_t)num_walls * sizeof(float)));
        cudaSafeCall(cudaMemcpy(wz_d, wall_z, (size_t)num_walls * sizeof(float), cudaMemcpyHostToDevice));
    }
    std::vector<int> nb_off(num_total + 1, 0), nb_flat;
    std::vector<int> comp_off(num_total + 1, 0);
    std::vector<barle::Byte> comp_flat;
    grid_s_type* grid_s_d = run_viewshed_out_of_core(
        grid_d, pp_d, wz_d, num_total, bins,
        [&](int voxel_offset, int chunk_count, int trimmed_max, const std::vector<int>& raw) {
            for (int i = 0; i < chunk_count; ++i) {
                nb_off[voxel_offset + i] = (int)nb_flat.size();
                size_t base = (size_t)i * trimmed_max;
                for (int k = 0; k < trimmed_max; ++k) {
                    int v = raw[base + k];
                    if (v == 0) break;
                    nb_flat.push_back(v);
                }
            }
            std::vector<int> co;
            std::vector<barle::Byte> cf;
            size_t rb = 0;
            barle::compress_all_neighbors(raw.data(), chunk_count, trimmed_max, co, cf, rb);
            int base_offset = (int)comp_flat.size();
            for (int i = 0; i < chunk_count; ++i) comp_off[voxel_offset + i] = base_offset + co[i];
            comp_flat.insert(comp_flat.end(), cf.begin(), cf.end());
        });
    nb_off[num_total] = (int)nb_flat.size();
    comp_off[num_total] = (int)comp_flat.size();

    size_t svf_bytes = (size_t)bins.hgrid_size_s * num_total;
    out->num_total = num_total;
    out->nnz = (long long)nb_flat.size();
    out->csr_off = (int*)std::malloc(sizeof(int) * (num_total + 1));
    out->csr_ids = (int*)std::malloc(sizeof(int) * (nb_flat.size() + 1));
    std::memcpy(out->csr_off, nb_off.data(), sizeof(int) * (num_total + 1));
    if (!nb_flat.empty()) std::memcpy(out->csr_ids, nb_flat.data(), sizeof(int) * nb_flat.size());
    out->barle_bytes = (long long)comp_flat.size();
    out->barle_off = (int*)std::malloc(sizeof(int) * (num_total + 1));
    out->barle = (unsigned char*)std::malloc(comp_flat.size() + 1);
    std::memcpy(out->barle_off, comp_off.data(), sizeof(int) * (num_total + 1));
    if (!comp_flat.empty()) std::memcpy(out->barle, comp_flat.data(), comp_flat.size());
    out->svf_words8 = (int)bins.hgrid_size_s;
    out->svf = (unsigned char*)std::malloc(svf_bytes + 1);
    cudaSafeCall(cudaMemcpy(out->svf, grid_s_d, svf_bytes, cudaMemcpyDeviceToHost));

    cudaSafeCall(cudaFree(grid_s_d));
    cudaSafeCall(cudaFree(grid_d));
    cudaSafeCall(cudaFree(pp_d));
    if (wz_d) cudaSafeCall(cudaFree(wz_d));
    return 0;
}

void ref_stage1_free(RefStage1* s)
{
    std::free(s->csr_off); std::free(s->csr_ids);
    std::free(s->barle_off); std::free(s->barle); std::free(s->svf);
    std::memset(s, 0, sizeof(*s));
}

static int call_api(int compressed, const float* grid, int W, int H, int num_total, int num_top,
                    const int* pix_parent, const float* wall_z, float maxz, const float* sun,
                    const float* dni, const float* dhi, const float* slopes, const float* aspects,
                    float* out)
{
    std::vector<SunSample> s = to_samples(sun);
    std::vector<float> dn(dni, dni + kHoursPerYear), df(dhi, dhi + kHoursPerYear);
    if (compressed)
        return compressed_gpu_irradiance(grid, W, H, num_total, num_top, pix_parent, wall_z, maxz,
                                         s, dn, df, slopes, aspects, out);
    return uncompressed_gpu_irradiance(grid, W, H, num_total, num_top, pix_parent, wall_z, maxz,
                                       s, dn, df, slopes, aspects, out);
}

int ref_uncompressed(const float* grid, int W, int H, int num_total, int num_top,
                     const int* pix_parent, const float* wall_z, float maxz, const float* sun,
                     const float* dni, const float* dhi, const float* slopes, const float* aspects,
                     float* out)
{
    return call_api(0, grid, W, H, num_total, num_top, pix_parent, wall_z, maxz, sun, dni, dhi,
                    slopes, aspects, out);
}

int ref_compressed(const float* grid, int W, int H, int num_total, int num_top,
                   const int* pix_parent, const float* wall_z, float maxz, const float* sun,
                   const float* dni, const float* dhi, const float* slopes, const float* aspects,
                   float* out)
{
    return call_api(1, grid, W, H, num_total, num_top, pix_parent, wall_z, maxz, sun, dni, dhi,
                    slopes, aspects, out);
}

}  // extern "C"
