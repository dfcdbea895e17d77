// Voxelization on the GPU: the column-drop wall voxels and the top slope /
// aspect of a heightmap, packed as the reference CLI packs them for the
// irradiance entry points (src/main.cpp:112-127).
//
// The reference computes these on the host (src/voxelization.cpp:10-97,
// detect_wall_voxels and compute_top_slope_aspect), one cell after the other.
// Here a count pass gives every cell its number of wall voxels, a scan turns
// the counts into offsets, and a write pass fills the voxel arrays:
//   voxels [0, T)        top voxel i = cell i (pixel_parent i), its slope
//                        and aspect from central differences;
//   voxels [T, T + walls) walls in raster order of their cell, from the top of
//                        the drop downwards (the order the reference appends
//                        them), at z0 - (v + 0.5) voxel_size, slope pi / 2,
//                        aspect from the openness of the four sides.
// Float operations are written out (no contraction) in the reference's order,
// so wall counts and heights are identical; angles come from CUDA's atan2f
// and may differ from the host library's in the last bits.
#include "sgb_internal.cuh"

namespace sgb {
namespace {

constexpr float kOpenOutside = -1e30f;   // voxelization.cpp:16
constexpr float kPiF = 3.14159265358979323846f;

__device__ __forceinline__ float height_at(const float* g, int W, int H, int x, int y)
{
    // clamped load: in bounds however the select is compiled
    const float h = g[(size_t)min(max(y, 0), H - 1) * W + min(max(x, 0), W - 1)];
    return (x >= 0 && x < W && y >= 0 && y < H) ? h : kOpenOutside;
}

// Wall voxels of cell (gx, gy) and the side heights their aspect needs.
__device__ __forceinline__ int wall_count(const float* g, int W, int H, int gx, int gy, float vs, float& z0, float& hE,
                                          float& hW, float& hN, float& hS)
{
    z0 = g[(size_t)gy * W + gx];
    hE = height_at(g, W, H, gx + 1, gy);
    hW = height_at(g, W, H, gx - 1, gy);
    hN = height_at(g, W, H, gx, gy - 1);
    hS = height_at(g, W, H, gx, gy + 1);
    const float half = kOpenOutside * 0.5f;
    const float cE = (hE <= half) ? z0 : hE;
    const float cW = (hW <= half) ? z0 : hW;
    const float cN = (hN <= half) ? z0 : hN;
    const float cS = (hS <= half) ? z0 : hS;
    const float mn = fminf(fminf(cE, cW), fminf(cN, cS));
    const float drop = __fsub_rn(z0, mn);
    if (!(drop > vs)) return 0;
    return (int)__fdiv_rn(drop, vs);
}

__global__ void k_vox_count(const float* __restrict__ g, int W, int H, float vs, int* __restrict__ counts)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W * H) return;
    float z0, hE, hW, hN, hS;
    counts[i] = wall_count(g, W, H, i % W, i / W, vs, z0, hE, hW, hN, hS);
}

__global__ void k_vox_write(const float* __restrict__ g, int W, int H, float vs, float scale,
                            const long long* __restrict__ off, int* __restrict__ parent, float* __restrict__ wall_z,
                            float* __restrict__ slopes, float* __restrict__ aspects)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int T = W * H;
    if (i >= T) return;
    const int gx = i % W, gy = i / W;
    // top voxel: central differences, clamped at the border (voxelization.cpp:66-97)
    {
        const int xl = max(gx - 1, 0), xr = min(gx + 1, W - 1);
        const int yu = max(gy - 1, 0), yd = min(gy + 1, H - 1);
        const float zl = g[(size_t)gy * W + xl], zr = g[(size_t)gy * W + xr];
        const float zu = g[(size_t)yu * W + gx], zd = g[(size_t)yd * W + gx];
        const float dx = __fdiv_rn(__fsub_rn(zr, zl), __fmul_rn((float)(xr - xl), scale));
        const float dy = __fdiv_rn(__fsub_rn(zd, zu), __fmul_rn((float)(yd - yu), scale));
        const float mag = __fsqrt_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
        parent[i] = i;
        slopes[i] = atan2f(mag, 1.0f);
        float a = atan2f(-dx, dy);
        if (a < 0.0f) a = __fadd_rn(a, 2.0f * kPiF);
        aspects[i] = a;
    }
    float z0, hE, hW, hN, hS;
    const int n = wall_count(g, W, H, gx, gy, vs, z0, hE, hW, hN, hS);
    const long long base = (long long)T + off[i];
    for (int v = 0; v < n; ++v) {
        const float zz = __fsub_rn(z0, __fmul_rn(__fadd_rn((float)v, 0.5f), vs));
        const float oE = fmaxf(0.0f, __fsub_rn(zz, hE));
        const float oW = fmaxf(0.0f, __fsub_rn(zz, hW));
        const float oN = fmaxf(0.0f, __fsub_rn(zz, hN));
        const float oS = fmaxf(0.0f, __fsub_rn(zz, hS));
        float a = atan2f(__fsub_rn(oE, oW), __fsub_rn(oN, oS));
        if (a < 0.0f) a = __fadd_rn(a, 2.0f * kPiF);
        parent[base + v] = i;
        wall_z[off[i] + v] = zz;
        slopes[base + v] = kPiF * 0.5f;
        aspects[base + v] = a;
    }
}

}  // namespace

cudaError_t launch_vox_count(const float* grid, int W, int H, float voxel_size, int* counts, cudaStream_t st)
{
    const int T = W * H;
    if (T <= 0) return cudaSuccess;
    k_vox_count<<<(T + 255) / 256, 256, 0, st>>>(grid, W, H, voxel_size, counts);
    return cudaGetLastError();
}

cudaError_t launch_vox_write(const float* grid, int W, int H, float voxel_size, float scale, const long long* off,
                             int* parent, float* wall_z, float* slopes, float* aspects, cudaStream_t st)
{
    const int T = W * H;
    if (T <= 0) return cudaSuccess;
    k_vox_write<<<(T + 255) / 256, 256, 0, st>>>(grid, W, H, voxel_size, scale, off, parent, wall_z, slopes, aspects);
    return cudaGetLastError();
}

}  // namespace sgb
