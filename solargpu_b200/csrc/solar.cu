// Solar pass: FP64 per-hour geometry table, per-voxel geometry, and the
// direct + Perez diffuse kernels (src/cuda/kernels/solar_kernel.cu:8-85).
//
// The reference recomputes the sun geometry and every Perez term
// (acosf/powf/cosf per voxel and hour, solar_kernel.cu:8-50, 66-74) for every
// voxel.  Those terms depend only on the hour, so here one FP64 kernel
// evaluates them once per daylight hour (k_hour_table); the per voxel-hour
// work is a dot product, a shadow-bit test and three FMAs (solar_I).
#include "solar_math.cuh"

namespace sgb {
namespace {

// Reference constants at their float values (solar_kernel.cu:8-50,
// src/cuda/device_globals.cu:50-57, include/pipeline_math_constants.h:15).
#define FC(x) ((double)(float)(x))
__constant__ double c_F[6][8] = {
    { FC(-0.0083117), FC(0.1299457), FC(0.3296958), FC(0.5682053), FC(0.8730280), FC(1.1326077), FC(1.0601591), FC(0.6777470) },
    { FC(0.5877285), FC(0.6825954), FC(0.4868735), FC(0.1874525), FC(-0.3920403), FC(-1.2367284), FC(-1.5999137), FC(-0.3272588) },
    { FC(-0.0620636), FC(-0.1513752), FC(-0.2210958), FC(-0.2951290), FC(-0.3616149), FC(-0.4118494), FC(-0.3589221), FC(-0.2504286) },
    { FC(-0.0596012), FC(-0.0189325), FC(0.0554140), FC(0.1088631), FC(0.2255647), FC(0.2877813), FC(0.2642124), FC(0.1561313) },
    { FC(0.0721249), FC(0.0659650), FC(-0.0639588), FC(-0.1519229), FC(-0.4620442), FC(-0.8230357), FC(-1.1272340), FC(-1.3765031) },
    { FC(-0.0220216), FC(-0.0288748), FC(-0.0260542), FC(-0.0139754), FC(0.0012448), FC(0.0558651), FC(0.1310694), FC(0.2506212) },
};

__global__ void k_hour_table(const float* __restrict__ nudged, const float* __restrict__ dni,
                             const float* __restrict__ dhi, const int* __restrict__ sun_dense,
                             const int* __restrict__ hour_index, int n_hours, int n_padded,
                             HourEntry* __restrict__ table)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_padded) return;
    HourEntry e;
    e.sx = e.sy = e.sz = e.dni_eff = e.c0 = e.c1 = e.c2 = 0.0f;
    e.dense = -1;
    if (j < n_hours) {
        const int k = hour_index[j];
        const double kDeg = FC(0.0174532925);
        const double pi_f = FC(3.14159265358979323846);
        const double alt = nudged[2 * k + 1];
        const double az = nudged[2 * k];
        const double cz = cos((90.0 - alt) * kDeg);
        const double z = acos(cz);
        const double sz = sin(z);
        const double dn = dni[k], df = dhi[k];
        // Perez sky model, solar_kernel.cu:8-50
        const double z_deg = z * (180.0 / pi_f);
        const double AM = 1.0 / (cz + FC(0.50572) * pow(FC(96.07995) - z_deg, FC(-1.6364)));
        const double b = fmax(FC(0.08715574), cz);
        const double z3 = z * z * z;
        double eps = ((df + dn / cos(z)) / df + FC(1.041) * z3) / (1.0 + FC(1.041) * z3);
        const double day = (double)(k / 24);
        const double B = 2.0 * pi_f * (day / 365.0);
        const double E0 = 1367.0 * (FC(1.00011) + FC(0.034221) * cos(B) + FC(0.00128) * sin(B)
                                    + FC(0.000719) * cos(2.0 * B) + FC(0.000077) * sin(2.0 * B));
        const double delta = (AM * df) / E0;
        eps = fmax(1.0, eps);   // NaN (DHI = DNI = 0) -> 1, as fmaxf does in the reference
        int bin = 7;
        if (eps < FC(1.065)) bin = 0;
        else if (eps < FC(1.230)) bin = 1;
        else if (eps < FC(1.500)) bin = 2;
        else if (eps < FC(1.950)) bin = 3;
        else if (eps < FC(2.800)) bin = 4;
        else if (eps < FC(4.500)) bin = 5;
        else if (eps < FC(6.200)) bin = 6;
        const double F1 = fmax(0.0, c_F[0][bin] + c_F[1][bin] * delta + c_F[2][bin] * z);
        const double F2 = c_F[3][bin] + c_F[4][bin] * delta + c_F[5][bin] * z;
        e.sx = (float)(sz * sin(az * kDeg));
        e.sy = (float)(-sz * cos(az * kDeg));
        e.sz = (float)cz;
        e.dni_eff = (float)fmax(dn, FC(1e-3));
        e.c0 = (float)(df * (1.0 - F1) * 0.5);
        e.c1 = (float)(df * F1 / b);
        e.c2 = (float)(df * F2);
        e.dense = sun_dense[k];
    }
    table[j] = e;
}

__global__ void k_voxel_geom(DevScene s, float4* __restrict__ geo_n, float4* __restrict__ geo_p)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= s.N) return;
    const int top = s.pix_parent[v];
    const int gx = top % s.W, gy = top / s.W;
    const float z = (v < s.T) ? s.grid[top] : s.wall_z[v - s.T];
    const float sl = s.slopes[v], as = s.aspects[v];
    const float ss = sinf(sl);
    geo_n[v] = make_float4(ss * sinf(as), -ss * cosf(as), cosf(sl), ss);
    geo_p[v] = make_float4((float)gx, (float)gy, z, 0.0f);
}

// slab[g * B + b] = I(g, j0 + b) for every top cell g.  A warp owns 32
// consecutive hours of the block (their table entries stay in registers)
// and sweeps a run of cells, writing one coalesced 128-byte row piece per
// cell; the voxel normal is a broadcast load.
constexpr int kSlabCellsPerWarp = 64;

__global__ void __launch_bounds__(256)
k_solar_slab(const float4* __restrict__ geo_n, int T, const uint32_t* __restrict__ shadow, int words32,
             const HourEntry* __restrict__ table, int j0, int B, float* __restrict__ slab)
{
    const int lane = threadIdx.x & 31;
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int hchunks = B >> 5;
    const int hc = (int)(wid % hchunks);
    const long long g0 = (wid / hchunks) * kSlabCellsPerWarp;
    if (g0 >= T) return;
    const int b = hc * 32 + lane;
    const HourEntry e = table[j0 + b];
    const int word = e.dense >= 0 ? (e.dense >> 5) : 0;
    const uint32_t mask = e.dense >= 0 ? (1u << (e.dense & 31)) : 0u;
    const long long g1 = min((long long)T, g0 + kSlabCellsPerWarp);
#pragma unroll 4
    for (long long g = g0; g < g1; ++g) {
        const float4 n4 = __ldg(geo_n + g);
        const uint32_t bit = (__ldg(shadow + g * words32 + word) & mask) ? 1u : 0u;
        slab[g * B + b] = solar_I(n4, e, bit);
    }
}

__global__ void __launch_bounds__(256)
k_solar_hour(const float4* __restrict__ geo_n, int N, const uint32_t* __restrict__ shadow, int words32,
             const HourEntry* __restrict__ table, int j, float* __restrict__ hourly)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const HourEntry e = table[j];
    hourly[v] = solar_I(__ldg(geo_n + v), e, shadow_bit(shadow, words32, v, e.dense));
}

// sums[v] = sum over all daylight hours of I(v, h), accumulated in FP64.
__global__ void __launch_bounds__(256)
k_solar_sum(const float4* __restrict__ geo_n, int N, const uint32_t* __restrict__ shadow, int words32,
            const HourEntry* __restrict__ table, int n_hours, double* __restrict__ sums)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const float4 n4 = __ldg(geo_n + v);
    double acc = 0.0;
    float part = 0.0f;
    for (int j = 0; j < n_hours; ++j) {
        const HourEntry e = table[j];
        part += solar_I(n4, e, shadow_bit(shadow, words32, v, e.dense));
        if ((j & 31) == 31) { acc += part; part = 0.0f; }
    }
    sums[v] = acc + part;
}

}  // namespace

cudaError_t launch_hour_table(const float* nudged, const float* dni, const float* dhi,
                              const int* sun_dense, const int* hour_index, int n_hours,
                              int n_padded, HourEntry* table, cudaStream_t st)
{
    k_hour_table<<<(n_padded + 127) / 128, 128, 0, st>>>(nudged, dni, dhi, sun_dense, hour_index,
                                                          n_hours, n_padded, table);
    return cudaGetLastError();
}

cudaError_t launch_voxel_geom(const DevScene& s, DevGeom g, cudaStream_t st)
{
    if (s.N <= 0) return cudaSuccess;
    k_voxel_geom<<<(s.N + 255) / 256, 256, 0, st>>>(s, g.geo_n, g.geo_p);
    return cudaGetLastError();
}

cudaError_t launch_solar_slab(const DevGeom& g, int T, const uint32_t* shadow, int words32,
                              const HourEntry* table, int j0, int B, float* slab, cudaStream_t st)
{
    if (B < 32 || (B & 31)) return cudaErrorInvalidValue;
    const long long warps = ((long long)T + kSlabCellsPerWarp - 1) / kSlabCellsPerWarp * (B / 32);
    k_solar_slab<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(g.geo_n, T, shadow, words32, table,
                                                                        j0, B, slab);
    return cudaGetLastError();
}

cudaError_t launch_solar_hour(const DevGeom& g, int N, const uint32_t* shadow, int words32,
                              const HourEntry* table, int j, float* hourly, cudaStream_t st)
{
    k_solar_hour<<<(N + 255) / 256, 256, 0, st>>>(g.geo_n, N, shadow, words32, table, j, hourly);
    return cudaGetLastError();
}

cudaError_t launch_solar_sum(const DevGeom& g, int N, const uint32_t* shadow, int words32,
                             const HourEntry* table, int n_hours, double* sums, cudaStream_t st)
{
    k_solar_sum<<<(N + 255) / 256, 256, 0, st>>>(g.geo_n, N, shadow, words32, table, n_hours, sums);
    return cudaGetLastError();
}

}  // namespace sgb
