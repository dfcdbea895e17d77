// Reflection pass over CSR or ba-RLE neighbor lists, and the annual
// accumulation (src/cuda/kernels/reflection_kernels.cu:18-183,
// src/cuda/kernels/solar_kernel.cu:79-85).
//
// Hour-block SpMM (k_reflect_block): the reference walks every voxel's list
// once per hour (4337 launches).  The reflection weight w(v, g) does not
// depend on the hour, so per block of B = 32*Q hours one warp owns a voxel:
// lanes hold hours, the list is decoded once, each (w, g) pair is computed
// once by one lane and broadcast through shared memory, and every lane adds
// w * I[g][h] for its hours with a coalesced 128-byte read of the slab row.
// The voxel's own direct + diffuse for the block is computed in the same
// kernel and the block sum goes into the annual accumulator (FP64, Kahan
// FP32 or plain FP32).
//
// ba-RLE decode is warp-parallel: a block header (<= 8 runs) is parsed by
// all lanes, run payload offsets come from a lane prefix sum, each lane
// decodes one delta, and ids follow from an inclusive warp scan of the
// signed deltas (val_i = val_{i-1} - delta_i, first value absolute), which
// is the reference's serial decoder (reflection_kernels.cu:132-180)
// evaluated in parallel.  Every byte read is checked against the voxel's
// range; a malformed stream sets kErrBarleStream and stops that voxel.
#include "solar_math.cuh"

namespace sgb {
namespace {

constexpr int kReflWarps = 8;
constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

// Visits a voxel's ba-RLE stream [base, base + size) in chunks of up to 32
// decoded ids, calling on_chunk(g) with g = id - 1 for this lane's element
// (or -1).  Warp-collective.
template <typename F>
__device__ __forceinline__ void barle_for_each_chunk(const unsigned char* __restrict__ bytes,
                                                     long long base, long long size, int lane,
                                                     int4* runs, int* err, F&& on_chunk)
{
    long long cur = 0;
    uint32_t carry = 0;
    bool first = true;
    while (cur < size) {
        if (cur + 3 > size) { if (lane == 0) atomicOr(err, kErrBarleStream); return; }
        const unsigned char* p = bytes + base + cur;
        const uint32_t bits = ((uint32_t)p[0] << 16) | ((uint32_t)p[1] << 8) | (uint32_t)p[2];
        int nc = 0;
        bool bad = false;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int code = (int)((bits >> (21 - 3 * r)) & 7u);
            if (code == 7) break;
            if (code > 4) bad = true;
            ++nc;
        }
        if (bad || cur + 3 + nc > size) { if (lane == 0) atomicOr(err, kErrBarleStream); return; }
        int w = 0, len = 0, pay = 0;
        if (lane < nc) {
            w = (int)((bits >> (21 - 3 * lane)) & 7u);
            len = p[3 + lane];
            pay = (w == 0) ? (len + 1) >> 1 : len * w;
        }
        int lp = len, pp = pay;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const int a = __shfl_up_sync(kFull, lp, o);
            const int b = __shfl_up_sync(kFull, pp, o);
            if (lane >= o) { lp += a; pp += b; }
        }
        const int total_len = __shfl_sync(kFull, lp, 7);
        const int total_pay = __shfl_sync(kFull, pp, 7);
        const long long pay_base = cur + 3 + nc;
        if (pay_base + total_pay > size) { if (lane == 0) atomicOr(err, kErrBarleStream); return; }
        if (lane < nc) runs[lane] = make_int4(w, len, lp - len, pp - pay);
        __syncwarp();
        const unsigned char* payload = bytes + base + pay_base;
        for (int e0 = 0; e0 < total_len; e0 += 32) {
            const int e = e0 + lane;
            const bool valid = e < total_len;
            uint32_t d = 0;
            if (valid) {
                int r = 0;
                for (int t = 1; t < nc; ++t) if (runs[t].z <= e) r = t;
                const int4 R = runs[r];
                const int i = e - R.z;
                const unsigned char* q = payload + R.w;
                if (R.x == 0) {
                    const uint32_t b = q[i >> 1];
                    d = (i & 1) ? (b & 15u) : (b >> 4);
                } else {
                    for (int b = 0; b < R.x; ++b) d = (d << 8) | q[i * R.x + b];
                }
            }
            uint32_t s = valid ? ((first && e == 0) ? d : 0u - d) : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFull, s, o);
                if (lane >= o) s += y;
            }
            const uint32_t val = carry + s;
            carry = __shfl_sync(kFull, val, min(31, total_len - e0 - 1));
            first = false;
            on_chunk((valid && val > 0u) ? (int)(val - 1u) : -1);
        }
        __syncwarp();
        cur = pay_base + total_pay;
    }
}

template <typename F>
__device__ __forceinline__ void csr_for_each_chunk(const long long* __restrict__ off,
                                                   const int* __restrict__ ids, int v, int lane,
                                                   F&& on_chunk)
{
    const long long s = off[v], e = off[v + 1];
    for (long long c = s; c < e; c += 32) {
        const long long i = c + lane;
        on_chunk(i < e ? __ldg(ids + i) - 1 : -1);
    }
}

template <int Q>
__device__ __forceinline__ void slab_chunk(int g, const float4 me_p, const float4 me_n,
                                           const float4* __restrict__ geo_p, int T,
                                           float2* wg, const float* __restrict__ slab, int lane,
                                           float (&acc)[Q])
{
    float w = 0.0f;
    if (g >= 0 && g < T) w = refl_weight(me_p, me_n, __ldg(geo_p + g));
    const unsigned bal = __ballot_sync(kFull, w != 0.0f);
    if (w != 0.0f) wg[__popc(bal & lanemask_lt(lane))] = make_float2(w, __int_as_float(g));
    __syncwarp();
    const int n = __popc(bal);
#pragma unroll 4
    for (int t = 0; t < n; ++t) {
        const float2 x = wg[t];
        const float* row = slab + (size_t)__float_as_int(x.y) * (32 * Q) + lane;
#pragma unroll
        for (int q = 0; q < Q; ++q) acc[q] = fmaf(x.x, __ldg(row + 32 * q), acc[q]);
    }
    __syncwarp();
}

__device__ __forceinline__ void accumulate(const Accum& a, int v, float x)
{
    if (a.mode == 0) {
        a.f64[v] += (double)x;
    } else if (a.mode == 1) {
        // Kahan-compensated FP32: explicit round-to-nearest ops, no reassociation.
        const float y = __fsub_rn(x, a.comp[v]);
        const float s = a.f32[v];
        const float t = __fadd_rn(s, y);
        a.comp[v] = __fsub_rn(__fsub_rn(t, s), y);
        a.f32[v] = t;
    } else {
        a.f32[v] = __fadd_rn(a.f32[v], x);
    }
}

template <int Q, int FMT>
__global__ void __launch_bounds__(kReflWarps * 32)
k_reflect_block(float4* __restrict__ geo_n_, float4* __restrict__ geo_p_, int N, int T,
                const uint32_t* __restrict__ shadow, int words32, const HourEntry* __restrict__ table,
                int j0, const float* __restrict__ slab, NeighborLists nl, Accum acc, int* err)
{
    __shared__ float2 s_wg[kReflWarps][32];
    __shared__ int4 s_runs[kReflWarps][8];
    const float4* geo_n = geo_n_;
    const float4* geo_p = geo_p_;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int stride = gridDim.x * kReflWarps;
    for (int v = blockIdx.x * kReflWarps + warp; v < N; v += stride) {
        const float4 me_p = __ldg(geo_p + v);
        const float4 me_n = __ldg(geo_n + v);
        float own[Q], r[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const HourEntry e = table[j0 + lane + 32 * q];
            own[q] = solar_I(me_n, e, shadow_bit(shadow, words32, v, e.dense));
            r[q] = 0.0f;
        }
        auto chunk = [&](int g) { slab_chunk<Q>(g, me_p, me_n, geo_p, T, s_wg[warp], slab, lane, r); };
        if (FMT == 0) {
            csr_for_each_chunk(nl.offsets, nl.ids, v, lane, chunk);
        } else {
            const long long b0 = nl.offsets[v];
            barle_for_each_chunk(nl.bytes, b0, nl.offsets[v + 1] - b0, lane, s_runs[warp], err, chunk);
        }
        float sum = 0.0f;
#pragma unroll
        for (int q = 0; q < Q; ++q) sum += own[q] + r[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
        if (lane == 0) accumulate(acc, v, sum);
    }
}

// Plain per-hour path (one launch per daylight hour, thread per voxel,
// serial list walk as in the reference): annual[v] += hourly[v] + R[v].
__device__ __forceinline__ void hour_add(float& R, int g, const float4 me_p, const float4 me_n,
                                         const float4* __restrict__ geo_p, int T,
                                         const float* __restrict__ hourly)
{
    if (g < 0 || g >= T) return;
    const float w = refl_weight(me_p, me_n, __ldg(geo_p + g));
    if (w != 0.0f) R = fmaf(w, __ldg(hourly + g), R);
}

template <int FMT>
__global__ void __launch_bounds__(256)
k_reflect_hour(const float4* __restrict__ geo_n, const float4* __restrict__ geo_p, int N, int T,
               const float* __restrict__ hourly, NeighborLists nl, Accum acc, int* err)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const float4 me_p = __ldg(geo_p + v);
    const float4 me_n = __ldg(geo_n + v);
    float R = 0.0f;
    if (FMT == 0) {
        for (long long k = nl.offsets[v]; k < nl.offsets[v + 1]; ++k)
            hour_add(R, __ldg(nl.ids + k) - 1, me_p, me_n, geo_p, T, hourly);
    } else {
        const long long base = nl.offsets[v];
        const long long size = nl.offsets[v + 1] - base;
        const unsigned char* data = nl.bytes + base;
        long long idx = 0;
        uint32_t prev = 0;
        bool first = true;
        while (idx < size) {
            if (idx + 3 > size) { atomicOr(err, kErrBarleStream); break; }
            const uint32_t bits = ((uint32_t)data[idx] << 16) | ((uint32_t)data[idx + 1] << 8) | data[idx + 2];
            idx += 3;
            int widths[8], nc = 0;
            bool bad = false;
            for (int j = 0; j < 8; ++j) {
                const int code = (int)((bits >> (21 - 3 * j)) & 7u);
                if (code == 7) break;
                if (code > 4) bad = true;
                widths[nc++] = code;
            }
            if (bad || idx + nc > size) { atomicOr(err, kErrBarleStream); break; }
            int lens[8];
            for (int j = 0; j < nc; ++j) lens[j] = data[idx++];
            for (int j = 0; j < nc && !bad; ++j) {
                const int w = widths[j], rl = lens[j];
                if (w == 0) {
                    for (int i = 0; i < rl;) {
                        if (idx >= size) { bad = true; break; }
                        const uint32_t packed = data[idx++];
                        uint32_t val = first ? (packed >> 4) : prev - (packed >> 4);
                        first = false; prev = val;
                        if (val > 0u) hour_add(R, (int)val - 1, me_p, me_n, geo_p, T, hourly);
                        if (++i < rl) {
                            val = prev - (packed & 15u);
                            prev = val;
                            if (val > 0u) hour_add(R, (int)val - 1, me_p, me_n, geo_p, T, hourly);
                            ++i;
                        }
                    }
                } else {
                    for (int i = 0; i < rl; ++i) {
                        if (idx + w > size) { bad = true; break; }
                        uint32_t dl = 0;
                        for (int b = 0; b < w; ++b) dl = (dl << 8) | data[idx++];
                        const uint32_t val = first ? dl : prev - dl;
                        first = false; prev = val;
                        if (val > 0u) hour_add(R, (int)val - 1, me_p, me_n, geo_p, T, hourly);
                    }
                }
            }
            if (bad) { atomicOr(err, kErrBarleStream); break; }
        }
    }
    accumulate(acc, v, __ldg(hourly + v) + R);
}

// Annual (linearity) form: out[v] = sums[v] + sum_g w(v, g) sums[g], FP64 sums.
template <int FMT>
__global__ void __launch_bounds__(kReflWarps * 32)
k_reflect_annual(const float4* __restrict__ geo_n, const float4* __restrict__ geo_p, int N, int T,
                 const double* __restrict__ sums, NeighborLists nl, double* __restrict__ out, int* err)
{
    __shared__ int4 s_runs[kReflWarps][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int stride = gridDim.x * kReflWarps;
    for (int v = blockIdx.x * kReflWarps + warp; v < N; v += stride) {
        const float4 me_p = __ldg(geo_p + v);
        const float4 me_n = __ldg(geo_n + v);
        double r = 0.0;
        auto chunk = [&](int g) {
            if (g >= 0 && g < T) {
                const float w = refl_weight(me_p, me_n, __ldg(geo_p + g));
                if (w != 0.0f) r += (double)w * sums[g];
            }
        };
        if (FMT == 0) {
            csr_for_each_chunk(nl.offsets, nl.ids, v, lane, chunk);
        } else {
            const long long b0 = nl.offsets[v];
            barle_for_each_chunk(nl.bytes, b0, nl.offsets[v + 1] - b0, lane, s_runs[warp], err, chunk);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(kFull, r, o);
        if (lane == 0) out[v] = sums[v] + r;
    }
}

__global__ void k_finalize(Accum a, int N, float* __restrict__ out)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    out[v] = (a.mode == 0) ? (float)a.f64[v] : a.f32[v];
}

__global__ void k_finalize_f64(const double* __restrict__ in, int N, float* __restrict__ out)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < N) out[v] = (float)in[v];
}

int refl_grid(int N)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const long long need = ((long long)N + kReflWarps - 1) / kReflWarps;
    const long long cap = (long long)sms * 8;
    return (int)(need < cap ? need : cap);
}

template <int Q>
cudaError_t launch_block_q(const DevGeom& g, int N, int T, const uint32_t* shadow, int words32,
                           const HourEntry* table, int j0, const float* slab, const NeighborLists& nl,
                           const Accum& acc, int* err, cudaStream_t st)
{
    const int grid = refl_grid(N);
    if (nl.format == 0)
        k_reflect_block<Q, 0><<<grid, kReflWarps * 32, 0, st>>>(g.geo_n, g.geo_p, N, T, shadow, words32,
                                                              table, j0, slab, nl, acc, err);
    else
        k_reflect_block<Q, 1><<<grid, kReflWarps * 32, 0, st>>>(g.geo_n, g.geo_p, N, T, shadow, words32,
                                                              table, j0, slab, nl, acc, err);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_reflect_block(const DevGeom& g, int N, int T, const uint32_t* shadow,
                                 int words32, const HourEntry* table, int j0, int B,
                                 const float* slab, const NeighborLists& nl, const Accum& acc,
                                 int* err, cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    switch (B) {
    case 32: return launch_block_q<1>(g, N, T, shadow, words32, table, j0, slab, nl, acc, err, st);
    case 64: return launch_block_q<2>(g, N, T, shadow, words32, table, j0, slab, nl, acc, err, st);
    case 128: return launch_block_q<4>(g, N, T, shadow, words32, table, j0, slab, nl, acc, err, st);
    case 256: return launch_block_q<8>(g, N, T, shadow, words32, table, j0, slab, nl, acc, err, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_reflect_hour(const DevGeom& g, int N, int T, const float* hourly,
                                const NeighborLists& nl, const Accum& acc, int* err,
                                cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    if (nl.format == 0)
        k_reflect_hour<0><<<(N + 255) / 256, 256, 0, st>>>(g.geo_n, g.geo_p, N, T, hourly, nl, acc, err);
    else
        k_reflect_hour<1><<<(N + 255) / 256, 256, 0, st>>>(g.geo_n, g.geo_p, N, T, hourly, nl, acc, err);
    return cudaGetLastError();
}

cudaError_t launch_reflect_annual(const DevGeom& g, int N, int T, const double* sums,
                                  const NeighborLists& nl, double* out, int* err,
                                  cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    const int grid = refl_grid(N);
    if (nl.format == 0)
        k_reflect_annual<0><<<grid, kReflWarps * 32, 0, st>>>(g.geo_n, g.geo_p, N, T, sums, nl, out, err);
    else
        k_reflect_annual<1><<<grid, kReflWarps * 32, 0, st>>>(g.geo_n, g.geo_p, N, T, sums, nl, out, err);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const Accum& acc, int N, float* out, cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    k_finalize<<<(N + 255) / 256, 256, 0, st>>>(acc, N, out);
    return cudaGetLastError();
}

cudaError_t launch_finalize_f64(const double* in, int N, float* out, cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    k_finalize_f64<<<(N + 255) / 256, 256, 0, st>>>(in, N, out);
    return cudaGetLastError();
}

}  // namespace sgb
