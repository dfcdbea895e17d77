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

#include <atomic>

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
        // Run table in registers: lane r < 8 holds run r (lanes nc..7 hold
        // empty runs starting at total_len, so they are never selected).
        const int estart = lp - len, boff = pp - pay;
        int st[7];
#pragma unroll
        for (int t = 0; t < 7; ++t) st[t] = __shfl_sync(kFull, estart, t + 1);
        const unsigned char* payload = bytes + base + pay_base;
        for (int e0 = 0; e0 < total_len; e0 += 32) {
            const int e = e0 + lane;
            const bool valid = e < total_len;
            int r = 0;
#pragma unroll
            for (int t = 0; t < 7; ++t) r += (e >= st[t]) ? 1 : 0;
            const int Rw = __shfl_sync(kFull, w, r);
            const int Rs = __shfl_sync(kFull, estart, r);
            const int Rb = __shfl_sync(kFull, boff, r);
            uint32_t d = 0;
            if (valid) {
                const int i = e - Rs;
                const unsigned char* q = payload + Rb;
                if (Rw == 0) {
                    const uint32_t b = q[i >> 1];
                    d = (i & 1) ? (b & 15u) : (b >> 4);
                } else {
                    for (int b = 0; b < Rw; ++b) d = (d << 8) | q[i * Rw + b];
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

// Hours of the block (B = 32*Q) owned by lane L: for Q <= 4 the Q contiguous
// hours L*Q .. L*Q+Q-1 (one Q-wide vector load); for Q = 8 the hours
// 4L .. 4L+3 and 128+4L .. 128+4L+3 (two float4 loads, each instruction a
// contiguous 512-byte span).  A warp reads one whole slab row per neighbor.
__device__ __forceinline__ int lane_hour(int Q, int lane, int q)
{
    return Q <= 4 ? lane * Q + q : 128 * (q >> 2) + 4 * lane + (q & 3);
}

template <int Q> struct SlabVec;
template <> struct SlabVec<1> { using T = float; };
template <> struct SlabVec<2> { using T = float2; };
template <> struct SlabVec<4> { using T = float4; };
template <> struct SlabVec<8> { using T = float4; };   // two float4 per lane

template <int Q>
__device__ __forceinline__ void fma_row(float (&acc)[Q], float w, const float* __restrict__ row, int lane)
{
    if constexpr (Q == 1) {
        acc[0] = fmaf(w, __ldg(row + lane), acc[0]);
    } else if constexpr (Q == 2) {
        const float2 x = __ldg(reinterpret_cast<const float2*>(row) + lane);
        acc[0] = fmaf(w, x.x, acc[0]);
        acc[1] = fmaf(w, x.y, acc[1]);
    } else {
#pragma unroll
        for (int h = 0; h < Q / 4; ++h) {
            const float4 x = __ldg(reinterpret_cast<const float4*>(row) + lane + 32 * h);
            acc[4 * h] = fmaf(w, x.x, acc[4 * h]);
            acc[4 * h + 1] = fmaf(w, x.y, acc[4 * h + 1]);
            acc[4 * h + 2] = fmaf(w, x.z, acc[4 * h + 2]);
            acc[4 * h + 3] = fmaf(w, x.w, acc[4 * h + 3]);
        }
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
#pragma unroll 8
    for (int t = 0; t < n; ++t) {
        const float2 x = wg[t];
        fma_row<Q>(acc, x.x, slab + (size_t)__float_as_int(x.y) * (32 * Q), lane);
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

// Voxels are visited in `order` (tile-major, see k_tile_order), CTA b taking
// groups of kReflWarps consecutive entries: the warps of a CTA hold nearby
// voxels (shared slab rows in L1) and all CTAs together sweep a compact
// window of the DSM (its slab rows stay in L2).
template <int Q, int FMT>
__global__ void __launch_bounds__(kReflWarps * 32)
k_reflect_block(float4* __restrict__ geo_n_, float4* __restrict__ geo_p_, int N, int T,
                const uint32_t* __restrict__ shadow, int words32, const HourEntry* __restrict__ table,
                int j0, const float* __restrict__ slab, NeighborLists nl, Accum acc,
                const int* __restrict__ order, int* err)
{
    __shared__ float2 s_wg[kReflWarps][32];
    __shared__ int4 s_runs[kReflWarps][8];
    const float4* geo_n = geo_n_;
    const float4* geo_p = geo_p_;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int grp = blockIdx.x; grp * kReflWarps < N; grp += gridDim.x) {
        const int i = grp * kReflWarps + warp;
        if (i >= N) continue;
        const int v = order ? __ldg(order + i) : i;
        const float4 me_p = __ldg(geo_p + v);
        const float4 me_n = __ldg(geo_n + v);
        float r[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) r[q] = 0.0f;
        auto chunk = [&](int g) { slab_chunk<Q>(g, me_p, me_n, geo_p, T, s_wg[warp], slab, lane, r); };
        if (FMT == 0) {
            csr_for_each_chunk(nl.offsets, nl.ids, v, lane, chunk);
        } else {
            const long long b0 = nl.offsets[v];
            barle_for_each_chunk(nl.bytes, b0, nl.offsets[v + 1] - b0, lane, s_runs[warp], err, chunk);
        }
        // the voxel's own direct + diffuse for its hours, added to R
        float sum = 0.0f;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const HourEntry e = table[j0 + lane_hour(Q, lane, q)];
            sum += solar_I(me_n, e, shadow_bit(shadow, words32, v, e.dense)) + r[q];
        }
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
    // shared by the threads of several contexts: written once, same value
    static std::atomic<int> cached{0};
    int sms = cached.load(std::memory_order_relaxed);
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
        cached.store(sms, std::memory_order_relaxed);
    }
    const long long need = ((long long)N + kReflWarps - 1) / kReflWarps;
    const long long cap = (long long)sms * 8;
    return (int)(need < cap ? need : cap);
}

template <int Q>
cudaError_t launch_block_q(const DevGeom& g, int N, int T, const uint32_t* shadow, int words32,
                           const HourEntry* table, int j0, const float* slab, const NeighborLists& nl,
                           const Accum& acc, const int* order, int* err, cudaStream_t st)
{
    const int grid = refl_grid(N);
    if (nl.format == 0)
        k_reflect_block<Q, 0><<<grid, kReflWarps * 32, 0, st>>>(g.geo_n, g.geo_p, N, T, shadow, words32,
                                                              table, j0, slab, nl, acc, order, err);
    else
        k_reflect_block<Q, 1><<<grid, kReflWarps * 32, 0, st>>>(g.geo_n, g.geo_p, N, T, shadow, words32,
                                                              table, j0, slab, nl, acc, order, err);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_reflect_block(const DevGeom& g, int N, int T, const uint32_t* shadow,
                                 int words32, const HourEntry* table, int j0, int B,
                                 const float* slab, const NeighborLists& nl, const Accum& acc,
                                 const int* order, int* err, cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    switch (B) {
    case 32: return launch_block_q<1>(g, N, T, shadow, words32, table, j0, slab, nl, acc, order, err, st);
    case 64: return launch_block_q<2>(g, N, T, shadow, words32, table, j0, slab, nl, acc, order, err, st);
    case 128: return launch_block_q<4>(g, N, T, shadow, words32, table, j0, slab, nl, acc, order, err, st);
    case 256: return launch_block_q<8>(g, N, T, shadow, words32, table, j0, slab, nl, acc, order, err, st);
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

// Visiting order of the reflection pass: cells in 32 x 32 tiles (tiles in
// serpentine row order, cells in Morton order inside a tile), each cell's
// top voxel and walls together.  Built as a counting sort keyed by the cell
// position in that order: count voxels per cell, exclusive scan, scatter
// with per-cell cursors.  The order of walls inside a cell is arbitrary and
// does not affect results (every voxel is reduced by its own warp).
namespace {
constexpr int kTileBits = 5;   // 32 x 32 cell tiles

__device__ __forceinline__ unsigned spread5(unsigned x)
{
    x &= 31u;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}

__device__ __forceinline__ long long cell_pos(int c, int W, int ntx)
{
    const int x = c % W, y = c / W;
    const int tx = x >> kTileBits, ty = y >> kTileBits;
    const long long tile = (long long)ty * ntx + ((ty & 1) ? (ntx - 1 - tx) : tx);
    return (tile << (2 * kTileBits)) | (spread5((unsigned)x) | (spread5((unsigned)y) << 1));
}

__global__ void k_order_count(const int* __restrict__ pp, int N, int T, int W, int ntx, int* __restrict__ cnt,
                              int* __restrict__ first_wall)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const long long pos = cell_pos(pp[v], W, ntx);
    atomicAdd(cnt + pos, 1);
    if (v >= T) atomicMin(first_wall + pos, v);
}

// Deterministic placement: the top voxel first, then the cell's walls in
// index order (they are contiguous by the voxel layout of src/main.cpp:112-127).
// A cell whose walls are not contiguous sets *flag and the fallback below
// places every voxel with atomic cursors instead (correct, order within a
// cell then arbitrary).
__global__ void k_order_scatter(const int* __restrict__ pp, int N, int T, int W, int ntx,
                                const int* __restrict__ cnt, const long long* __restrict__ base,
                                const int* __restrict__ first_wall, int* __restrict__ order, int* __restrict__ flag)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const long long pos = cell_pos(pp[v], W, ntx);
    const long long rank = v < T ? 0 : 1 + (long long)v - first_wall[pos];
    if (rank < cnt[pos]) order[base[pos] + rank] = v;
    else atomicOr(flag, 1);
}

__global__ void k_order_scatter_fallback(const int* __restrict__ pp, int N, int W, int ntx,
                                         unsigned long long* __restrict__ cursor, int* __restrict__ order,
                                         const int* __restrict__ flag)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N || *flag == 0) return;
    order[atomicAdd(cursor + cell_pos(pp[v], W, ntx), 1ull)] = v;
}
}  // namespace

long long order_positions(int W, int H)
{
    const long long ntx = (W + (1 << kTileBits) - 1) >> kTileBits;
    const long long nty = (H + (1 << kTileBits) - 1) >> kTileBits;
    return ntx * nty << (2 * kTileBits);
}

cudaError_t launch_voxel_order(const int* pix_parent, int N, int T, int W, int H, int* counts,
                               int* first_wall, long long* cursor, long long* scan_tmp, int* order,
                               cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    const int ntx = (W + (1 << kTileBits) - 1) >> kTileBits;
    const long long npos = order_positions(W, H);
    int* flag = first_wall + npos;
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * npos, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(first_wall, 0x7F, sizeof(int) * npos, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(flag, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    k_order_count<<<(N + 255) / 256, 256, 0, st>>>(pix_parent, N, T, W, ntx, counts, first_wall);
    e = launch_scan_counts(counts, (int)npos, 0, cursor, scan_tmp, nullptr, st);
    if (e != cudaSuccess) return e;
    k_order_scatter<<<(N + 255) / 256, 256, 0, st>>>(pix_parent, N, T, W, ntx, counts, cursor, first_wall,
                                                    order, flag);
    k_order_scatter_fallback<<<(N + 255) / 256, 256, 0, st>>>(pix_parent, N, W, ntx,
                                                             reinterpret_cast<unsigned long long*>(cursor),
                                                             order, flag);
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
