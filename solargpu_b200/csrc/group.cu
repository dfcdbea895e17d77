// Grouped reflection: the hour-block product with neighbor sharing.
//
// The reflection sum R[v, h] = sum_g w(v, g) I[g, h] is bound by moving
// slab rows I[g, block] through L1: one row per (voxel, neighbor).  Voxels
// that are close in the visiting order (same 32 x 32 tile, Morton-adjacent)
// see many of the same cells, so here they are processed V at a time:
//
//   build (once per run, hour-independent): for each group of V consecutive
//     voxels of the visiting order, every nonzero weight w(v, g) of the V
//     lists is computed (same FP32 formula as the per-block kernel,
//     reflection_kernels.cu:18-38), the (g, v, w) triples are sorted by g in
//     shared memory and merged into union entries {g, w[0..V-1]}, sorted by
//     cell, stored once;
//   per hour block: one warp per group streams its union entries, loads each
//     slab row once and applies the V weights (V FMAs per loaded value), then
//     adds each voxel's own direct + diffuse and accumulates per voxel.
//
// The lists are decoded exactly once per run (CSR, or ba-RLE through the
// warp-parallel decoder).  Groups whose nonzero-neighbor total exceeds the
// shared-memory capacity are written unmerged (one nonzero weight per entry),
// which is slower but exact.  Entry order is deterministic, so results are
// bit-reproducible run to run.
#include "solar_math.cuh"

#include <atomic>

namespace sgb {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kBuildWarps = 4;
constexpr int kBuildCap = 2048;        // (cell, slot, w) triples per group held in shared memory
constexpr int kGroupWarps = 8;

__device__ __forceinline__ unsigned lanemask_lt(int lane) { return (1u << lane) - 1u; }

// ---- list iteration (same decoder as the per-block kernel in reflect.cu) ----

template <typename F>
__device__ __forceinline__ void csr_chunks(const long long* __restrict__ off, const int* __restrict__ ids,
                                           int v, int lane, F&& f)
{
    const long long s = off[v], e = off[v + 1];
    for (long long c = s; c < e; c += 32) {
        const long long i = c + lane;
        f(i < e ? __ldg(ids + i) - 1 : -1);
    }
}

template <typename F>
__device__ __forceinline__ void barle_chunks(const unsigned char* __restrict__ bytes, long long base,
                                             long long size, int lane, int* err, F&& f)
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
            f((valid && val > 0u) ? (int)(val - 1u) : -1);
        }
        cur = pay_base + total_pay;
    }
}

template <int FMT, typename F>
__device__ __forceinline__ void list_chunks(const NeighborLists& nl, int v, int lane, int* err, F&& f)
{
    if (FMT == 0) {
        csr_chunks(nl.offsets, nl.ids, v, lane, f);
    } else {
        const long long b0 = nl.offsets[v];
        barle_chunks(nl.bytes, b0, nl.offsets[v + 1] - b0, lane, err, f);
    }
}

// ---- build ------------------------------------------------------------------
//
// Phase A (one warp per voxel, no shared memory): the nonzero weights of
// each voxel's list, in visiting order p = 0..N-1 -> weighted lists
// (cell, w) at woff[p].  With V = 1 these are the union entries.
// Phase B (V > 1, one warp per group): the entries of the group's V voxels
// are contiguous in the weighted lists; they are sorted by (cell, slot) in
// shared memory and merged into entries {cell, w[0..V-1]}.

template <int FMT, int PASS>
__global__ void __launch_bounds__(256)
k_wlist(const float4* __restrict__ geo_n, const float4* __restrict__ geo_p, int N, int T,
        NeighborLists nl, const int* __restrict__ order, int* __restrict__ counts,
        const long long* __restrict__ woff, int* __restrict__ cells, float* __restrict__ wts, int* err)
{
    const int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (p >= N) return;
    const int v = order[p];
    const float4 me_p = __ldg(geo_p + v), me_n = __ldg(geo_n + v);
    long long e = PASS == 1 ? woff[p] : 0;
    list_chunks<FMT>(nl, v, lane, err, [&](int g) {
        float w = 0.0f;
        if (g >= 0 && g < T) w = refl_weight(me_p, me_n, __ldg(geo_p + g));
        const unsigned bal = __ballot_sync(kFull, w != 0.0f);
        if (PASS == 1 && w != 0.0f) {
            const long long o = e + __popc(bal & lanemask_lt(lane));
            cells[o] = g;
            wts[o] = w;
        }
        e += __popc(bal);
    });
    if (PASS == 0 && lane == 0) counts[p] = (int)e;
}

// PASS 0: counts[q] = union entries of group q.  PASS 1: writes them at goff[q].
template <int V, int PASS>
__global__ void __launch_bounds__(kBuildWarps * 32)
k_group_merge(int N, const long long* __restrict__ woff, const int* __restrict__ wcell,
              const float* __restrict__ wts, int* __restrict__ counts, const long long* __restrict__ goff,
              int* __restrict__ cell_out, float* __restrict__ w_out)
{
    extern __shared__ uint32_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* keys = smem + warp * (2 * kBuildCap);
    float* vals = reinterpret_cast<float*>(keys + kBuildCap);
    const int q = blockIdx.x * kBuildWarps + warp;
    const int G = (N + V - 1) / V;
    if (q >= G) return;
    const int p0 = q * V, gs = min(V, N - p0);
    long long bnd[V + 1];
#pragma unroll
    for (int s = 0; s <= V; ++s) bnd[s] = woff[p0 + min(s, gs)];
    const long long e0 = bnd[0];
    const int n = (int)(bnd[V] - e0);
    if (n > kBuildCap) {
        // Too many for shared memory: unmerged, one nonzero weight per entry.
        if (PASS == 0) { if (lane == 0) counts[q] = n; return; }
        const long long o0 = goff[q];
        for (int i = lane; i < n; i += 32) {
            int s = 0;
#pragma unroll
            for (int t = 1; t < V; ++t) s += (e0 + i >= bnd[t]) ? 1 : 0;
            cell_out[o0 + i] = wcell[e0 + i];
#pragma unroll
            for (int t = 0; t < V; ++t) w_out[(o0 + i) * V + t] = (t == s) ? wts[e0 + i] : 0.0f;
        }
        return;
    }
    int n2 = 32;
    while (n2 < n) n2 <<= 1;
    for (int i = lane; i < n2; i += 32) {
        if (i < n) {
            int s = 0;
#pragma unroll
            for (int t = 1; t < V; ++t) s += (e0 + i >= bnd[t]) ? 1 : 0;
            keys[i] = ((uint32_t)wcell[e0 + i] << 3) | (uint32_t)s;
            vals[i] = wts[e0 + i];
        } else {
            keys[i] = 0xFFFFFFFFu;
            vals[i] = 0.0f;
        }
    }
    __syncwarp();
    for (int size = 2; size <= n2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < (n2 >> 1); t += 32) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const bool up = (i & size) == 0;
                const uint32_t a = keys[i], b = keys[j];
                if ((a > b) == up) {
                    keys[i] = b; keys[j] = a;
                    const float x = vals[i]; vals[i] = vals[j]; vals[j] = x;
                }
            }
            __syncwarp();
        }
    }
    if (PASS == 0) {
        int distinct = 0;
        for (int i0 = 0; i0 < n; i0 += 32) {
            const int i = i0 + lane;
            const bool head = i < n && (i == 0 || (keys[i] >> 3) != (keys[i - 1] >> 3));
            distinct += __popc(__ballot_sync(kFull, head));
        }
        if (lane == 0) counts[q] = distinct;
        return;
    }
    const long long o0 = goff[q];
    const long long ne = goff[q + 1] - o0;
    for (long long i = lane; i < ne * V; i += 32) w_out[o0 * V + i] = 0.0f;
    __syncwarp();
    int run = -1;
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        const bool head = i < n && (i == 0 || (keys[i] >> 3) != (keys[i - 1] >> 3));
        const unsigned bal = __ballot_sync(kFull, head);
        const int r = run + __popc(bal & (lanemask_lt(lane) | (1u << lane)));
        if (i < n) {
            if (head) cell_out[o0 + r] = (int)(keys[i] >> 3);
            w_out[(o0 + r) * V + (keys[i] & 7u)] = vals[i];
        }
        run += __popc(bal);
    }
}

// ---- per hour block ---------------------------------------------------------

__device__ __forceinline__ int lane_hour(int Q, int lane, int q)
{
    return Q <= 4 ? lane * Q + q : 128 * (q >> 2) + 4 * lane + (q & 3);
}

template <int Q>
__device__ __forceinline__ void load_row(float (&x)[Q], const float* __restrict__ row, int lane)
{
    if constexpr (Q == 1) {
        x[0] = __ldg(row + lane);
    } else if constexpr (Q == 2) {
        const float2 a = __ldg(reinterpret_cast<const float2*>(row) + lane);
        x[0] = a.x; x[1] = a.y;
    } else {
#pragma unroll
        for (int h = 0; h < Q / 4; ++h) {
            const float4 a = __ldg(reinterpret_cast<const float4*>(row) + lane + 32 * h);
            x[4 * h] = a.x; x[4 * h + 1] = a.y; x[4 * h + 2] = a.z; x[4 * h + 3] = a.w;
        }
    }
}

__device__ __forceinline__ void accumulate_g(const Accum& a, int v, float x)
{
    if (a.mode == 0) {
        a.f64[v] += (double)x;
    } else if (a.mode == 1) {
        const float y = __fsub_rn(x, a.comp[v]);
        const float s = a.f32[v];
        const float t = __fadd_rn(s, y);
        a.comp[v] = __fsub_rn(__fsub_rn(t, s), y);
        a.f32[v] = t;
    } else {
        a.f32[v] = __fadd_rn(a.f32[v], x);
    }
}

template <int Q, int V>
__global__ void __launch_bounds__(kGroupWarps * 32)
k_reflect_group(int N, const float* __restrict__ slab, const long long* __restrict__ goff,
                const int* __restrict__ gcell, const float* __restrict__ gw, const int* __restrict__ order,
                Accum acc)
{
    __shared__ int s_cell[kGroupWarps][32];
    __shared__ __align__(16) float s_w[kGroupWarps][32][V];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int G = (N + V - 1) / V;
    for (int q = blockIdx.x * kGroupWarps + warp; q < G; q += gridDim.x * kGroupWarps) {
        float a[V][Q];
#pragma unroll
        for (int s = 0; s < V; ++s)
#pragma unroll
            for (int h = 0; h < Q; ++h) a[s][h] = 0.0f;
        const long long e0 = goff[q], e1 = goff[q + 1];
        for (long long c = e0; c < e1; c += 32) {
            const int m = (int)min(32LL, e1 - c);
            if (lane < m) {
                s_cell[warp][lane] = __ldg(gcell + c + lane);
                if constexpr (V >= 4) {
                    const float4* src = reinterpret_cast<const float4*>(gw + (c + lane) * V);
#pragma unroll
                    for (int t = 0; t < V / 4; ++t)
                        reinterpret_cast<float4*>(s_w[warp][lane])[t] = __ldg(src + t);
                } else {
#pragma unroll
                    for (int t = 0; t < V; ++t) s_w[warp][lane][t] = __ldg(gw + (c + lane) * V + t);
                }
            }
            __syncwarp();
#pragma unroll (V <= 1 ? 8 : V == 2 ? 4 : 2)
            for (int t = 0; t < m; ++t) {
                float x[Q];
                load_row<Q>(x, slab + (size_t)s_cell[warp][t] * (32 * Q), lane);
                float w[V];
                if constexpr (V >= 4) {
#pragma unroll
                    for (int u = 0; u < V / 4; ++u) {
                        const float4 ww = reinterpret_cast<const float4*>(s_w[warp][t])[u];
                        w[4 * u] = ww.x; w[4 * u + 1] = ww.y; w[4 * u + 2] = ww.z; w[4 * u + 3] = ww.w;
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < V; ++u) w[u] = s_w[warp][t][u];
                }
#pragma unroll
                for (int s = 0; s < V; ++s)
#pragma unroll
                    for (int h = 0; h < Q; ++h) a[s][h] = fmaf(w[s], x[h], a[s][h]);
            }
            __syncwarp();
        }
        const int gs = min(V, N - q * V);
#pragma unroll
        for (int s = 0; s < V; ++s) {
            if (s < gs) {
                // the voxel's own direct + diffuse: its slab row (k_solar_slab
                // computes rows for every voxel when the slab serves this kernel)
                const int v = __ldg(order + q * V + s);
                float own[Q];
                load_row<Q>(own, slab + (size_t)v * (32 * Q), lane);
                float sum = 0.0f;
#pragma unroll
                for (int h = 0; h < Q; ++h) sum += own[h] + a[s][h];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
                if (lane == 0) accumulate_g(acc, v, sum);
            }
        }
    }
}

int sm_count()
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
    return sms;
}

template <int V, int PASS>
cudaError_t merge_pass(int N, const long long* woff, const int* wcell, const float* wts, int* counts,
                       const long long* goff, int* cell, float* w, cudaStream_t st)
{
    const size_t smem = (size_t)kBuildWarps * 2 * kBuildCap * sizeof(uint32_t);
    cudaError_t e = cudaFuncSetAttribute(k_group_merge<V, PASS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    const int G = (N + V - 1) / V;
    k_group_merge<V, PASS><<<(G + kBuildWarps - 1) / kBuildWarps, kBuildWarps * 32, smem, st>>>(
        N, woff, wcell, wts, counts, goff, cell, w);
    return cudaGetLastError();
}

template <int Q, int V>
cudaError_t group_q(int N, const float* slab, const GroupLists& gl, const int* order, const Accum& acc,
                    cudaStream_t st)
{
    const int G = (N + V - 1) / V;
    const long long need = ((long long)G + kGroupWarps - 1) / kGroupWarps;
    const long long cap = (long long)sm_count() * 8;
    const int grid = (int)(need < cap ? need : cap);
    k_reflect_group<Q, V><<<grid, kGroupWarps * 32, 0, st>>>(N, slab, gl.offsets, gl.cells, gl.weights, order,
                                                              acc);
    return cudaGetLastError();
}

}  // namespace

int group_count(int N, int V) { return (N + V - 1) / V; }

cudaError_t launch_weight_lists(int pass, const DevGeom& g, int N, int T, const NeighborLists& nl,
                                const int* order, int* counts, const long long* woff, int* cells,
                                float* wts, int* err, cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    const long long threads = (long long)N * 32;
    const unsigned grid = (unsigned)((threads + 255) / 256);
    if (nl.format == 0) {
        if (pass == 0) k_wlist<0, 0><<<grid, 256, 0, st>>>(g.geo_n, g.geo_p, N, T, nl, order, counts, woff, cells, wts, err);
        else k_wlist<0, 1><<<grid, 256, 0, st>>>(g.geo_n, g.geo_p, N, T, nl, order, counts, woff, cells, wts, err);
    } else {
        if (pass == 0) k_wlist<1, 0><<<grid, 256, 0, st>>>(g.geo_n, g.geo_p, N, T, nl, order, counts, woff, cells, wts, err);
        else k_wlist<1, 1><<<grid, 256, 0, st>>>(g.geo_n, g.geo_p, N, T, nl, order, counts, woff, cells, wts, err);
    }
    return cudaGetLastError();
}

cudaError_t launch_group_merge(int pass, int V, int N, const long long* woff, const int* wcell,
                               const float* wts, int* counts, const long long* goff, int* cell, float* w,
                               cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    switch (V) {
    case 2: return pass == 0 ? merge_pass<2, 0>(N, woff, wcell, wts, counts, goff, cell, w, st)
                             : merge_pass<2, 1>(N, woff, wcell, wts, counts, goff, cell, w, st);
    case 4: return pass == 0 ? merge_pass<4, 0>(N, woff, wcell, wts, counts, goff, cell, w, st)
                             : merge_pass<4, 1>(N, woff, wcell, wts, counts, goff, cell, w, st);
    case 8: return pass == 0 ? merge_pass<8, 0>(N, woff, wcell, wts, counts, goff, cell, w, st)
                             : merge_pass<8, 1>(N, woff, wcell, wts, counts, goff, cell, w, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_reflect_group(int N, int B, const float* slab, const GroupLists& gl, const int* order,
                                 const Accum& acc, cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    if (gl.V == 8) {
        switch (B) {
        case 32: return group_q<1, 8>(N, slab, gl, order, acc, st);
        case 64: return group_q<2, 8>(N, slab, gl, order, acc, st);
        case 128: return group_q<4, 8>(N, slab, gl, order, acc, st);
        default: return cudaErrorInvalidValue;
        }
    }
    if (gl.V == 4) {
        switch (B) {
        case 32: return group_q<1, 4>(N, slab, gl, order, acc, st);
        case 64: return group_q<2, 4>(N, slab, gl, order, acc, st);
        case 128: return group_q<4, 4>(N, slab, gl, order, acc, st);
        case 256: return group_q<8, 4>(N, slab, gl, order, acc, st);
        default: return cudaErrorInvalidValue;
        }
    }
    if (gl.V == 2) {
        switch (B) {
        case 64: return group_q<2, 2>(N, slab, gl, order, acc, st);
        case 128: return group_q<4, 2>(N, slab, gl, order, acc, st);
        case 256: return group_q<8, 2>(N, slab, gl, order, acc, st);
        case 512: return group_q<16, 2>(N, slab, gl, order, acc, st);
        default: return cudaErrorInvalidValue;
        }
    }
    if (gl.V == 1) {
        switch (B) {
        case 64: return group_q<2, 1>(N, slab, gl, order, acc, st);
        case 128: return group_q<4, 1>(N, slab, gl, order, acc, st);
        case 256: return group_q<8, 1>(N, slab, gl, order, acc, st);
        case 512: return group_q<16, 1>(N, slab, gl, order, acc, st);
        default: return cudaErrorInvalidValue;
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace sgb
