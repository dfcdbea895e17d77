// Tiled reflection: the hour-block product with the neighbor rows of a group
// of voxels staged through shared memory.
//
// R[v, h] = sum_g w(v, g) I[g, h] needs one slab row I[g, block] per
// (voxel, nonzero neighbor).  Voxels that are close in the visiting order see
// mostly the same cells: on the 256 x 256 city the union of the lists of 64
// consecutive voxels is 7.6x smaller than their sum (10.6x for 128).  So:
//
//   build (once per run, hour-independent): voxels are cut into aligned
//     groups of at most G positions of the visiting order (halved until the
//     group's nonzero entries fit kTileCap); per group, the union of its
//     cells (sorted descending, as the ba-RLE lists are) replaces the cells
//     in the weighted-list buffer, and each entry becomes (slot, w) with
//     slot = the cell's index in the union, entries of a voxel in ascending
//     slot order;
//   per hour block: a CTA takes a group; a producer warp streams the union
//     rows I[g, block] into a ring of shared-memory stages with
//     cp.async.bulk (one bulk copy per 1 KB row, completion counted on an
//     mbarrier); 16 consumer warps each own 4 voxels (G = 64: with 17
//     warps a sub-partition holds 5, which caps registers at 96 a thread,
//     room for 4 voxels x 8 hours of accumulators), keep their entry
//     windows in registers and apply the entries whose slot falls in the
//     current stage (lanes hold hours, FMA per hour as in k_reflect_group),
//     then add each voxel's own direct + diffuse and accumulate.
//
// Per voxel, entries are applied in ascending slot order = descending cell
// order, which is the ba-RLE list order, so on ba-RLE lists the result is
// bit-identical to the per-voxel kernel (group size 1).  Every wait on an
// mbarrier is bounded (kWaitNs): on expiry the kernel sets kErrWaitTimeout,
// stops, lets its own bulk copies land (bounded as well) and returns.
#include "solar_math.cuh"

namespace sgb {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kTileCap = 16384;             // entries of one group held by the build
constexpr int kBuildThreads = 512;
constexpr int kConsumerWarps = 16;
constexpr int kStages = 3;
constexpr int kStageBytes = 72 * 1024;
constexpr unsigned long long kWaitNs = 1000000000ull;   // 1 s
constexpr int kMaxDevices = 64;

// ---- grouping ----------------------------------------------------------------

// flag[p] = 1 where a group starts: the largest aligned block of size
// G, G/2, ..., 1 containing p whose entries fit kTileCap (blocks nest, so
// every member of a block picks the same block).
__global__ void k_tile_flags(int N, int G, const long long* __restrict__ woff, int* __restrict__ flag)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    int L = G;
    int b = p - p % L;
    while (L > 1) {
        const int e = min(b + L, N);
        if (woff[e] - woff[b] <= kTileCap) break;
        L >>= 1;
        b = p - p % L;
    }
    flag[p] = (p == b) ? 1 : 0;
}

__global__ void k_tile_starts(int N, const int* __restrict__ flag, const long long* __restrict__ pos,
                              int* __restrict__ start)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < N && flag[p]) start[pos[p]] = p;
    if (p == 0) start[pos[N]] = N;
}

// ---- build -------------------------------------------------------------------

__device__ __forceinline__ void block_bitonic(uint32_t* keys, float* vals, int n2, bool descending)
{
    for (int size = 2; size <= n2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < (n2 >> 1); t += blockDim.x) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const bool up = ((i & size) == 0) != descending;
                const uint32_t a = keys[i], b = keys[j];
                if ((a > b) == up) {
                    keys[i] = b;
                    keys[j] = a;
                    if (vals) {
                        const float x = vals[i];
                        vals[i] = vals[j];
                        vals[j] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// One CTA per group.  Shared memory: a hash set of the group's cells
// (2 x kTileCap slots, load <= 1/2), reused afterwards for the (voxel, slot)
// keys and weights; the union (kTileCap).
__global__ void __launch_bounds__(kBuildThreads)
k_tile_build(const int* __restrict__ start, const long long* __restrict__ woff, int* __restrict__ cells,
             float* __restrict__ wts, unsigned short* __restrict__ slots, int* __restrict__ unions,
             unsigned long long* __restrict__ rows_total, int* __restrict__ err)
{
    constexpr int kHashSlots = 2 * kTileCap;
    extern __shared__ __align__(16) uint32_t sm[];
    uint32_t* table = sm;                                     // [kHashSlots], key = cell + 1, 0 = empty
    uint32_t* keys = sm;                                      // [kTileCap] after the union is built
    float* vals = reinterpret_cast<float*>(sm + kTileCap);    // [kTileCap]
    uint32_t* uni = sm + kHashSlots;                          // [kTileCap]
    __shared__ int s_off[257];
    __shared__ int s_count;
    const int q = blockIdx.x;
    const int p0 = start[q], p1 = start[q + 1];
    const int nv = p1 - p0;
    const long long e0 = woff[p0];
    const long long nl = woff[p1] - e0;
    if (nl > kTileCap || nv > 256) {
        if (threadIdx.x == 0) {
            atomicOr(err, kErrListCapacity);
            unions[q] = 0;
        }
        return;
    }
    const int n = (int)nl;
    for (int j = threadIdx.x; j <= nv; j += blockDim.x) s_off[j] = (int)(woff[p0 + j] - e0);
    for (int i = threadIdx.x; i < kHashSlots; i += blockDim.x) table[i] = 0u;
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();

    // distinct cells: linear-probing insert; the inserting thread appends
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t key = (uint32_t)cells[e0 + i] + 1u;
        uint32_t h = (key * 2654435761u) >> 17;   // 15 bits: kHashSlots = 32768
        for (int probe = 0; probe < kHashSlots; ++probe) {
            const uint32_t prev = atomicCAS(&table[h], 0u, key);
            if (prev == 0u) {
                uni[atomicAdd(&s_count, 1)] = key;
                break;
            }
            if (prev == key) break;
            h = (h + 1u) & (kHashSlots - 1);
        }
    }
    __syncthreads();
    const int u = s_count;
    int u2 = 64;
    while (u2 < u) u2 <<= 1;
    for (int i = u + threadIdx.x; i < u2; i += blockDim.x) uni[i] = 0u;
    __syncthreads();
    block_bitonic(uni, nullptr, u2, true);   // descending cell order
    int* ucell = reinterpret_cast<int*>(uni);
    for (int i = threadIdx.x; i < u; i += blockDim.x) ucell[i] = (int)uni[i] - 1;
    __syncthreads();

    // entries -> (local voxel << 16 | slot), weights alongside
    int n2 = kBuildThreads;
    while (n2 < n) n2 <<= 1;
    bool unsorted = false;
    for (int i = threadIdx.x; i < n2; i += blockDim.x) {
        uint32_t k = 0xFFFFFFFFu;
        float w = 0.0f;
        if (i < n) {
            const int cell = cells[e0 + i];
            int lo = 0, hi = u - 1;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (ucell[mid] > cell) lo = mid + 1; else hi = mid;
            }
            int a = 0, b = nv;   // largest j with s_off[j] <= i
            while (b - a > 1) {
                const int mid = (a + b) >> 1;
                if (s_off[mid] <= i) a = mid; else b = mid;
            }
            k = ((uint32_t)a << 16) | (uint32_t)lo;
            w = wts[e0 + i];
        }
        keys[i] = k;
        vals[i] = w;
    }
    __syncthreads();
    for (int i = threadIdx.x + 1; i < n; i += blockDim.x) unsorted |= keys[i] < keys[i - 1];
    if (__syncthreads_or(unsorted)) block_bitonic(keys, vals, n2, false);

    for (int i = threadIdx.x; i < u; i += blockDim.x) cells[e0 + i] = ucell[i];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        slots[e0 + i] = (unsigned short)(keys[i] & 0xFFFFu);
        wts[e0 + i] = vals[i];
    }
    if (threadIdx.x == 0) {
        unions[q] = u;
        atomicAdd(rows_total, (unsigned long long)u);
    }
}

// ---- per hour block ----------------------------------------------------------

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of the given parity; false if it did not complete
// within kWaitNs or another role gave up (abort != 0).
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, const volatile int* abort)
{
    unsigned long long t0 = 0;
    for (unsigned i = 0;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 63u) {
            if (abort && *abort) return false;
            const unsigned long long t = global_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > kWaitNs) return false;
        }
    }
}

__device__ __forceinline__ void mbar_arrive(unsigned bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

template <int Q>
__device__ __forceinline__ void global_row(float (&x)[Q], const float* __restrict__ row, int lane)
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

// Same lane layout from a shared-memory row.
template <int Q>
__device__ __forceinline__ void smem_row(float (&x)[Q], const float* row, int lane)
{
    if constexpr (Q == 1) {
        x[0] = row[lane];
    } else if constexpr (Q == 2) {
        const float2 a = reinterpret_cast<const float2*>(row)[lane];
        x[0] = a.x; x[1] = a.y;
    } else {
#pragma unroll
        for (int h = 0; h < Q / 4; ++h) {
            const float4 a = reinterpret_cast<const float4*>(row)[lane + 32 * h];
            x[4 * h] = a.x; x[4 * h + 1] = a.y; x[4 * h + 2] = a.z; x[4 * h + 3] = a.w;
        }
    }
}

__device__ __forceinline__ void tile_accumulate(const Accum& a, int v, float x)
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

// Entry window of one voxel, relative to the group's first entry: lane l
// holds entry wbase + l.
struct Window {
    int e, end, wbase;
    int slot;
    float w;
};

template <int Q, int VPW>
__global__ void __launch_bounds__((kConsumerWarps + 1) * 32, 1)
k_reflect_tile(const float* __restrict__ slab, TileLists tl, const int* __restrict__ order, Accum acc,
               int* __restrict__ err)
{
    constexpr int kRowFloats = 32 * Q;
    constexpr int kRowBytes = kRowFloats * 4;
    constexpr int R = kStageBytes / kRowBytes;   // union rows per stage
    constexpr int kCellsPerLane = (R + 31) / 32;
    extern __shared__ __align__(128) float stage_mem[];
    __shared__ __align__(8) unsigned long long bar_full[kStages], bar_empty[kStages];
    __shared__ volatile int s_abort;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar_full[s])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bar_empty[s])),
                         "r"(kConsumerWarps));
        }
        s_abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == kConsumerWarps) {
        // ---- producer: union rows of each group into the stage ring
        long long k = 0;   // chunks issued by this CTA
        bool ok = true;
        for (int q = blockIdx.x; q < tl.NG && ok; q += gridDim.x) {
            const long long ubase = tl.woff[tl.start[q]];
            const int u = tl.unions[q];
            for (int c0 = 0; c0 < u && ok; c0 += R, ++k) {
                const int s = (int)(k % kStages);
                const int rows = min(R, u - c0);
                int cell[kCellsPerLane];   // loaded before the wait so the wait hides their latency
#pragma unroll
                for (int i = 0; i < kCellsPerLane; ++i) {
                    const int r = lane + 32 * i;
                    cell[i] = r < rows ? __ldg(tl.cells + ubase + c0 + r) : 0;
                }
                if (k >= kStages)
                    ok = mbar_wait(smem_u32(&bar_empty[s]), (unsigned)(((k / kStages) - 1) & 1), &s_abort);
                if (!ok) break;
                const unsigned full = smem_u32(&bar_full[s]);
                if (lane == 0) mbar_expect(full, (unsigned)(rows * kRowBytes));
                __syncwarp();
                const unsigned dst = smem_u32(stage_mem) + (unsigned)(s * kStageBytes);
#pragma unroll
                for (int i = 0; i < kCellsPerLane; ++i) {
                    const int r = lane + 32 * i;
                    if (r < rows)
                        bulk_g2s(dst + (unsigned)(r * kRowBytes), slab + (size_t)cell[i] * kRowFloats, kRowBytes,
                                 full);
                }
            }
        }
        if (!ok) {
            if (lane == 0) atomicOr(err, kErrWaitTimeout);
            s_abort = 1;
        }
        // let this CTA's copies land before it exits
        if (lane == 0) {
            for (long long j = (k > kStages ? k - kStages : 0); j < k; ++j)
                mbar_wait(smem_u32(&bar_full[j % kStages]), (unsigned)((j / kStages) & 1), nullptr);
        }
        return;
    }

    // ---- consumers
    long long k = 0;
    for (int q = blockIdx.x; q < tl.NG; q += gridDim.x) {
        const int p0 = tl.start[q], p1 = tl.start[q + 1];
        const int u = tl.unions[q];
        const long long gbase = tl.woff[p0];
        const unsigned short* gslots = tl.slots + gbase;
        const float* gw = tl.weights + gbase;
        float a[VPW][Q];
        Window win[VPW];
#pragma unroll
        for (int t = 0; t < VPW; ++t) {
            const int p = p0 + warp + kConsumerWarps * t;
            const bool has = p < p1;
            win[t].e = has ? (int)(tl.woff[p] - gbase) : 0;
            win[t].end = has ? (int)(tl.woff[p + 1] - gbase) : 0;
            win[t].wbase = win[t].e - 32;   // empty window: loaded on first use
            win[t].slot = 0x7FFFFFFF;
            win[t].w = 0.0f;
#pragma unroll
            for (int h = 0; h < Q; ++h) a[t][h] = 0.0f;
        }
        for (int c0 = 0; c0 < u; c0 += R, ++k) {
            const int s = (int)(k % kStages);
            if (!mbar_wait(smem_u32(&bar_full[s]), (unsigned)((k / kStages) & 1), &s_abort)) {
                if (lane == 0) atomicOr(err, kErrWaitTimeout);
                s_abort = 1;
                return;
            }
            const float* rows = stage_mem + (size_t)s * (kStageBytes / 4);
            const int lim = c0 + R;
#pragma unroll
            for (int t = 0; t < VPW; ++t) {
                Window& W = win[t];
                while (W.e < W.end) {
                    if (W.e - W.wbase >= 32) {
                        W.wbase = W.e;
                        const int i = W.e + lane;
                        W.slot = i < W.end ? (int)__ldg(gslots + i) : 0x7FFFFFFF;
                        W.w = i < W.end ? __ldg(gw + i) : 0.0f;
                    }
                    const int m = __popc(__ballot_sync(kFull, W.slot < lim));   // sorted: a prefix
                    const int cur = W.e - W.wbase;
                    if (cur >= m) break;
                    int j = cur;
                    for (; j + 1 < m; j += 2) {
                        const int s0 = __shfl_sync(kFull, W.slot, j) - c0;
                        const int s1 = __shfl_sync(kFull, W.slot, j + 1) - c0;
                        const float w0 = __shfl_sync(kFull, W.w, j);
                        const float w1 = __shfl_sync(kFull, W.w, j + 1);
                        float x0[Q], x1[Q];
                        smem_row<Q>(x0, rows + (size_t)s0 * kRowFloats, lane);
                        smem_row<Q>(x1, rows + (size_t)s1 * kRowFloats, lane);
#pragma unroll
                        for (int h = 0; h < Q; ++h) a[t][h] = fmaf(w0, x0[h], a[t][h]);
#pragma unroll
                        for (int h = 0; h < Q; ++h) a[t][h] = fmaf(w1, x1[h], a[t][h]);
                    }
                    if (j < m) {
                        const int s0 = __shfl_sync(kFull, W.slot, j) - c0;
                        const float w0 = __shfl_sync(kFull, W.w, j);
                        float x0[Q];
                        smem_row<Q>(x0, rows + (size_t)s0 * kRowFloats, lane);
#pragma unroll
                        for (int h = 0; h < Q; ++h) a[t][h] = fmaf(w0, x0[h], a[t][h]);
                    }
                    W.e = W.wbase + m;
                    if (m < 32) break;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar_empty[s]));
        }
#pragma unroll
        for (int t = 0; t < VPW; ++t) {
            const int p = p0 + warp + kConsumerWarps * t;
            if (p < p1) {
                // the voxel's own direct + diffuse is its own slab row
                const int v = __ldg(order + p);
                float own[Q];
                global_row<Q>(own, slab + (size_t)v * kRowFloats, lane);
                float sum = 0.0f;
#pragma unroll
                for (int h = 0; h < Q; ++h) sum += own[h] + a[t][h];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
                if (lane == 0) tile_accumulate(acc, v, sum);
            }
        }
    }
}

int tile_sms()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

template <int Q, int VPW>
cudaError_t tile_q(const float* slab, const TileLists& tl, const int* order, const Accum& acc, int* err,
                   cudaStream_t st)
{
    const size_t smem = (size_t)kStages * kStageBytes;
    static bool attr[kMaxDevices] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        const cudaError_t e = cudaFuncSetAttribute(k_reflect_tile<Q, VPW>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    const int grid = tl.NG < tile_sms() ? tl.NG : tile_sms();
    k_reflect_tile<Q, VPW><<<grid, (kConsumerWarps + 1) * 32, smem, st>>>(slab, tl, order, acc, err);
    return cudaGetLastError();
}

}  // namespace

int tile_voxels_per_warp(int G) { return G / kConsumerWarps; }

cudaError_t launch_tile_groups(int N, int G, const long long* woff, int* flag, long long* pos,
                               long long* scan_tmp, int* start, cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((N + 255) / 256);
    k_tile_flags<<<grid, 256, 0, st>>>(N, G, woff, flag);
    cudaError_t e = launch_scan_counts(flag, N, 0, pos, scan_tmp, nullptr, st);
    if (e != cudaSuccess) return e;
    k_tile_starts<<<grid, 256, 0, st>>>(N, flag, pos, start);
    return cudaGetLastError();
}

cudaError_t launch_tile_build(int NG, const int* start, const long long* woff, int* cells, float* wts,
                              unsigned short* slots, int* unions, long long* rows_total, int* err, cudaStream_t st)
{
    if (NG <= 0) return cudaSuccess;
    const size_t smem = (size_t)3 * kTileCap * 4;
    static bool attr[kMaxDevices] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
        const cudaError_t e = cudaFuncSetAttribute(k_tile_build, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
        if (e != cudaSuccess) return e;
        attr[dev] = true;
    }
    cudaError_t e = cudaMemsetAsync(rows_total, 0, sizeof(long long), st);
    if (e != cudaSuccess) return e;
    k_tile_build<<<NG, kBuildThreads, smem, st>>>(start, woff, cells, wts, slots, unions,
                                                  reinterpret_cast<unsigned long long*>(rows_total), err);
    return cudaGetLastError();
}

cudaError_t launch_reflect_tile(int B, const float* slab, const TileLists& tl, const int* order, const Accum& acc,
                                int* err, cudaStream_t st)
{
    if (tl.NG <= 0) return cudaSuccess;
    const int vpw = tl.G / kConsumerWarps;
    if (vpw == 4) {
        switch (B) {
        case 64: return tile_q<2, 4>(slab, tl, order, acc, err, st);
        case 128: return tile_q<4, 4>(slab, tl, order, acc, err, st);
        case 256: return tile_q<8, 4>(slab, tl, order, acc, err, st);
        default: return cudaErrorInvalidValue;
        }
    }
    return cudaErrorInvalidValue;
}

}  // namespace sgb
