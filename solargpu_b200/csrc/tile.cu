// Tiled reflection: the hour-block product with the neighbor rows of a group
// of voxels staged through shared memory.
//
// R[v, h] = sum_g w(v, g) I[g, h] needs one slab row I[g, block] per
// (voxel, nonzero neighbor).  Voxels that are close in the visiting order see
// mostly the same cells: on the 256 x 256 city the union of the lists of 64
// consecutive voxels is 7.6x smaller than their sum, and 4 consecutive voxels
// share 1.9x.  So, once per run (hour-independent):
//
//   groups   aligned runs of at most 64 positions of the visiting order,
//            halved until the group's nonzero entries fit kTileCap;
//   union    the group's distinct cells, sorted descending (the ba-RLE list
//            order), replace the cells in the weighted-list buffer; each
//            entry gets its slot (index in the union);
//   quads    the slot lists of each 4 consecutive voxels are merged: one
//            entry per distinct slot with the 4 weights (0 where a voxel
//            lacks the slot);
//   chunks   the union is cut into chunks of R rows (what one shared-memory
//            stage holds); the merged entries are laid out chunk by chunk,
//            quads in order inside a chunk, with a table of quad offsets.
//
// Per hour block, a CTA per group in turn (persistent grid): 4 producer warps
// copy each chunk's R union rows I[g, block] (one cp.async.bulk per 1 KB
// row, one row per thread) plus its entry block and table into a stage;
// completion is counted in bytes on the stage's mbarrier.  16 consumer warps
// each own a quad: for every entry of the chunk, one shared-memory row read
// feeds 4 x Q FMAs per lane (lanes hold hours).  After the last chunk each
// voxel adds its own direct + diffuse (its own slab row) and accumulates.
//
// Per voxel the FMAs run in ascending slot order = descending cell order,
// with exact zero terms where the quad's other voxels have a slot, so on
// ba-RLE lists the result is bit-identical to the per-voxel kernel (group
// size 1).  Every wait on an mbarrier is bounded (kWaitNs): on expiry the
// kernel sets kErrWaitTimeout, stops, lets its bulk copies land (bounded as
// well) and returns.
#include "solar_math.cuh"

#include <atomic>

namespace sgb {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kTileCap = 16384;             // entries of one group held by the build
constexpr int kBuildThreads = 512;
constexpr int kConsumerWarps = 16;
constexpr int kProducerWarps = 4;            // 20 warps: 5 a sub-partition, 96 registers a thread
constexpr int kStages = 2;
constexpr unsigned long long kWaitNs = 1000000000ull;   // 1 s
constexpr int kMaxDevices = 64;
constexpr int kQuad = 4;                    // voxels merged per consumer warp

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

__device__ __forceinline__ void block_bitonic(uint32_t* keys, int n2, bool descending)
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
                }
            }
            __syncthreads();
        }
    }
}

// One CTA per group.  Shared memory: a hash set of the group's cells
// (2 x kTileCap slots, load <= 1/2) and the union (kTileCap).
__global__ void __launch_bounds__(kBuildThreads)
k_tile_build(const int* __restrict__ start, const long long* __restrict__ woff, int* __restrict__ cells,
             unsigned short* __restrict__ slots, int* __restrict__ unions,
             unsigned long long* __restrict__ rows_total, int* __restrict__ err)
{
    constexpr int kHashSlots = 2 * kTileCap;
    extern __shared__ __align__(16) uint32_t sm[];
    uint32_t* table = sm;                                     // [kHashSlots], key = cell + 1, 0 = empty
    uint32_t* uni = sm + kHashSlots;                          // [kTileCap]
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
    block_bitonic(uni, u2, true);   // descending cell order
    int* ucell = reinterpret_cast<int*>(uni);
    for (int i = threadIdx.x; i < u; i += blockDim.x) ucell[i] = (int)uni[i] - 1;
    __syncthreads();

    // each entry's slot (its cell's index in the union); entry order and
    // weights are unchanged (the quad merge sorts by slot)
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int cell = cells[e0 + i];
        int lo = 0, hi = u - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (ucell[mid] > cell) lo = mid + 1; else hi = mid;
        }
        slots[e0 + i] = (unsigned short)lo;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < u; i += blockDim.x) cells[e0 + i] = ucell[i];
    if (threadIdx.x == 0) {
        unions[q] = u;
        atomicAdd(rows_total, (unsigned long long)u);
    }
}

// ---- layout: merged quads, chunk-major -------------------------------------
//
// Consumer warp w of a group owns the quad of positions p0 + 4w .. p0 + 4w + 3.
// The slot lists of a quad's 4 voxels are merged (one entry per distinct
// slot, the 4 weights alongside, 0 where a voxel lacks the slot), and the
// group's merged entries are laid out chunk by chunk (chunk c = slots
// [cR, cR + R), the rows one stage holds), quads in order inside a chunk,
// slots ascending inside a quad.  Each chunk's block is padded to a multiple
// of 8 entries so that it can be bulk-copied (16-byte sizes and addresses).
// Per chunk a table of kTabInts ints: [0..16] = exclusive offsets of the 16
// quads inside the block (tab[16] = entries), [17] = block start relative to
// the group's first entry, [18] = padded entry count.
//
// One CTA per group, one warp per quad.  A bitmap over the union slots marks
// the quad's slots; ranks come from prefix popcounts.  PASS 0 counts (padded
// entries and chunks per group), PASS 1 writes at the scanned offsets; ew
// must be zero beforehand.

constexpr int kTabInts = 20;
constexpr int kMaxChunks = kTileCap / 32 + 1;   // R >= 32

__device__ __forceinline__ int bit_rank(const uint32_t* bits, const int* pre, int x)
{
    return pre[x >> 5] + __popc(bits[x >> 5] & ((1u << (x & 31)) - 1u));
}

template <int PASS>
__global__ void __launch_bounds__(kConsumerWarps * 32)
k_tile_layout(int R, const int* __restrict__ start, const int* __restrict__ unions,
              const long long* __restrict__ woff, const unsigned short* __restrict__ slots,
              const float* __restrict__ wts, int* __restrict__ gcnt, int* __restrict__ gnch,
              const long long* __restrict__ gbase, const long long* __restrict__ tbase, int* __restrict__ table,
              unsigned short* __restrict__ erow, float4* __restrict__ ew)
{
    constexpr int kWords = kTileCap / 32;
    extern __shared__ __align__(16) uint32_t lsm[];
    uint32_t* s_bits = lsm;                                                     // [16][kWords + 1]
    int* s_pre = reinterpret_cast<int*>(lsm + kConsumerWarps * (kWords + 1));   // [16][kWords + 1]
    int* s_cw = s_pre + kConsumerWarps * (kWords + 1);                          // [kMaxChunks][17]
    int* s_cs = s_cw + kMaxChunks * 17;                                         // [kMaxChunks + 1]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = blockIdx.x;
    const int p0 = start[q], p1 = start[q + 1];
    const int u = unions[q];
    const int words = (u + 31) >> 5;
    const int nch = (u + R - 1) / R;
    uint32_t* bits = s_bits + warp * (kWords + 1);
    int* pre = s_pre + warp * (kWords + 1);
    const int lead = p0 + kQuad * warp;
    const int n = lead < p1 ? min(kQuad, p1 - lead) : 0;
    for (int w = lane; w <= words; w += 32) bits[w] = 0u;
    __syncwarp();
    long long e0 = 0, e1 = 0, b1 = 0, b2 = 0, b3 = 0;
    if (n > 0) {
        e0 = woff[lead];
        e1 = woff[lead + n];
        b1 = woff[lead + 1];
        b2 = n > 2 ? woff[lead + 2] : e1;
        b3 = n > 3 ? woff[lead + 3] : e1;
        for (long long i = e0 + lane; i < e1; i += 32) {
            const int sl = slots[i];
            atomicOr(&bits[sl >> 5], 1u << (sl & 31));
        }
    }
    __syncwarp();
    int carry = 0;
    for (int w0 = 0; w0 <= words; w0 += 32) {
        const int w = w0 + lane;
        const int c = w < words ? __popc(bits[w]) : 0;
        int inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, inc, o);
            if (lane >= o) inc += y;
        }
        if (w <= words) pre[w] = carry + inc - c;
        carry += __shfl_sync(kFull, inc, 31);
    }
    __syncwarp();
    // entries of this quad per chunk
    for (int c = lane; c < nch; c += 32) {
        const int lo = c * R, hi = min(lo + R, u);
        s_cw[c * 17 + warp] = bit_rank(bits, pre, hi) - bit_rank(bits, pre, lo);
    }
    __syncthreads();
    // per chunk: exclusive offsets over quads, padded block sizes
    for (int c = threadIdx.x; c < nch; c += blockDim.x) {
        int acc = 0;
        for (int w = 0; w < kConsumerWarps; ++w) {
            const int x = s_cw[c * 17 + w];
            s_cw[c * 17 + w] = acc;
            acc += x;
        }
        s_cw[c * 17 + 16] = acc;
        s_cs[c] = (acc + 7) & ~7;
    }
    __syncthreads();
    if (warp == 0) {   // exclusive scan of the padded block sizes
        int run = 0;
        for (int c0 = 0; c0 < nch; c0 += 32) {
            const int c = c0 + lane;
            const int x = c < nch ? s_cs[c] : 0;
            int inc = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFull, inc, o);
                if (lane >= o) inc += y;
            }
            __syncwarp();
            if (c < nch) s_cs[c] = run + inc - x;
            run += __shfl_sync(kFull, inc, 31);
        }
        if (lane == 0) s_cs[nch] = run;
    }
    __syncthreads();
    if (PASS == 0) {
        if (threadIdx.x == 0) {
            gcnt[q] = s_cs[nch];
            gnch[q] = nch;
        }
        return;
    }
    const long long gb = gbase[q];
    int* tab = table + tbase[q] * kTabInts;
    for (int i = threadIdx.x; i < nch * kTabInts; i += blockDim.x) {
        const int c = i / kTabInts, k = i % kTabInts;
        int v = 0;
        if (k <= 16) v = s_cw[c * 17 + k];
        else if (k == 17) v = s_cs[c];
        else if (k == 18) v = s_cs[c + 1] - s_cs[c];
        tab[i] = v;
    }
    if (n > 0) {
        for (long long i = e0 + lane; i < e1; i += 32) {
            const int sl = slots[i];
            const int c = sl / R;
            const long long d = gb + s_cs[c] + s_cw[c * 17 + warp] + bit_rank(bits, pre, sl) -
                                bit_rank(bits, pre, c * R);
            const int t = (i >= b1) + (i >= b2) + (i >= b3);
            erow[d] = (unsigned short)(sl - c * R);
            reinterpret_cast<float*>(ew + d)[t] = wts[i];
        }
    }
}

size_t layout_smem()
{
    return sizeof(uint32_t) * (size_t)(2 * kConsumerWarps * (kTileCap / 32 + 1) + kMaxChunks * 17 + kMaxChunks + 1);
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

// One stage of the ring: R union rows, then the chunk's entry block (4
// weights, row index) and its quad table.
template <int Q>
struct StageLayout {
    static constexpr int kRowBytes = 32 * Q * 4;
    static constexpr int kBudget = 113 * 1024;
    static constexpr int R = ((kBudget - kTabInts * 4) / (kRowBytes + kConsumerWarps * 18)) & ~7;
    static constexpr int kMaxEntries = kConsumerWarps * R;   // one entry per quad and row at most
    static constexpr int kW = R * kRowBytes;                  // float4 weights
    static constexpr int kRow = kW + kMaxEntries * 16;         // u16 row indices
    static constexpr int kTab = kRow + kMaxEntries * 2;        // table
    static constexpr int kBytes = kTab + kTabInts * 4;
    static_assert(kW % 16 == 0 && kRow % 16 == 0 && kTab % 16 == 0 && kBytes % 16 == 0, "16-byte stage parts");
};

template <int Q>
__global__ void __launch_bounds__((kConsumerWarps + kProducerWarps) * 32, 1)
k_reflect_tile(const float* __restrict__ slab, TileLists tl, const int* __restrict__ order, Accum acc,
               int* __restrict__ err)
{
    using L = StageLayout<Q>;
    constexpr int kRowFloats = 32 * Q;
    constexpr int kRowBytes = L::kRowBytes;
    constexpr int R = L::R;
    constexpr int kProducers = kProducerWarps * 32;
    constexpr int kRowsPerThread = (R + kProducers - 1) / kProducers;
    extern __shared__ __align__(128) unsigned char stage_mem[];
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

    if (warp >= kConsumerWarps) {
        // ---- producer: per chunk, the union rows, the entry block and its table
        long long k = 0;   // chunks issued by this CTA
        bool ok = true;
        for (int q = blockIdx.x; q < tl.NG && ok; q += gridDim.x) {
            const long long ubase = tl.woff[tl.start[q]];
            const long long gb = tl.gbase[q];
            const int* tab = tl.table + tl.tbase[q] * kTabInts;
            const int u = tl.unions[q];
            // this thread's rows r0 + kProducers * i of every chunk; the next
            // chunk's cells and table entries are loaded one chunk ahead
            const int r0 = (warp - kConsumerWarps) * 32 + lane;
            int ncell[kRowsPerThread];
#pragma unroll
            for (int i = 0; i < kRowsPerThread; ++i) {
                const int r = r0 + kProducers * i;
                ncell[i] = r < min(R, u) ? __ldg(tl.cells + ubase + r) : 0;
            }
            int nbstart = u > 0 ? __ldg(tab + 17) : 0;
            int nbcount = u > 0 ? __ldg(tab + 18) : 0;
            for (int c0 = 0, c = 0; c0 < u && ok; c0 += R, ++c, ++k) {
                const int s = (int)(k % kStages);
                const int rows = min(R, u - c0);
                int cell[kRowsPerThread];
#pragma unroll
                for (int i = 0; i < kRowsPerThread; ++i) cell[i] = ncell[i];
                const int bstart = nbstart, bcount = nbcount;
                if (c0 + R < u) {
#pragma unroll
                    for (int i = 0; i < kRowsPerThread; ++i) {
                        const int r = r0 + kProducers * i;
                        ncell[i] = r < min(R, u - c0 - R) ? __ldg(tl.cells + ubase + c0 + R + r) : 0;
                    }
                    nbstart = __ldg(tab + (c + 1) * kTabInts + 17);
                    nbcount = __ldg(tab + (c + 1) * kTabInts + 18);
                }
                if (k >= kStages)
                    ok = mbar_wait(smem_u32(&bar_empty[s]), (unsigned)(((k / kStages) - 1) & 1), &s_abort);
                if (!ok) break;
                const unsigned full = smem_u32(&bar_full[s]);
                const unsigned dst = smem_u32(stage_mem) + (unsigned)(s * L::kBytes);
                if (r0 == 0) {
                    mbar_expect(full, (unsigned)(rows * kRowBytes + bcount * 18 + kTabInts * 4));
                    bulk_g2s(dst + L::kTab, tab + c * kTabInts, kTabInts * 4, full);
                    if (bcount > 0) {
                        bulk_g2s(dst + L::kW, tl.ew + gb + bstart, (unsigned)(bcount * 16), full);
                        bulk_g2s(dst + L::kRow, tl.erow + gb + bstart, (unsigned)(bcount * 2), full);
                    }
                }
#pragma unroll
                for (int i = 0; i < kRowsPerThread; ++i) {
                    const int r = r0 + kProducers * i;
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
        // let the copies of this warp (and the CTA) land before it exits
        if (lane == 0) {
            for (long long j = (k > kStages ? k - kStages : 0); j < k; ++j)
                mbar_wait(smem_u32(&bar_full[j % kStages]), (unsigned)((j / kStages) & 1), nullptr);
        }
        return;
    }

    // ---- consumers: warp w owns the quad of positions p0 + 4w .. p0 + 4w + 3
    long long k = 0;
    for (int q = blockIdx.x; q < tl.NG; q += gridDim.x) {
        const int p0 = tl.start[q], p1 = tl.start[q + 1];
        const int u = tl.unions[q];
        const int lead = p0 + kQuad * warp;
        float a[kQuad][Q];
#pragma unroll
        for (int t = 0; t < kQuad; ++t)
#pragma unroll
            for (int h = 0; h < Q; ++h) a[t][h] = 0.0f;
        for (int c0 = 0; c0 < u; c0 += R, ++k) {
            const int s = (int)(k % kStages);
            if (!mbar_wait(smem_u32(&bar_full[s]), (unsigned)((k / kStages) & 1), &s_abort)) {
                if (lane == 0) atomicOr(err, kErrWaitTimeout);
                s_abort = 1;
                return;
            }
            const unsigned char* st = stage_mem + (size_t)s * L::kBytes;
            const float* rows = reinterpret_cast<const float*>(st);
            const float4* wv = reinterpret_cast<const float4*>(st + L::kW);
            const unsigned short* rv = reinterpret_cast<const unsigned short*>(st + L::kRow);
            const int* tab = reinterpret_cast<const int*>(st + L::kTab);
            const int b = tab[warp], e = tab[warp + 1];
            // A zero weight (a voxel of the quad without this neighbor) adds
            // an exact +0 to nonnegative sums, so its FMAs are skipped; the
            // weights are the same in all lanes, so the branches are uniform.
#pragma unroll 2
            for (int i = b; i < e; ++i) {
                const int r = rv[i];
                const float4 w = wv[i];
                float x[Q];
                smem_row<Q>(x, rows + r * kRowFloats, lane);
                if (w.x != 0.0f) {
#pragma unroll
                    for (int h = 0; h < Q; ++h) a[0][h] = fmaf(w.x, x[h], a[0][h]);
                }
                if (w.y != 0.0f) {
#pragma unroll
                    for (int h = 0; h < Q; ++h) a[1][h] = fmaf(w.y, x[h], a[1][h]);
                }
                if (w.z != 0.0f) {
#pragma unroll
                    for (int h = 0; h < Q; ++h) a[2][h] = fmaf(w.z, x[h], a[2][h]);
                }
                if (w.w != 0.0f) {
#pragma unroll
                    for (int h = 0; h < Q; ++h) a[3][h] = fmaf(w.w, x[h], a[3][h]);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&bar_empty[s]));
        }
#pragma unroll
        for (int t = 0; t < kQuad; ++t) {
            const int p = lead + t;
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

// Sets the dynamic shared-memory limit of a kernel once per device.
template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes, std::atomic<bool> (&done)[kMaxDevices])
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!done[dev].load(std::memory_order_acquire)) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        done[dev].store(true, std::memory_order_release);
    }
    return cudaSuccess;
}

template <int Q>
cudaError_t tile_q(const float* slab, const TileLists& tl, const int* order, const Accum& acc, int* err,
                   cudaStream_t st)
{
    if (tl.R != StageLayout<Q>::R) return cudaErrorInvalidValue;
    const size_t smem = (size_t)kStages * StageLayout<Q>::kBytes;
    static std::atomic<bool> attr[kMaxDevices];
    cudaError_t e = allow_smem(k_reflect_tile<Q>, smem, attr);
    if (e != cudaSuccess) return e;
    const int grid = tl.NG < tile_sms() ? tl.NG : tile_sms();
    k_reflect_tile<Q><<<grid, (kConsumerWarps + kProducerWarps) * 32, smem, st>>>(slab, tl, order, acc, err);
    return cudaGetLastError();
}

}  // namespace

int tile_rows_per_stage(int B)
{
    switch (B) {
    case 64: return StageLayout<2>::R;
    case 128: return StageLayout<4>::R;
    case 256: return StageLayout<8>::R;
    default: return 0;
    }
}

cudaError_t launch_tile_groups(int N, int G, const long long* woff, int* flag, long long* pos,
                               long long* scan_tmp, int* start, cudaStream_t st)
{
    if (N <= 0) return cudaSuccess;
    if (G != kQuad * kConsumerWarps) return cudaErrorInvalidValue;
    const unsigned grid = (unsigned)((N + 255) / 256);
    k_tile_flags<<<grid, 256, 0, st>>>(N, G, woff, flag);
    cudaError_t e = launch_scan_counts(flag, N, 0, pos, scan_tmp, nullptr, st);
    if (e != cudaSuccess) return e;
    k_tile_starts<<<grid, 256, 0, st>>>(N, flag, pos, start);
    return cudaGetLastError();
}

cudaError_t launch_tile_build(int NG, const int* start, const long long* woff, int* cells, unsigned short* slots,
                              int* unions, long long* rows_total, int* err, cudaStream_t st)
{
    if (NG <= 0) return cudaSuccess;
    const size_t smem = (size_t)3 * kTileCap * 4;
    static std::atomic<bool> attr[kMaxDevices];
    cudaError_t e = allow_smem(k_tile_build, smem, attr);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(rows_total, 0, sizeof(long long), st);
    if (e != cudaSuccess) return e;
    k_tile_build<<<NG, kBuildThreads, smem, st>>>(start, woff, cells, slots, unions,
                                                  reinterpret_cast<unsigned long long*>(rows_total), err);
    return cudaGetLastError();
}

cudaError_t launch_tile_layout(int pass, int NG, int R, const int* start, const int* unions, const long long* woff,
                               const unsigned short* slots, const float* wts, int* gcnt, int* gnch,
                               const long long* gbase, const long long* tbase, int* table,
                               unsigned short* erow, float4* ew, cudaStream_t st)
{
    if (NG <= 0) return cudaSuccess;
    if (R < 32) return cudaErrorInvalidValue;
    const size_t smem = layout_smem();
    static std::atomic<bool> attr0[kMaxDevices], attr1[kMaxDevices];
    cudaError_t e = pass == 0 ? allow_smem(k_tile_layout<0>, smem, attr0) : allow_smem(k_tile_layout<1>, smem, attr1);
    if (e != cudaSuccess) return e;
    if (pass == 0)
        k_tile_layout<0><<<NG, kConsumerWarps * 32, smem, st>>>(R, start, unions, woff, slots, wts, gcnt, gnch,
                                                                gbase, tbase, table, erow, ew);
    else
        k_tile_layout<1><<<NG, kConsumerWarps * 32, smem, st>>>(R, start, unions, woff, slots, wts, gcnt, gnch,
                                                                gbase, tbase, table, erow, ew);
    return cudaGetLastError();
}

cudaError_t launch_reflect_tile(int B, const float* slab, const TileLists& tl, const int* order, const Accum& acc,
                                int* err, cudaStream_t st)
{
    if (tl.NG <= 0) return cudaSuccess;
    if (tl.G != kQuad * kConsumerWarps) return cudaErrorInvalidValue;
    switch (B) {
    case 64: return tile_q<2>(slab, tl, order, acc, err, st);
    case 128: return tile_q<4>(slab, tl, order, acc, err, st);
    case 256: return tile_q<8>(slab, tl, order, acc, err, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace sgb
