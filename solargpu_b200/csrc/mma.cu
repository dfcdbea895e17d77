// Hour-block reflection on the tensor cores (tcgen05).
//
// R[v, h] = sum_g w(v, g) I[g, h] is, for a group of 128 voxels that are
// close in the visiting order, a dense product over the union U of their
// neighbor cells:  D[128 voxels][256 hours] = W[128][U] x I[U][256].  W is
// sparse (a voxel sees ~7-10% of its group's union), but the tensor cores run
// the dense product faster than CUDA cores run the sparse one, and every
// slab row staged for the group feeds 128 voxels at once.
//
// Once per run (hour-independent):
//   union    each aligned group of 128 visiting positions: its distinct cells
//            (shared-memory hash set), sorted descending, written over the
//            start of the group's weighted-list cells; every weighted entry
//            gets its slot (index in the union);
//   layout   the union is cut into chunks of 64 rows (the MMA K per stage);
//            per chunk, its entries are stored as (byte offset in the
//            shared-memory W tile, fp16 hi, fp16 lo): the weights of voxel t
//            are scaled by 2^-e_t (e_t: the exponent of its largest weight)
//            and split as w = hi + lo, so the two fp16 MMAs carry ~22 bits of
//            each weight; 2^e_t is kept per position for the epilogue.
//
// Per hour block (B = 256 hours), a persistent CTA walks its groups:
//   producers (4 warps)  copy each chunk's 64 union rows of the fp16 slab
//                        (I[g][256 hours], 512 B a row) with 16-byte cp.async
//                        straight into the MN-major 128-byte-swizzled layout
//                        the MMA reads (B operand, N = hours) -- 4 slab
//                        stages, the copies of 3 chunks in flight -- then
//                        fence the async proxy and arrive on the stage's
//                        full barrier;
//   builders (3 warps)   zero one of 3 W stages (K-major, 128-byte swizzle,
//                        A operand, M = voxels) and scatter the chunk's
//                        entries, fence, arrive;
//   MMA (1 thread)       tcgen05.mma kind::f16 M128 N256 K16, 4 per chunk
//                        and tile (hi, lo), into one of two TMEM accumulators
//                        (2 x 256 columns), tcgen05.commit frees the stage;
//   epilogue (4 warps)   thread t = TMEM lane t = voxel t of the group: reads
//                        its 256 hours with tcgen05.ld, adds its own direct +
//                        diffuse (FP32, solar_I from the hour table), sums the
//                        hours and accumulates (FP64, Kahan or plain), while
//                        the MMAs of the next group fill the other accumulator.
//
// fp16 I values (RN, unbiased) and split fp16 weights keep the annual error
// far below 1e-4 (the rounding errors of I are independent across hours).
// Every mbarrier wait is bounded (1 s); on expiry the kernel flags
// kErrWaitTimeout, stops issuing, lets its copies and MMAs finish (bounded)
// and frees TMEM before it exits.
#include "solar_math.cuh"

#include <atomic>
#include <cstdlib>
#include <functional>
#include <queue>
#include <utility>
#include <vector>

#include <cuda_fp16.h>

namespace sgb {
namespace {

constexpr int kGroup = 128;                 // voxels per group = MMA M = TMEM lanes
constexpr int kHours = 256;                 // hours per block = MMA N
constexpr int kChunk = 64;                  // union rows per stage = MMA K per stage
constexpr int kBStages = 4;                 // slab-row stages (gathered: latency to hide)
constexpr int kAStages = 3;                 // weight-tile stages (built from registers)
constexpr int kCopyLag = kBStages - 2;      // a producer publishes chunk k - kCopyLag after issuing chunk k
constexpr int kUnionCap = 16384;            // distinct cells of a group the build handles
constexpr int kHashSlots = 2 * kUnionCap;
constexpr int kSmallCap = 8192;             // first pass: unions up to this many cells
constexpr int kBuildThreads = 1024;
constexpr int kLayoutThreads = 512;
constexpr int kMaxChunks = kUnionCap / kChunk;
constexpr unsigned long long kWaitNs = 1000000000ull;   // 1 s
constexpr int kMaxDevices = 64;

// warp roles of the hour-block kernel
constexpr int kProducerWarps = 4;           // warps 0-3
constexpr int kEpilogueWarp0 = 4;           // warps 4-7 (TMEM lane quarters 0-3)
constexpr int kMmaWarp = 8;
constexpr int kBuilderWarp0 = 9;            // warps 9-11
constexpr int kBuilderWarps = 3;
constexpr int kThreads = 12 * 32;

// shared memory: 3 x (W hi tile | W lo tile), 4 x slab rows (the hour table
// is read through L1: every epilogue lane reads the same entry)
constexpr int kTileA = kGroup * kChunk * 2;        // 16 KB, fp16 [128][64], K-major, 128B swizzle
constexpr int kTileB = kChunk * kHours * 2;        // 32 KB, fp16 [64 rows][256 hours], MN-major, 128B swizzle
constexpr int kAStageBytes = 2 * kTileA;           // 32 KB: hi and lo tiles
constexpr int kBRegion = kAStages * kAStageBytes;  // slab stages start here
constexpr int kSmemBytes = kBRegion + kBStages * kTileB + 1024;   // 225 KB + 1024-byte alignment slack
static_assert(kSmemBytes <= 227 * 1024 - 512, "dynamic + static shared memory of one CTA");

// Instruction descriptor, kind::f16: f32 accumulator, fp16 A and B, A
// K-major, B MN-major, N = 256, M = 128.
constexpr unsigned kIdesc = (1u << 4) | (1u << 16) | ((unsigned)(kHours >> 3) << 17) | ((unsigned)(kGroup >> 4) << 24);

// ---- union of each group ------------------------------------------------------

__device__ __forceinline__ void block_sort_desc(uint32_t* keys, int n2)
{
    for (int size = 2; size <= n2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < (n2 >> 1); t += blockDim.x) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const bool desc = (i & size) == 0;
                const uint32_t a = keys[i], b = keys[j];
                if ((a < b) == desc) {
                    keys[i] = b;
                    keys[j] = a;
                }
            }
            __syncthreads();
        }
    }
}

// The union of group q, in one CTA: cells[e] (0-based cell of weighted entry
// e) are replaced, from woff[p0] on, by the group's union (descending);
// slots[e] = index of the entry's cell in it.  Returns false, writing
// nothing, when the union has more than CAP cells.
template <int CAP>
__device__ bool union_group(int q, int N, const long long* __restrict__ woff, int* __restrict__ cells,
                            unsigned short* __restrict__ slots, int* __restrict__ unions, int* __restrict__ nch,
                            uint32_t* sm, int* s_count)
{
    constexpr int kSlots = 2 * CAP;
    constexpr int kBits = CAP == 16384 ? 15 : CAP == 8192 ? 14 : 0;
    static_assert(kBits > 0, "union cap of 8192 or 16384 cells");
    uint32_t* table = sm;                 // [kSlots], key = cell + 1, 0 = empty
    uint32_t* uni = sm + kSlots;          // [CAP]
    const int p0 = q * kGroup, p1 = min(N, p0 + kGroup);
    const long long e0 = woff[p0], e1 = woff[p1];
    for (int i = threadIdx.x; i < kSlots; i += blockDim.x) table[i] = 0u;
    if (threadIdx.x == 0) *s_count = 0;
    __syncthreads();
    for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const uint32_t key = (uint32_t)cells[e] + 1u;
        uint32_t h = (key * 2654435761u) >> (32 - kBits);
        for (int probe = 0; probe < kSlots; ++probe) {
            const uint32_t prev = atomicCAS(&table[h], 0u, key);
            if (prev == 0u) {
                const int at = atomicAdd(s_count, 1);
                if (at < CAP) uni[at] = key;
                break;
            }
            if (prev == key) break;
            h = (h + 1u) & (kSlots - 1);
        }
    }
    __syncthreads();
    const int u = *s_count;
    if (u > CAP) return false;   // uniform: every thread read the same count
    int u2 = 64;
    while (u2 < u) u2 <<= 1;
    for (int i = u + threadIdx.x; i < u2; i += blockDim.x) uni[i] = 0u;
    __syncthreads();
    block_sort_desc(uni, u2);
    int* ucell = reinterpret_cast<int*>(uni);
    for (int i = threadIdx.x; i < u; i += blockDim.x) ucell[i] = (int)uni[i] - 1;
    __syncthreads();
    for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int cell = cells[e];
        int lo = 0, hi = u - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (ucell[mid] > cell) lo = mid + 1; else hi = mid;
        }
        slots[e] = (unsigned short)lo;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < u; i += blockDim.x) cells[e0 + i] = ucell[i];
    if (threadIdx.x == 0) {
        unions[q] = u;
        nch[q] = (u + kChunk - 1) / kChunk;
    }
    return true;
}

// First pass, one CTA per group with room for kSmallCap cells (96 KB of
// shared memory: two CTAs a SM); a group with a larger union is listed in
// retry[1 ..] (count in retry[0]) and left untouched.
__global__ void __launch_bounds__(kBuildThreads)
k_mma_union_small(int N, const long long* __restrict__ woff, int* __restrict__ cells,
                  unsigned short* __restrict__ slots, int* __restrict__ unions, int* __restrict__ nch,
                  int* __restrict__ retry, int hand_on_all)
{
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ int s_count;
    const int q = blockIdx.x;
    if ((hand_on_all || !union_group<kSmallCap>(q, N, woff, cells, slots, unions, nch, sm, &s_count)) &&
        threadIdx.x == 0)
        retry[1 + atomicAdd(retry, 1)] = q;
}

// Second pass over the listed groups with room for kUnionCap cells; a union
// above that leaves the group untouched and counts it in *over.
__global__ void __launch_bounds__(kBuildThreads)
k_mma_union_large(int N, const long long* __restrict__ woff, int* __restrict__ cells,
                  unsigned short* __restrict__ slots, int* __restrict__ unions, int* __restrict__ nch,
                  const int* __restrict__ retry, int* __restrict__ over)
{
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ int s_count;
    const int n = retry[0];
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int q = retry[1 + i];
        if (!union_group<kUnionCap>(q, N, woff, cells, slots, unions, nch, sm, &s_count) && threadIdx.x == 0) {
            atomicAdd(over, 1);
            unions[q] = 0;
            nch[q] = 0;
        }
        __syncthreads();
    }
}

// Byte offset of W element (voxel t, row k of the chunk) in the K-major,
// 128-byte-swizzled tile: 8-voxel atoms of 1024 bytes, 128 bytes (64 fp16)
// a voxel, 16-byte pieces XOR-ed with the voxel's row in the atom.
__device__ __forceinline__ unsigned a_offset(int t, int k)
{
    const int r = t & 7;
    return (unsigned)((t >> 3) * 1024 + r * 128 + (((k >> 3) ^ r) << 4) + ((k & 7) << 1));
}

// One CTA per group.  PASS 0: entries per chunk (ccnt at cbase[q]) and the
// per-position scale 2^e; PASS 1: the entries at coff (ent must not be
// read before).  Groups that overflowed the union cap have no chunks.
template <int PASS>
__global__ void __launch_bounds__(kLayoutThreads)
k_mma_layout(int N, const long long* __restrict__ woff, const unsigned short* __restrict__ slots,
             const float* __restrict__ wts, const int* __restrict__ nch, const long long* __restrict__ cbase,
             int* __restrict__ ccnt, const long long* __restrict__ coff, uint2* __restrict__ ent,
             float* __restrict__ scale)
{
    __shared__ int s_cnt[kMaxChunks];
    __shared__ int s_exp[kGroup];
    const int q = blockIdx.x;
    const int p0 = q * kGroup, p1 = min(N, p0 + kGroup);
    const int nc = nch[q];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = threadIdx.x; c < nc; c += blockDim.x) s_cnt[c] = 0;
    // exponent of each voxel's largest weight (weights are > 0)
    for (int t = warp; t < kGroup; t += kLayoutThreads / 32) {
        const int p = p0 + t;
        float m = 0.0f;
        if (p < p1)
            for (long long e = woff[p] + lane; e < woff[p + 1]; e += 32) m = fmaxf(m, wts[e]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
        int ex = 0;
        if (m > 0.0f) frexpf(m, &ex);   // m in [2^(ex-1), 2^ex)
        if (lane == 0) {
            s_exp[t] = ex;
            if (PASS == 0 && p < p1) scale[p] = ldexpf(1.0f, ex);
        }
    }
    __syncthreads();
    if (nc == 0) return;
    const long long cb = cbase[q];
    // voxel t owns entries [woff[p0 + t], woff[p0 + t + 1])
    for (int t = warp; t < p1 - p0; t += kLayoutThreads / 32) {
        const int p = p0 + t;
        const float sc = ldexpf(1.0f, -s_exp[t]);
        for (long long e = woff[p] + lane; e < woff[p + 1]; e += 32) {
            const int sl = slots[e];
            const int c = sl / kChunk;
            const int at = atomicAdd(&s_cnt[c], 1);
            if (PASS == 1) {
                const float w = wts[e] * sc;   // exact: a power-of-two scale
                const __half hi = __float2half_rn(w);
                const __half lo = __float2half_rn(w - __half2float(hi));
                const __half2 hl = __halves2half2(hi, lo);
                ent[coff[cb + c] + at] = make_uint2(a_offset(t, sl - c * kChunk), *reinterpret_cast<const unsigned*>(&hl));
            }
        }
    }
    if (PASS == 0) {
        __syncthreads();
        for (int c = threadIdx.x; c < nc; c += blockDim.x) ccnt[cb + c] = s_cnt[c];
    }
}

// I[g][b] (fp16) for the top cells and the block's hours.
constexpr int kSlabCellsPerWarp = 64;

__global__ void __launch_bounds__(256)
k_solar_slab16(const float4* __restrict__ geo_n, int T, const uint32_t* __restrict__ shadow, int words32,
               const HourEntry* __restrict__ table, int j0, __half* __restrict__ slab)
{
    const int lane = threadIdx.x & 31;
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int hchunks = kHours >> 5;
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
        slab[g * kHours + b] = __float2half_rn(solar_I(n4, e, bit));
    }
}

// ---- hour-block kernel ----------------------------------------------------------

__device__ __forceinline__ unsigned su32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long gtime()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase of the given parity; false on expiry or when another
// role gave up.
__device__ __forceinline__ bool bar_wait(unsigned bar, unsigned parity, const volatile int* fail,
                                         unsigned long long limit = kWaitNs)
{
    unsigned long long t0 = 0;
    for (unsigned i = 0;; ++i) {
        unsigned ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 63u) == 63u) {
            if (fail && *fail) return false;
            const unsigned long long t = gtime();
            if (t0 == 0) t0 = t;
            else if (t - t0 > limit) return false;
        }
    }
}

__device__ __forceinline__ void bar_arrive(unsigned bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// K-major, 128-byte swizzle (layout 2, sm_100 version 1): 8-row atoms 1024
// bytes apart (SBO), leading offset unused.
__device__ __forceinline__ unsigned long long desc_k_sw128(unsigned addr)
{
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | (1ull << 16) | ((unsigned long long)(1024 >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}

// MN-major, 128-byte swizzle: atoms of 8 K-rows x 64 fp16 (1024 bytes); the
// next 64 hours (MN) are 8 KB further (LBO), the next 8 rows (K) 1 KB (SBO).
__device__ __forceinline__ unsigned long long desc_mn_sw128(unsigned addr)
{
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)(8192 >> 4) << 16) |
           ((unsigned long long)(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void mma_f16(unsigned d, unsigned long long a, unsigned long long b, unsigned acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(kIdesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(unsigned bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void accumulate(const Accum& a, int v, float x)
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

struct MmaTiles {
    int N, NG;
    const int* order;          // [N] voxel at each visiting position
    const long long* woff;     // [N + 1]; the union of group q starts at woff[128 q]
    const int* cells;          // union cells (descending) per group
    const int* unions;         // [NG] union size
    const long long* cbase;    // [NG + 1] first chunk of each group
    const long long* coff;     // [C + 1] first entry of each chunk
    const uint2* ent;          // entries: x = byte offset in the W tile, y = half2 (hi, lo)
    const float* scale;        // [N] 2^e per visiting position
    const int* sched;          // [gridDim.x + 1] offsets, then the groups of each CTA
};

// Walks the (group, chunk) sequence of one CTA: the CTA's groups in its
// schedule, chunks of 64 union rows inside each group (groups with an empty
// union have none) -- the order every role follows.
struct Cursor {
    int i, iend, q, c, u;
    long long ub;   // first union cell of group q
    long long cb;   // first chunk of group q
    __device__ Cursor(const MmaTiles& mt, int cta)
        : i(__ldg(mt.sched + cta)), iend(__ldg(mt.sched + cta + 1)), q(0), c(0), u(0), ub(0), cb(0)
    {
        settle(mt);
    }
    __device__ bool valid() const { return i < iend; }
    __device__ void settle(const MmaTiles& mt)
    {
        const int* list = mt.sched + gridDim.x + 1;
        for (; i < iend; ++i, c = 0) {
            q = __ldg(list + i);
            u = __ldg(mt.unions + q);
            if (c * kChunk < u) break;
        }
        if (i < iend) {
            ub = __ldg(mt.woff + (long long)q * kGroup);
            cb = __ldg(mt.cbase + q);
        }
    }
    __device__ void advance(const MmaTiles& mt)
    {
        ++c;
        if (c * kChunk >= u) {
            ++i;
            c = 0;
            settle(mt);
        }
    }
    // cell of row r of the current chunk (padding rows repeat row 0: their weights are 0)
    __device__ int row_cell(const MmaTiles& mt, int r, bool want) const
    {
        if (!want) return 0;
        const int rows = min(kChunk, u - c * kChunk);
        return __ldg(mt.cells + ub + (long long)c * kChunk + (r < rows ? r : 0));
    }
};

__global__ void __launch_bounds__(kThreads, 1)
k_reflect_mma(const __half* __restrict__ slab, MmaTiles mt, const float4* __restrict__ geo_n,
              const uint32_t* __restrict__ shadow, int words32, const HourEntry* __restrict__ table, int j0,
              Accum acc, int* __restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char dsm[];
    __shared__ __align__(8) unsigned long long full[kBStages], emptyB[kBStages], aready[kAStages], emptyA[kAStages],
        dfull[2], dempty[2], drain;
    __shared__ unsigned s_tmem;
    __shared__ volatile int s_fail;
    __shared__ volatile int s_bok;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned base = (su32(dsm) + 1023u) & ~1023u;               // stages, 1024-byte aligned
    unsigned char* gbase = dsm + (base - su32(dsm));
    const HourEntry* tab = table + j0;

    if (warp == kMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&s_tmem)), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kBStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(&full[s])), "r"(kProducerWarps));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(&emptyB[s])), "r"(1));
        }
        for (int s = 0; s < kAStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(&aready[s])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(&emptyA[s])), "r"(1));
        }
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(&dfull[b])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(&dempty[b])), "r"(4));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(&drain)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = s_tmem;
    bool ok = true;

    if (warp < kProducerWarps) {
        // ---- producers: 16 rows a warp, one 16-byte piece a lane per row; the
        // cell ids of the next chunk load while its stage is still in use
        long long k = 0;
        const int r0 = warp * 16;
        Cursor cur(mt, blockIdx.x);
        int my = cur.valid() ? cur.row_cell(mt, r0 + lane, lane < 16) : 0;
        while (cur.valid() && ok) {
            const int s = (int)(k % kBStages);
            const bool w_ok = k < kBStages || bar_wait(su32(&emptyB[s]), (unsigned)(((k / kBStages) - 1) & 1), &s_fail);
            if (!__all_sync(0xFFFFFFFFu, w_ok)) {   // the warp decides as one
                ok = false;
                break;
            }
            const int cur_cell = my;
            const unsigned bst = base + (unsigned)(kBRegion + s * kTileB);
            const int na = lane >> 3, cc = lane & 7;
#pragma unroll 4
            for (int i = 0; i < 16; ++i) {
                const int kr = r0 + i;
                const int cell = __shfl_sync(0xFFFFFFFFu, cur_cell, i);
                const __half* src = slab + (size_t)cell * kHours + lane * 8;
                const int r8 = kr & 7;
                const unsigned dst = bst + (unsigned)(na * 8192 + (kr >> 3) * 1024 + r8 * 128 + ((cc ^ r8) << 4));
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
            if (k >= kCopyLag) {
                // chunk k - 2's copies have landed (the last 2 groups may be
                // pending): publish them to the tensor cores
                static_assert(kCopyLag == 2, "wait_group count below");
                asm volatile("cp.async.wait_group 2;" ::: "memory");
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) bar_arrive(su32(&full[(k - kCopyLag) % kBStages]));
            }
            // the next chunk's cell ids (a new group first reads its union
            // size and base: those loads stay off the copy and arrive path)
            cur.advance(mt);
            my = cur.valid() ? cur.row_cell(mt, r0 + lane, lane < 16) : 0;
            ++k;
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0)
            for (long long j = k >= kCopyLag ? k - kCopyLag : 0; j < k; ++j) bar_arrive(su32(&full[j % kBStages]));
        if (!ok) {
            if (lane == 0) atomicOr(err, kErrWaitTimeout);
            s_fail = 1;
        }
    } else if (warp == kMmaWarp) {
        // ---- one thread issues the MMAs
        if (lane == 0) {
            long long k = 0;
            int gi = 0;
            const int* list = mt.sched + gridDim.x + 1;
            const int i1 = __ldg(mt.sched + blockIdx.x + 1);
            for (int i = __ldg(mt.sched + blockIdx.x); i < i1 && ok; ++i, ++gi) {
                const int q = __ldg(list + i);
                const int b = gi & 1;
                if (gi >= 2 && !bar_wait(su32(&dempty[b]), (unsigned)(((gi >> 1) - 1) & 1), &s_fail)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const int u = mt.unions[q];
                const unsigned d = tmem + (unsigned)(b * kHours);
                for (int c = 0; c * kChunk < u; ++c, ++k) {
                    const int s = (int)(k % kBStages), t = (int)(k % kAStages);
                    if (!bar_wait(su32(&full[s]), (unsigned)((k / kBStages) & 1), &s_fail) ||
                        !bar_wait(su32(&aready[t]), (unsigned)((k / kAStages) & 1), &s_fail)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const unsigned sa = base + (unsigned)(t * kAStageBytes);
                    const unsigned sb = base + (unsigned)(kBRegion + s * kTileB);
                    const int ks = (min(kChunk, u - c * kChunk) + 15) >> 4;
                    for (int j = 0; j < ks; ++j) {
                        const unsigned long long db = desc_mn_sw128(sb + 2048u * j);
                        mma_f16(d, desc_k_sw128(sa + 32u * j), db, (c > 0 || j > 0) ? 1u : 0u);
                        mma_f16(d, desc_k_sw128(sa + kTileA + 32u * j), db, 1u);
                    }
                    // both stages are free once these MMAs have read them
                    mma_commit(su32(&emptyB[s]));
                    mma_commit(su32(&emptyA[t]));
                }
                if (!ok) break;
                mma_commit(su32(&dfull[b]));       // the group's accumulator is complete
            }
            if (!ok) {
                atomicOr(err, kErrWaitTimeout);
                s_fail = 1;
            }
        }
        __syncwarp();
    } else if (warp >= kBuilderWarp0) {
        // ---- builders: zero the W tiles, scatter the chunk's weights; the
        // entries of the next chunk are loaded into registers while the
        // builders wait for its stage
        const int bt = threadIdx.x - kBuilderWarp0 * 32;
        constexpr int kBuilders = kBuilderWarps * 32;
        constexpr int kPref = 16;   // entries a thread holds ahead (8: +11%, 12: +1.6%, 20: +2%); more load at scatter
        Cursor cur(mt, blockIdx.x);
        uint2 pre[kPref];
        long long pe0 = 0, pe1 = 0;
        auto prefetch = [&]() {
            pe0 = pe1 = 0;
            if (cur.valid()) {
                const long long ci = cur.cb + cur.c;
                pe0 = __ldg(mt.coff + ci);
                pe1 = __ldg(mt.coff + ci + 1);
            }
#pragma unroll
            for (int i = 0; i < kPref; ++i) {
                const long long e = pe0 + bt + (long long)i * kBuilders;
                pre[i] = e < pe1 ? __ldg(mt.ent + e) : make_uint2(0xFFFFFFFFu, 0u);
            }
        };
        prefetch();
        long long k = 0;
        while (cur.valid() && ok) {
            const int s = (int)(k % kAStages);
            // one thread waits for the stage; every builder takes its decision
            if (bt == 0)
                s_bok = (k < kAStages || bar_wait(su32(&emptyA[s]), (unsigned)(((k / kAStages) - 1) & 1), &s_fail))
                            ? 1 : 0;
            asm volatile("bar.sync 1, %0;" ::"r"(kBuilders) : "memory");
            ok = s_bok != 0;
            if (!ok) break;
            unsigned char* sa = gbase + (size_t)s * kAStageBytes;
            uint4* z = reinterpret_cast<uint4*>(sa);
            for (int i = bt; i < 2 * kTileA / 16; i += kBuilders) z[i] = make_uint4(0u, 0u, 0u, 0u);
            asm volatile("bar.sync 1, %0;" ::"r"(kBuilders) : "memory");
#pragma unroll
            for (int i = 0; i < kPref; ++i) {
                if (pre[i].x != 0xFFFFFFFFu) {
                    *reinterpret_cast<unsigned short*>(sa + pre[i].x) = (unsigned short)(pre[i].y & 0xFFFFu);
                    *reinterpret_cast<unsigned short*>(sa + kTileA + pre[i].x) = (unsigned short)(pre[i].y >> 16);
                }
            }
            for (long long e = pe0 + bt + (long long)kPref * kBuilders; e < pe1; e += kBuilders) {
                const uint2 en = __ldg(mt.ent + e);
                *reinterpret_cast<unsigned short*>(sa + en.x) = (unsigned short)(en.y & 0xFFFFu);
                *reinterpret_cast<unsigned short*>(sa + kTileA + en.x) = (unsigned short)(en.y >> 16);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("bar.sync 1, %0;" ::"r"(kBuilders) : "memory");
            if (bt == 0) bar_arrive(su32(&aready[s]));
            // the next chunk's entries load while the builders wait for its stage
            // (after the arrive: their latency stays off the MMA's path)
            cur.advance(mt);
            prefetch();
            ++k;
        }
        if (!ok) {
            if (bt == 0) atomicOr(err, kErrWaitTimeout);
            s_fail = 1;
        }
    } else {
        // ---- epilogue: thread t = TMEM lane t = voxel t of the group
        const int t = threadIdx.x - kEpilogueWarp0 * 32;
        const unsigned lane_base = (unsigned)((warp & 3) * 32) << 16;
        int gi = 0;
        const int* list = mt.sched + gridDim.x + 1;
        const int i1 = __ldg(mt.sched + blockIdx.x + 1);
        for (int i = __ldg(mt.sched + blockIdx.x); i < i1 && ok; ++i, ++gi) {
            const int q = __ldg(list + i);
            const int b = gi & 1;
            const bool w_ok = bar_wait(su32(&dfull[b]), (unsigned)((gi >> 1) & 1), &s_fail, 2 * kWaitNs);
            if (!__all_sync(0xFFFFFFFFu, w_ok)) {   // tcgen05.ld below needs the whole warp
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int p = q * kGroup + t;
            const bool valid = p < mt.N;
            const int v = valid ? __ldg(mt.order + p) : 0;
            const float4 n4 = __ldg(geo_n + v);
            const float sc = valid ? __ldg(mt.scale + p) : 0.0f;
            const bool any = mt.unions[q] > 0;
            float sum = 0.0f;
            for (int c0 = 0; c0 < kHours; c0 += 32) {
                unsigned r[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                    "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                      "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                      "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                    : "r"(tmem + lane_base + (unsigned)(b * kHours + c0)));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const HourEntry e = tab[c0 + i];
                    const float own = solar_I(n4, e, shadow_bit(shadow, words32, v, e.dense));
                    const float refl = any ? __uint_as_float(r[i]) * sc : 0.0f;
                    sum += own + refl;
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) bar_arrive(su32(&dempty[b]));
            if (valid) accumulate(acc, v, sum);
        }
        if (!ok) {
            if (lane == 0) atomicOr(err, kErrWaitTimeout);
            s_fail = 1;
        }
    }

    // Drain: every MMA this CTA issued completes before TMEM is freed
    // (tcgen05.commit tracks all of the issuing thread's earlier MMAs).
    __syncthreads();
    if (warp == kMmaWarp) {
        if (lane == 0) {
            mma_commit(su32(&drain));
            if (!bar_wait(su32(&drain), 0u, nullptr, 2 * kWaitNs)) atomicOr(err, kErrWaitTimeout);
        }
        __syncwarp();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

int mma_sms()
{
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

}  // namespace

int mma_group_count(int N) { return (N + kGroup - 1) / kGroup; }

int mma_grid(int N)
{
    const int NG = mma_group_count(N);
    return NG < mma_sms() ? NG : mma_sms();
}

void mma_schedule(int N, const long long* cbase, int* sched)
{
    const int NG = mma_group_count(N);
    const int P = mma_grid(N);
    if (NG <= 0 || P <= 0) return;
    // a group costs its chunks plus about one chunk of switching (the epilogue
    // of its accumulator, the first copies of the next group)
    constexpr long long kGroupCost = 1;
    std::vector<int> owner(NG), count(P, 0);
    std::priority_queue<std::pair<long long, int>, std::vector<std::pair<long long, int>>,
                        std::greater<std::pair<long long, int>>> load;
    for (int b = 0; b < P; ++b) load.push({0, b});
    for (int q = 0; q < NG; ++q) {
        const auto top = load.top();
        load.pop();
        owner[q] = top.second;
        ++count[top.second];
        load.push({top.first + (cbase[q + 1] - cbase[q]) + kGroupCost, top.second});
    }
    sched[0] = 0;
    for (int b = 0; b < P; ++b) sched[b + 1] = sched[b] + count[b];
    std::vector<int> at(sched, sched + P);
    int* list = sched + P + 1;
    for (int q = 0; q < NG; ++q) list[at[owner[q]]++] = q;   // increasing within each CTA
}

cudaError_t launch_mma_union(int N, const long long* woff, int* cells, unsigned short* slots, int* unions, int* nch,
                             int* over, int* retry, cudaStream_t st)
{
    const int NG = mma_group_count(N);
    if (NG <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(retry, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    const size_t small = sizeof(uint32_t) * (size_t)(3 * kSmallCap);
    const size_t large = sizeof(uint32_t) * (size_t)(kHashSlots + kUnionCap);
    static std::atomic<bool> attr_s[kMaxDevices], attr_l[kMaxDevices];
    if ((e = allow_smem(k_mma_union_small, small, attr_s)) != cudaSuccess) return e;
    if ((e = allow_smem(k_mma_union_large, large, attr_l)) != cudaSuccess) return e;
    // SGB_UNION_SECOND_PASS=1 hands every group to the second pass (tests use
    // it to check that pass; the unions are the same either way)
    const char* env = std::getenv("SGB_UNION_SECOND_PASS");
    const int all = (env && env[0] == '1') ? 1 : 0;
    k_mma_union_small<<<NG, kBuildThreads, small, st>>>(N, woff, cells, slots, unions, nch, retry, all);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // the groups the first pass listed (usually few; the grid exits at once when none)
    k_mma_union_large<<<mma_sms(), kBuildThreads, large, st>>>(N, woff, cells, slots, unions, nch, retry, over);
    return cudaGetLastError();
}

cudaError_t launch_mma_layout(int pass, int N, const long long* woff, const unsigned short* slots, const float* wts,
                              const int* nch, const long long* cbase, int* ccnt, const long long* coff, uint2* ent,
                              float* scale, cudaStream_t st)
{
    const int NG = mma_group_count(N);
    if (NG <= 0) return cudaSuccess;
    if (pass == 0)
        k_mma_layout<0><<<NG, kLayoutThreads, 0, st>>>(N, woff, slots, wts, nch, cbase, ccnt, coff, ent, scale);
    else
        k_mma_layout<1><<<NG, kLayoutThreads, 0, st>>>(N, woff, slots, wts, nch, cbase, ccnt, coff, ent, scale);
    return cudaGetLastError();
}

cudaError_t launch_solar_slab16(const DevGeom& g, int T, const uint32_t* shadow, int words32, const HourEntry* table,
                                int j0, void* slab16, cudaStream_t st)
{
    if (T <= 0) return cudaSuccess;
    const long long warps = ((long long)T + kSlabCellsPerWarp - 1) / kSlabCellsPerWarp * (kHours / 32);
    k_solar_slab16<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(g.geo_n, T, shadow, words32, table, j0,
                                                                          static_cast<__half*>(slab16));
    return cudaGetLastError();
}

cudaError_t launch_reflect_mma(const void* slab16, const MmaLists& ml, const DevGeom& g, const uint32_t* shadow,
                               int words32, const HourEntry* table, int j0, const Accum& acc, int* err,
                               cudaStream_t st)
{
    const int NG = mma_group_count(ml.N);
    if (NG <= 0) return cudaSuccess;
    static std::atomic<bool> attr[kMaxDevices];
    cudaError_t e = allow_smem(k_reflect_mma, (size_t)kSmemBytes, attr);
    if (e != cudaSuccess) return e;
    if (!ml.sched) return cudaErrorInvalidValue;
    MmaTiles mt{ml.N, NG, ml.order, ml.woff, ml.cells, ml.unions, ml.cbase, ml.coff,
                reinterpret_cast<const uint2*>(ml.ent), ml.scale, ml.sched};
    const int grid = mma_grid(ml.N);
    k_reflect_mma<<<grid, kThreads, kSmemBytes, st>>>(static_cast<const __half*>(slab16), mt, g.geo_n, shadow,
                                                       words32, table, j0, acc, err);
    return cudaGetLastError();
}

}  // namespace sgb
