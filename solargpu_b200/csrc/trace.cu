// Stage 1: hemispherical DDA viewshed over the heightmap.
//
// The per-ray arithmetic follows the reference kernel
// calc_kernel_hemispherical_viewshed_GPU (src/cuda/kernels/viewshed_kernels.cu:7-59)
// operation for operation, with explicit round-to-nearest intrinsics so the
// hit cell is bit-identical: the ray height oz + Cdir.z * t is one fused
// multiply-add, exactly as nvcc contracts it in the reference build.
//
// The B200 layout differs from the reference:
//   * one launch traces all 2592 directions (the reference launches once per
//     direction and synchronises after each);
//   * a warp holds 32 consecutive voxels that walk the same direction in
//     lockstep, so height loads of neighbouring rays share cache lines;
//   * hits go to a per-voxel raw row [chunk][D] written 16 directions at a
//     time as 64-byte vectors; the first-occurrence dedupe (the reference's
//     O(k) global-memory scan per hit, viewshed_kernels.cu:49-55) is a
//     separate warp-per-voxel pass with a shared-memory hash set and
//     ballot/popc compaction that keeps direction order;
//   * shadow bits are packed 32 per word, voxel-major ([N][words32]), and
//     written once per word;
//   * an upper ray also ends, with no hit, once it rises above every cell it
//     can still reach (the early-exit tables of cone.cu): the reference's
//     result with fewer steps.
#include "sgb_internal.cuh"

#include <algorithm>
#include <cstdlib>

namespace sgb {
namespace {

constexpr int kTraceBlock = 128;
constexpr int kDirParts = 32;      // blocks per voxel block, each 1/32 of the directions (16: +0.6% at 1024^2)
constexpr int kDedupeWarps = 4;
constexpr int kHashSlots = 4096;   // > 2592 possible distinct hits per voxel
constexpr int kDedupeBatch = 9;    // 2592 = 9 batches of 9 rounds of 32 directions

// The tracer reads the heightmap from a copy with a one-cell border of +inf
// ([H + 2][W + 2], cell (x, y) at (x + 1) + (y + 1) * (W + 2)).  A ray that
// steps off the grid meets the border, whose height test is always true, so
// the loop needs no per-axis step counts; the cell it stopped on tells a
// border stop (no hit, as the reference's bounds check) from a hit.  Heights
// inside the grid are the caller's, +inf included.  Each load's index is
// clamped into the copy (one unsigned min a step), so every load stays inside
// it whatever the float tests do; a ray never leaves the copy (the border
// ends it first), and one that did would end on the clamped border cell and
// return -1.  (The clamp measured 2.7% faster than a compare and branch.)
//
// With CONE, an upper ray also reads its direction's early-exit table
// (cone.cu) every kBoundEvery steps: a ray above the bound of a cell it has
// passed can hit nothing from there on (every later cell is reachable from
// that cell), so it ends with no hit, as the reference's range test would
// end it or as it would leave the grid.  (Reading the bound every step,
// packed with the height, cost more in loads than the steps it saved.)
constexpr int kBoundEvery = 12;   // steps between bound checks (4: +7.4%, 8: +1.4%, 16: +1.7% at 1024^2)

__device__ __forceinline__ void dda_step(float& t, float& tMaxX, float& tMaxY, int& cell, int sx, int step_y,
                                         const DirEntry& d)
{
    // one step, as selects: lanes that step on different axes stay
    // converged (measured 119.6 -> 116.5 ms at 1024^2 against branches)
    const bool xs = tMaxX < tMaxY;
    t = fminf(tMaxX, tMaxY);   // = xs ? tMaxX : tMaxY (equal when not xs and equal)
    cell += xs ? sx : step_y;
    const float nx = __fadd_rn(tMaxX, d.dX), ny = __fadd_rn(tMaxY, d.dY);
    tMaxX = xs ? nx : tMaxX;
    tMaxY = xs ? tMaxY : ny;
}

template <bool UP, bool CONE>
__device__ __forceinline__ int trace_ray(const float* __restrict__ gpad, const float* __restrict__ bound, int W,
                                         int H, float maxz, int gx, int gy, float base_z, const DirEntry& d)
{
    // Cdir * 2.0f is exact, so these match the reference fused or not.
    const float ox = __fadd_rn((float)gx, __fmul_rn(d.cx, 2.0f));
    const float oy = __fadd_rn((float)gy, __fmul_rn(d.cy, 2.0f));
    const float oz = __fadd_rn(base_z, __fmul_rn(d.cz, 2.0f));
    int ix = __float2int_rd(ox);
    int iy = __float2int_rd(oy);
    const bool px = d.cx >= 0.0f;
    const bool py = d.cy >= 0.0f;
    float tMaxX = __fdiv_rn(px ? __fsub_rn(__fadd_rn((float)ix, 1.0f), ox) : __fsub_rn(ox, (float)ix), d.ax);
    float tMaxY = __fdiv_rn(py ? __fsub_rn(__fadd_rn((float)iy, 1.0f), oy) : __fsub_rn(oy, (float)iy), d.ay);
    const int sx = px ? 1 : -1;
    const int sy = py ? 1 : -1;
    // The first step checks both coordinates (the start cell, never tested,
    // may lie up to two cells outside the grid); after it the ray is inside
    // and moves one cell a step, so it stops on the border at the latest.
    float t;
    if (tMaxX < tMaxY) { t = tMaxX; ix += sx; tMaxX = __fadd_rn(tMaxX, d.dX); }
    else               { t = tMaxY; iy += sy; tMaxY = __fadd_rn(tMaxY, d.dY); }
    if ((unsigned)ix >= (unsigned)W || (unsigned)iy >= (unsigned)H) return 0;
    // A start height of NaN or +inf gives no hit in the reference (every test
    // on it is false, or true only for the height range); it would also keep
    // the border test false, so it ends here.  -inf still stops on the border.
    if (oz != oz || oz == __int_as_float(0x7f800000)) return 0;
    const int Wp = W + 2;
    const int step_y = py ? Wp : -Wp;
    int cell = (ix + 1) + (iy + 1) * Wp;
    const unsigned last = (unsigned)Wp * (unsigned)(H + 2) - 1u;
    float zr;
    // the reference tests the height range before the hit; both end the ray,
    // and which one it was is decided once, after the loop
    if constexpr (CONE) {
        for (;;) {
            // The bound of the cell the group of steps starts on also bounds
            // every cell after it, so its load has the whole group to arrive.
            const float b = __ldg(bound + min((unsigned)cell, last));
#pragma unroll
            for (int k = 0; k < kBoundEvery; ++k) {
                zr = __fmaf_rn(d.cz, t, oz);
                if (zr > maxz || __fsub_rn(__ldg(gpad + min((unsigned)cell, last)), zr) > 0.01f) goto stopped;
                dda_step(t, tMaxX, tMaxY, cell, sx, step_y, d);
            }
            if (__fmaf_rn(d.cz, t, oz) > b) return (unsigned)cell > last ? -1 : 0;
        }
    } else {
        for (;;) {
            zr = __fmaf_rn(d.cz, t, oz);
            if ((UP ? (zr > maxz) : (zr < 0.0f)) || __fsub_rn(__ldg(gpad + min((unsigned)cell, last)), zr) > 0.01f)
                goto stopped;
            dda_step(t, tMaxX, tMaxY, cell, sx, step_y, d);
        }
    }
stopped:
    if ((unsigned)cell > last) return -1;
    if (UP ? (zr > maxz) : (zr < 0.0f)) return 0;
    const int r = cell / Wp, q = cell - r * Wp;
    if (q == 0 || q > W || r == 0 || r > H) return 0;   // the border: the ray left the grid
    return (q - 1) + (r - 1) * W + 1;
}

// 16 blocks of 128 threads per SM: at most 32 registers a thread, so the SM
// holds 64 warps of rays (measured 116.4 -> 109.7 ms at 1024^2 against 38
// registers and 12 blocks).
__global__ void __launch_bounds__(kTraceBlock, 16)
k_trace(DevScene s, const DirEntry* __restrict__ dirs, int D, int words32,
        int voxel_offset, int chunk_count, int* __restrict__ raw, uint32_t* __restrict__ shadow,
        const int* __restrict__ perm, int* __restrict__ err)
{
    __shared__ int stage[kRawGroup][kTraceBlock];
    const int lv = blockIdx.x * kTraceBlock + threadIdx.x;
    const bool active = lv < chunk_count;
    // Row lv traces voxel voxel_offset + perm[lv] (visiting order: Morton-
    // adjacent lanes walk similar rays) or voxel_offset + lv.
    const int v = voxel_offset + (perm ? __ldg(perm + (active ? lv : 0)) : (active ? lv : 0));
    const int top = __ldg(s.pix_parent + v);
    const int gx = top % s.W;
    const int gy = top / s.W;
    const float base_z = (v < s.T) ? __ldg(s.grid + top) : __ldg(s.wall_z + (v - s.T));

    // this block's directions: groups [gb, ge) of kRawGroup
    const int ngroups = (D + kRawGroup - 1) / kRawGroup;
    const int gb = (int)((long long)ngroups * blockIdx.y / gridDim.y);
    const int ge = (int)((long long)ngroups * (blockIdx.y + 1) / gridDim.y);
    uint32_t acc = 0;
    int cur_word = -1;
    int* row = raw + (size_t)(active ? lv : 0) * D;
    for (int g0 = gb * kRawGroup; g0 < ge * kRawGroup; g0 += kRawGroup) {
        for (int k = 0; k < kRawGroup; ++k) {
            const DirEntry d = dirs[g0 + k];
            // up/down and the table are the same for the whole warp (one direction at a time)
            int hit = 0;
            if (active) {
                if (!((d.meta >> 16) & 1))
                    hit = trace_ray<false, false>(s.gpad, nullptr, s.W, s.H, s.maxz, gx, gy, base_z, d);
                else if (s.cone)
                    hit = trace_ray<true, true>(s.gpad, s.cone + s.cone_stride * ((d.meta >> 17) & (kMaxConeTables - 1)),
                                                s.W, s.H, s.maxz, gx, gy, base_z, d);
                else
                    hit = trace_ray<true, false>(s.gpad, nullptr, s.W, s.H, s.maxz, gx, gy, base_z, d);
            }
            if (hit < 0) {
                atomicOr(err, kErrTraceBounds);
                hit = 0;
            }
            stage[k][threadIdx.x] = hit;
            const int dense = (d.meta & 0xFFFF) - 1;   // warp-uniform
            if (dense >= 0) {
                const int w = dense >> 5;
                if (w != cur_word) {
                    // a word may be shared with the neighbouring direction part
                    if (active && acc) atomicOr(shadow + (size_t)v * words32 + cur_word, acc);
                    acc = 0;
                    cur_word = w;
                }
                if (hit) acc |= 1u << (dense & 31);
            }
        }
        if (active) {
            int4* dst = reinterpret_cast<int4*>(row + g0);
#pragma unroll
            for (int q = 0; q < kRawGroup / 4; ++q)
                dst[q] = make_int4(stage[4 * q][threadIdx.x], stage[4 * q + 1][threadIdx.x],
                                   stage[4 * q + 2][threadIdx.x], stage[4 * q + 3][threadIdx.x]);
        }
    }
    if (active && acc && cur_word >= 0) atomicOr(shadow + (size_t)v * words32 + cur_word, acc);
}

__global__ void k_pad_grid(const float* __restrict__ grid, int W, int H, float* __restrict__ gpad)
{
    const int Wp = W + 2;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)Wp * (H + 2)) return;
    const int x = (int)(i % Wp) - 1, y = (int)(i / Wp) - 1;
    // the load is clamped into the grid, so it stays in bounds however the
    // select below is compiled
    const float h = grid[(size_t)min(max(y, 0), H - 1) * W + min(max(x, 0), W - 1)];
    gpad[i] = (x >= 0 && x < W && y >= 0 && y < H) ? h : __int_as_float(0x7f800000);
}

__device__ __forceinline__ uint32_t hash_slot(uint32_t x, int bits)
{
    x *= 0x9E3779B1u;
    return x >> (32 - bits);
}

// One warp per voxel: keeps the first occurrence of each hit id in direction
// order and compacts the row in place; counts[perm[lv]] = list length.
//
// SLOTS is the warp's shared-memory hash set.  The first pass uses a small
// set (4 KB a warp, so many warps fit an SM) and gives up on a voxel whose
// insert needs more than kProbes probes: it then writes nothing of the round
// it is in and records the row in `ovf`.  Rounds before it were compacted in
// place and the ones after it are untouched, so every entry between the
// compacted prefix and the current round repeats an id of the prefix: the
// second pass (4096 slots, more than the 2592 possible distinct ids) run over
// the whole row gives the same first-occurrence list.
constexpr int kSmallSlots = 1024;
constexpr int kProbes = 32;   // default probe bound of the first pass (SGB_DEDUPE_PROBES overrides it)

template <int SLOTS, bool FIRST>
__global__ void __launch_bounds__(kDedupeWarps * 32)
k_dedupe(int chunk_count, int D, int* __restrict__ raw, int* __restrict__ counts, int* __restrict__ err,
         const int* __restrict__ perm, int* __restrict__ ovf, int probes)
{
    constexpr int kBits = SLOTS == 4096 ? 12 : SLOTS == 1024 ? 10 : 0;
    static_assert(kBits > 0, "hash set of 1024 or 4096 slots");
    extern __shared__ uint32_t tab_all[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    uint32_t* tab = tab_all + warp * SLOTS;
    // FIRST: row lv; else rows listed in ovf[1..ovf[0]], grid-strided
    const int w0 = blockIdx.x * kDedupeWarps + warp;
    const int nrows = FIRST ? chunk_count : ovf[0];
    for (int wi = w0; wi < nrows; wi += FIRST ? nrows : gridDim.x * kDedupeWarps) {
        const int lv = FIRST ? wi : ovf[1 + wi];
        uint4* t4 = reinterpret_cast<uint4*>(tab);
        for (int i = lane; i < SLOTS / 4; i += 32) t4[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();
        int* row = raw + (size_t)lv * D;
        int n = 0;
        bool gave_up = false;
        // Rounds of 32 directions, kDedupeBatch rounds loaded ahead (they are
        // all read before any in-place write can reach their slots).
        for (int base = 0; base < D && !gave_up; base += 32 * kDedupeBatch) {
            int hv[kDedupeBatch];
#pragma unroll
            for (int u = 0; u < kDedupeBatch; ++u) {
                const int d = base + 32 * u + lane;
                hv[u] = (d < D) ? row[d] : 0;
            }
#pragma unroll
            for (int u = 0; u < kDedupeBatch; ++u) {
                const int h = hv[u];
                const unsigned same = __match_any_sync(0xFFFFFFFFu, h);
                const bool leader = (__ffs(same) - 1) == lane;
                bool fresh = false, full = false;
                if (h != 0 && leader) {
                    uint32_t slot = hash_slot((uint32_t)h, kBits);
                    const int bound = FIRST ? probes : SLOTS;
                    int probe = 0;
                    for (; probe < bound; ++probe) {
                        const uint32_t old = atomicCAS(&tab[slot], 0u, (uint32_t)h);
                        if (old == 0u) { fresh = true; break; }
                        if (old == (uint32_t)h) break;
                        slot = (slot + 1) & (SLOTS - 1);
                    }
                    full = probe == bound;
                }
                if (__any_sync(0xFFFFFFFFu, full)) {
                    if (FIRST) {
                        if (lane == 0) ovf[1 + atomicAdd(ovf, 1)] = lv;
                    } else if (lane == 0) {
                        atomicOr(err, kErrHashFull);
                    }
                    gave_up = true;
                    break;
                }
                const unsigned bal = __ballot_sync(0xFFFFFFFFu, fresh);
                // Writes land below base + 32 * (u + 1): every slot there was read.
                if (fresh) row[n + __popc(bal & ((1u << lane) - 1u))] = h;
                n += __popc(bal);
            }
        }
        if (!gave_up && lane == 0) counts[perm ? perm[lv] : lv] = n;
        __syncwarp();
        if (FIRST) break;
    }
}

// ---- exclusive scan of int counts into int64 offsets (3 phases) ----------
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ long long warp_incl_scan(long long x, int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Block-wide exclusive scan; returns this thread's exclusive prefix and the block total.
__device__ long long block_excl_scan(long long x, long long* total)
{
    __shared__ long long warp_sums[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long inc = warp_incl_scan(x, lane);
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        long long ws = lane < nw ? warp_sums[lane] : 0;
        ws = warp_incl_scan(ws, lane);
        if (lane < nw) warp_sums[lane] = ws;
    }
    __syncthreads();
    const long long before = warp > 0 ? warp_sums[warp - 1] : 0;
    *total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + inc - x;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_tiles(const int* __restrict__ counts, int n, long long* __restrict__ offsets,
             long long* __restrict__ tile_sums)
{
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    long long v[kScanItems];
    long long local = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = (base + i < n) ? counts[base + i] : 0;
        local += v[i];
    }
    long long total;
    long long run = block_excl_scan(local, &total);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) offsets[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_tile_sums(long long* __restrict__ tile_sums, int ntiles, long long base,
                 long long* __restrict__ offsets, int n)
{
    long long carry = base;
    for (int i0 = 0; i0 < ntiles; i0 += kScanThreads) {
        const int i = i0 + threadIdx.x;
        const long long x = i < ntiles ? tile_sums[i] : 0;
        long long total;
        const long long ex = block_excl_scan(x, &total);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) offsets[n] = carry;
}

__global__ void k_scan_add(long long* __restrict__ offsets, int n, const long long* __restrict__ tile_sums)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) offsets[i] += tile_sums[i / kScanTile];
}

__global__ void __launch_bounds__(256)
k_gather_csr(int chunk_count, int D, const int* __restrict__ raw, const long long* __restrict__ offsets,
             int* __restrict__ csr_ids, const int* __restrict__ inv)
{
    const int lv = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (lv >= chunk_count) return;
    const long long o = offsets[lv];
    const int k = (int)(offsets[lv + 1] - o);
    const int* row = raw + (size_t)(inv ? inv[lv] : lv) * D;
    for (int i = lane; i < k; i += 32) csr_ids[o + i] = row[i];
}

}  // namespace

cudaError_t launch_pad_grid(const float* grid, int W, int H, float* gpad, cudaStream_t st)
{
    const long long n = (long long)(W + 2) * (H + 2);
    if (n <= 0) return cudaSuccess;
    k_pad_grid<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(grid, W, H, gpad);
    return cudaGetLastError();
}

cudaError_t launch_trace(const DevScene& s, const DirEntry* dirs, int D, int words32,
                         int voxel_offset, int chunk_count, int* raw, uint32_t* shadow,
                         const int* perm, int* err, cudaStream_t st)
{
    if (chunk_count <= 0) return cudaSuccess;
    if (!s.gpad) return cudaErrorInvalidValue;
    // D is a multiple of kRawGroup (rows are written kRawGroup directions at a time)
    if (D % kRawGroup != 0) return cudaErrorInvalidValue;
    const dim3 grid((chunk_count + kTraceBlock - 1) / kTraceBlock, kDirParts);
    k_trace<<<grid, kTraceBlock, 0, st>>>(s, dirs, D, words32, voxel_offset, chunk_count, raw, shadow, perm, err);
    return cudaGetLastError();
}

cudaError_t launch_dedupe(int chunk_count, int D, int* raw, int* counts, int* err, const int* perm, int* ovf,
                          cudaStream_t st)
{
    if (chunk_count <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(ovf, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    const size_t small = (size_t)kDedupeWarps * kSmallSlots * sizeof(uint32_t);
    const int grid = (chunk_count + kDedupeWarps - 1) / kDedupeWarps;
    // The probe bound only decides which rows go to the second pass (the
    // lists are the same either way); tests lower it to exercise that pass.
    int probes = kProbes;
    if (const char* env = std::getenv("SGB_DEDUPE_PROBES")) probes = std::max(1, std::min(kSmallSlots, std::atoi(env)));
    k_dedupe<kSmallSlots, true><<<grid, kDedupeWarps * 32, small, st>>>(chunk_count, D, raw, counts, err, perm, ovf,
                                                                         probes);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // the rows the first pass gave up on (usually none: the grid exits at once)
    const size_t big = (size_t)kDedupeWarps * kHashSlots * sizeof(uint32_t);
    e = cudaFuncSetAttribute(k_dedupe<kHashSlots, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_dedupe<kHashSlots, false><<<3 * sms, kDedupeWarps * 32, big, st>>>(chunk_count, D, raw, counts, err, perm, ovf,
                                                                          kHashSlots);
    return cudaGetLastError();
}

size_t scan_scratch_elems(int n)
{
    return (size_t)((n + kScanTile - 1) / kScanTile) + 1;
}

cudaError_t launch_scan_counts(const int* counts, int n, long long base, long long* offsets,
                               long long* block_sums, int* /*unused*/, cudaStream_t st)
{
    const int ntiles = (n + kScanTile - 1) / kScanTile;
    if (n > 0) k_scan_tiles<<<ntiles, kScanThreads, 0, st>>>(counts, n, offsets, block_sums);
    k_scan_tile_sums<<<1, kScanThreads, 0, st>>>(block_sums, ntiles, base, offsets, n);
    if (n > 0) k_scan_add<<<(n + 255) / 256, 256, 0, st>>>(offsets, n, block_sums);
    return cudaGetLastError();
}

cudaError_t launch_gather_csr(int chunk_count, int D, const int* raw, const long long* offsets,
                              int* csr_ids, const int* inv, cudaStream_t st)
{
    if (chunk_count <= 0) return cudaSuccess;
    const long long threads = (long long)chunk_count * 32;
    k_gather_csr<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(chunk_count, D, raw, offsets, csr_ids, inv);
    return cudaGetLastError();
}

namespace {
__global__ void k_invert(const int* __restrict__ perm, int n, int* __restrict__ inv)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inv[perm[i]] = i;
}
}  // namespace

namespace {
__global__ void k_chunk_flags(const int* __restrict__ order, int N, int v0, int n, int* __restrict__ flag)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < N) flag[p] = (unsigned)(order[p] - v0) < (unsigned)n ? 1 : 0;
}

__global__ void k_chunk_scatter(const int* __restrict__ order, int N, int v0, const int* __restrict__ flag,
                                const long long* __restrict__ pos, int* __restrict__ perm)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < N && flag[p]) perm[pos[p]] = order[p] - v0;
}
}  // namespace

cudaError_t launch_chunk_order(const int* order, int N, int v0, int n, int* flag, long long* pos,
                               long long* scan_tmp, int* perm, cudaStream_t st)
{
    if (N <= 0 || n <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((N + 255) / 256);
    k_chunk_flags<<<grid, 256, 0, st>>>(order, N, v0, n, flag);
    cudaError_t e = launch_scan_counts(flag, N, 0, pos, scan_tmp, nullptr, st);
    if (e != cudaSuccess) return e;
    k_chunk_scatter<<<grid, 256, 0, st>>>(order, N, v0, flag, pos, perm);
    return cudaGetLastError();
}

cudaError_t launch_invert(const int* perm, int n, int* inv, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_invert<<<(n + 255) / 256, 256, 0, st>>>(perm, n, inv);
    return cudaGetLastError();
}

}  // namespace sgb
