// ba-RLE writer on the GPU, byte-exact to the reference host encoder
// (src/barle_compression.cpp:156-187, format in include/barle_compression.h:7-44):
//   ids sorted descending (the lists are already unique), deltas with the
//   first value absolute, width classes 4/8/16/24/32 bits, maximal
//   same-width runs, the two-pass run optimiser, runs split at 255, then
//   blocks of <= 8 runs: 3 big-endian bytes of 3-bit codes (pad 7), one
//   length byte per run, then payload (4-bit deltas two per byte, high nibble
//   first; wider deltas big-endian).
//
// One warp per voxel.  The sort (bitonic, shared memory), delta/width
// classification and run detection (ballot + popc) are warp-parallel; the
// run optimiser is the reference's sequential fixpoint and runs on one lane
// over the (short) run list; payload bytes are written lane-parallel.
// Two passes: k_barle_size computes each stream's byte count (and leaves the
// sorted list and, room permitting, its optimised runs in the row), a scan
// turns counts into offsets, k_barle_write packs the bytes.
#include "sgb_internal.cuh"

namespace sgb {
namespace {

constexpr int kEncWarps = 4;        // large instance
constexpr int kIdsCap = 4096;
constexpr int kRunsCap = 2624;
constexpr int kSmallWarps = 8;      // small instance
constexpr int kSmallIds = 1024;
constexpr int kW4 = 0, kEnd = 7;

__device__ __forceinline__ int width_class(uint32_t x)
{
    return x <= 15u ? 0 : x <= 255u ? 1 : x <= 65535u ? 2 : x <= 16777215u ? 3 : 4;
}

__device__ __forceinline__ uint32_t delta_at(const uint32_t* ids, int i)
{
    return i == 0 ? ids[0] : ids[i - 1] - ids[i];
}

__device__ __forceinline__ uint32_t pack_run(int w, int len) { return ((uint32_t)w << 24) | (uint32_t)len; }
__device__ __forceinline__ int run_w(uint32_t r) { return (int)(r >> 24); }
__device__ __forceinline__ int run_len(uint32_t r) { return (int)(r & 0xFFFFFFu); }

// Descending bitonic sort of s[0..n2) (n2 a power of two >= 32), warp-wide.
__device__ void warp_sort_desc(uint32_t* s, int n2, int lane)
{
    for (int size = 2; size <= n2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = lane; t < (n2 >> 1); t += 32) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const bool desc = (i & size) == 0;
                const uint32_t a = s[i], b = s[j];
                if ((a < b) == desc) { s[i] = b; s[j] = a; }
            }
            __syncwarp();
        }
    }
}

// Builds the optimised run list of a sorted id list into runs[]; returns the
// run count (warp-uniform).  runs[r] = pack_run(width, len).
__device__ int build_runs(const uint32_t* ids, int k, uint32_t* runs, int lane)
{
    // 1. maximal same-width runs (detect_runs, barle_compression.cpp:90-105)
    int nr = 0;
    for (int base = 0; base < k; base += 32) {
        const int i = base + lane;
        int w = -1;
        bool start = false;
        if (i < k) {
            w = width_class(delta_at(ids, i));
            start = (i == 0) || (w != width_class(delta_at(ids, i - 1)));
        }
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, start);
        if (start) runs[nr + __popc(bal & ((1u << lane) - 1u))] = pack_run(w, i);   // len slot holds start
        nr += __popc(bal);
    }
    __syncwarp();
    // starts -> lengths
    for (int r0 = 0; r0 < nr; r0 += 32) {
        const int r = r0 + lane;
        uint32_t cur = 0, nxt_start = (uint32_t)k;
        if (r < nr) {
            cur = runs[r];
            if (r + 1 < nr) nxt_start = (uint32_t)run_len(runs[r + 1]);
        }
        __syncwarp();
        if (r < nr) runs[r] = pack_run(run_w(cur), (int)nxt_start - run_len(cur));
        __syncwarp();
    }
    // 2. optimize_runs (barle_compression.cpp:112-152), sequential on lane 0
    if (lane == 0 && nr >= 2) {
        bool changed = true, single = false;
        while (changed) {
            changed = false;
            int nn = 0, i = 0;
            while (i < nr - 1) {
                const uint32_t a = runs[i], b = runs[i + 1];
                if (run_len(b) == 1 && run_w(b) + 1 == run_w(a)) {
                    changed = true;
                    runs[nn++] = pack_run(run_w(a), run_len(a) + 1);
                    i += 2;
                } else {
                    runs[nn++] = a;
                    ++i;
                }
            }
            if (i < nr) runs[nn++] = runs[i];
            if (nn == 1) { nr = 1; single = true; break; }
            nr = nn;   // unchanged passes rewrite the same list
        }
        if (!single) {
            int nn = 0, i = 0;
            while (i < nr) {
                const int w = run_w(runs[i]);
                int len = run_len(runs[i]);
                int j = i + 1;
                while (j < nr && run_w(runs[j]) == w) { len += run_len(runs[j]); ++j; }
                runs[nn++] = pack_run(w, len);
                i = j;
            }
            nr = nn;
        }
    }
    nr = __shfl_sync(0xFFFFFFFFu, nr, 0);
    __syncwarp();
    return nr;
}

__device__ __forceinline__ int payload_bytes(int w, int len)
{
    return w == kW4 ? (len + 1) >> 1 : len * w;
}

__device__ int load_sorted(const int* row, int k, uint32_t* ids, int lane, bool sort)
{
    int n2 = 32;
    while (n2 < k) n2 <<= 1;
    for (int i = lane; i < n2; i += 32) ids[i] = i < k ? (uint32_t)row[i] : 0u;
    __syncwarp();
    if (sort) warp_sort_desc(ids, n2, lane);
    return n2;
}

// Two instances per pass: the small one (lists <= kSmallIds ids, 8 KB of
// shared memory per warp, 8 warps per block) takes almost every voxel; the
// large one takes only the longer lists (up to one id per direction).
template <int IDS, int RUNS, int WARPS, bool LARGE>
__global__ void __launch_bounds__(WARPS * 32)
k_barle_size(int chunk_count, int D, int* __restrict__ raw, const int* __restrict__ counts,
             int* __restrict__ sizes, int* __restrict__ err, const int* __restrict__ perm)
{
    extern __shared__ uint32_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* ids = smem + warp * (IDS + RUNS);
    uint32_t* runs = ids + IDS;
    const int lv = blockIdx.x * WARPS + warp;   // row
    if (lv >= chunk_count) return;
    const int u = perm ? perm[lv] : lv;          // voxel of the row
    const int k = counts[u];
    if (LARGE != (k > kSmallIds)) return;
    if (k <= 0) { if (lane == 0) sizes[u] = 0; return; }
    if (k > D || k > RUNS) { if (lane == 0) { sizes[u] = 0; atomicOr(err, kErrListCapacity); } return; }
    int* row = raw + (size_t)lv * D;
    load_sorted(row, k, ids, lane, true);
    for (int i = lane; i < k; i += 32) row[i] = (int)ids[i];   // keep the sorted list for the write pass
    const int nr = build_runs(ids, k, runs, lane);
    // and, where the row has room after the list, its optimised runs (the
    // write pass then skips build_runs): row[k] = run count, runs after it
    if (k < D) {
        const bool fits = k + 1 + nr <= D;
        if (lane == 0) row[k] = fits ? nr : -1;
        if (fits)
            for (int r = lane; r < nr; r += 32) row[k + 1 + r] = (int)runs[r];
    }
    int pieces = 0, payload = 0;
    for (int r = lane; r < nr; r += 32) {
        const int w = run_w(runs[r]), len = run_len(runs[r]);
        const int full = len / 255, rem = len % 255;
        pieces += full + (rem > 0);
        payload += full * payload_bytes(w, 255) + payload_bytes(w, rem);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        pieces += __shfl_xor_sync(0xFFFFFFFFu, pieces, o);
        payload += __shfl_xor_sync(0xFFFFFFFFu, payload, o);
    }
    if (lane == 0) sizes[u] = 3 * ((pieces + 7) / 8) + pieces + payload;
}

template <int IDS, int RUNS, int WARPS, bool LARGE>
__global__ void __launch_bounds__(WARPS * 32)
k_barle_write(int chunk_count, int D, const int* __restrict__ raw, const int* __restrict__ counts,
              const long long* __restrict__ offsets, unsigned char* __restrict__ out,
              int* __restrict__ err, const int* __restrict__ inv)
{
    extern __shared__ uint32_t smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* ids = smem + warp * (IDS + RUNS);
    uint32_t* runs = ids + IDS;
    const int lv = blockIdx.x * WARPS + warp;
    if (lv >= chunk_count) return;
    const int k = counts[lv];
    if (LARGE != (k > kSmallIds)) return;
    if (k <= 0 || k > D || k > RUNS) return;
    const int* row = raw + (size_t)(inv ? inv[lv] : lv) * D;
    load_sorted(row, k, ids, lane, false);   // already sorted by k_barle_size
    // the runs k_barle_size left after the list, else built again
    int nr = k < D ? row[k] : -1;
    if (nr >= 0 && k + 1 + nr <= D) {
        for (int r = lane; r < nr; r += 32) runs[r] = (uint32_t)row[k + 1 + r];
        __syncwarp();
    } else {
        nr = build_runs(ids, k, runs, lane);
    }
    // split_long_runs (barle_compression.cpp:29-44), expanded in place from the back
    if (lane == 0) {
        int ns = 0;
        for (int r = 0; r < nr; ++r) ns += (run_len(runs[r]) + 254) / 255;
        int pos = ns;
        for (int r = nr - 1; r >= 0; --r) {
            const int w = run_w(runs[r]), len = run_len(runs[r]);
            const int np = (len + 254) / 255;
            pos -= np;
            for (int p = np - 1; p >= 0; --p) {
                const int pl = (p == np - 1) ? len - 255 * (np - 1) : 255;
                runs[pos + p] = pack_run(w, pl);
            }
        }
        nr = ns;
    }
    nr = __shfl_sync(0xFFFFFFFFu, nr, 0);
    __syncwarp();
    unsigned char* dst = out + offsets[lv];
    const long long limit = offsets[lv + 1] - offsets[lv];
    long long boff = 0;
    int estart = 0;
    for (int p = 0; p < nr; ++p) {
        if ((p & 7) == 0) {
            const int cnt = min(8, nr - p);
            if (lane == 0) {
                uint32_t bits = 0;
                for (int j = 0; j < 8; ++j) {
                    const int code = (j < cnt) ? run_w(runs[p + j]) : kEnd;
                    bits |= (uint32_t)(code & 7) << ((7 - j) * 3);
                }
                if (boff + 3 + cnt <= limit) {
                    dst[boff] = (unsigned char)(bits >> 16);
                    dst[boff + 1] = (unsigned char)(bits >> 8);
                    dst[boff + 2] = (unsigned char)bits;
                }
            }
            if (lane < cnt && boff + 3 + cnt <= limit) dst[boff + 3 + lane] = (unsigned char)run_len(runs[p + lane]);
            boff += 3 + cnt;
        }
        const int w = run_w(runs[p]), len = run_len(runs[p]);
        const int nb = payload_bytes(w, len);
        if (boff + nb > limit) { if (lane == 0) atomicOr(err, kErrListCapacity); return; }
        if (w == kW4) {
            for (int b = lane; b < nb; b += 32) {
                const int e = estart + 2 * b;
                const uint32_t v1 = delta_at(ids, e);
                const uint32_t v2 = (2 * b + 1 < len) ? delta_at(ids, e + 1) : 0u;
                dst[boff + b] = (unsigned char)((v1 << 4) | (v2 & 0x0Fu));
            }
        } else {
            for (int i = lane; i < len; i += 32) {
                const uint32_t x = delta_at(ids, estart + i);
                unsigned char* q = dst + boff + (long long)i * w;
                for (int b = 0; b < w; ++b) q[b] = (unsigned char)(x >> (8 * (w - 1 - b)));
            }
        }
        boff += nb;
        estart += len;
    }
}

}  // namespace

template <int IDS, int RUNS, int WARPS, bool LARGE>
cudaError_t size_pass(int chunk_count, int D, int* raw, const int* counts, int* sizes, int* err, const int* perm,
                      cudaStream_t st)
{
    const size_t smem = (size_t)WARPS * (IDS + RUNS) * sizeof(uint32_t);
    cudaError_t e = cudaFuncSetAttribute(k_barle_size<IDS, RUNS, WARPS, LARGE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_barle_size<IDS, RUNS, WARPS, LARGE><<<(chunk_count + WARPS - 1) / WARPS, WARPS * 32, smem, st>>>(
        chunk_count, D, raw, counts, sizes, err, perm);
    return cudaGetLastError();
}

template <int IDS, int RUNS, int WARPS, bool LARGE>
cudaError_t write_pass(int chunk_count, int D, const int* raw, const int* counts, const long long* offsets,
                       unsigned char* out, int* err, const int* inv, cudaStream_t st)
{
    const size_t smem = (size_t)WARPS * (IDS + RUNS) * sizeof(uint32_t);
    cudaError_t e = cudaFuncSetAttribute(k_barle_write<IDS, RUNS, WARPS, LARGE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_barle_write<IDS, RUNS, WARPS, LARGE><<<(chunk_count + WARPS - 1) / WARPS, WARPS * 32, smem, st>>>(
        chunk_count, D, raw, counts, offsets, out, err, inv);
    return cudaGetLastError();
}

cudaError_t launch_barle_size(int chunk_count, int D, int* raw, const int* counts, int* sizes, int* err,
                              const int* perm, cudaStream_t st)
{
    if (chunk_count <= 0) return cudaSuccess;
    cudaError_t e = size_pass<kSmallIds, kSmallIds, kSmallWarps, false>(chunk_count, D, raw, counts, sizes, err,
                                                                        perm, st);
    if (e != cudaSuccess) return e;
    return size_pass<kIdsCap, kRunsCap, kEncWarps, true>(chunk_count, D, raw, counts, sizes, err, perm, st);
}

cudaError_t launch_barle_write(int chunk_count, int D, const int* raw, const int* counts,
                               const long long* offsets, unsigned char* out, int* err, const int* inv,
                               cudaStream_t st)
{
    if (chunk_count <= 0) return cudaSuccess;
    cudaError_t e = write_pass<kSmallIds, kSmallIds, kSmallWarps, false>(chunk_count, D, raw, counts, offsets,
                                                                         out, err, inv, st);
    if (e != cudaSuccess) return e;
    return write_pass<kIdsCap, kRunsCap, kEncWarps, true>(chunk_count, D, raw, counts, offsets, out, err, inv, st);
}

cudaError_t launch_barle_size(int chunk_count, int D, int* raw, const int* counts,
                              int* sizes, int* err, cudaStream_t st)
{
    return launch_barle_size(chunk_count, D, raw, counts, sizes, err, nullptr, st);
}

cudaError_t launch_barle_write(int chunk_count, int D, const int* raw, const int* counts,
                               const long long* offsets, unsigned char* out, int* err,
                               cudaStream_t st)
{
    return launch_barle_write(chunk_count, D, raw, counts, offsets, out, err, nullptr, st);
}

}  // namespace sgb
