// ba-RLE encoding of caller-provided CSR neighbor lists without any device
// allocation (solar_gpu_barle_encode_noalloc in include/solargpu_b200.h).
//
// Who needs this: a caller whose device memory belongs to someone else --
// an engine or simulation framework that reserves the GPU's memory up front
// and forbids allocations outside its own pool, or a latency-critical loop
// that cannot afford cudaMalloc/cudaFree (both can synchronise the whole
// device).  Such a caller hands in device buffers for the lists and for the
// output; every temporary this encoder needs (a padded row per list, which
// the encoder sorts in place, per-list counts and sizes, the scan's partial
// sums and an error flag) lives in one fixed static device array below.
//
// Limits and sharing:
//   * at most kNoAllocLists lists per call, each at most kNoAllocRowLen ids
//     (the tracer emits at most one id per traced direction, so its lists
//     never exceed that); larger requests are rejected before device work;
//   * the array exists once on every device that loads this library and stays
//     allocated until the process exits (about 10.6 MB);
//   * every call on a device uses the same array and leaves its contents
//     behind; what must start at zero is cleared by each call; two calls
//     whose work overlaps on the GPU (different streams, or host threads
//     without ordering between them) race on the array and corrupt each
//     other's results -- serialise them;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and keeps it, keyed by
//     the device's current CUDA context: after cudaDeviceReset, or once the
//     primary context was destroyed and created again, the next call looks
//     the address up again.  Make the first call in each context before any
//     stream capture on the device;
//   * each list must hold distinct ids >= 1 (the tracer's lists always do);
//     the reference encoder would drop duplicates and stop at a 0, so such
//     lists are rejected instead of being encoded differently.
#include <cuda.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "solargpu_b200.h"
#include "sgb_internal.cuh"

namespace sgb {
namespace {

constexpr int kNoAllocLists = 1024;
constexpr int kNoAllocRowLen = kMaxDirs;   // 2592: one id per traced direction at most
constexpr int kMaxDevices = 64;
constexpr int kErrBadIds = 1 << 16;         // a zero, negative or repeated id (this file's own flag bit)

// Scratch layout (bytes): rows | counts | sizes | scan partial sums | error flag
constexpr size_t kRowsBytes = sizeof(int) * (size_t)kNoAllocLists * kNoAllocRowLen;
constexpr size_t kCountsOff = kRowsBytes;
constexpr size_t kSizesOff = kCountsOff + sizeof(int) * kNoAllocLists;
constexpr size_t kScanOff = kSizesOff + sizeof(int) * kNoAllocLists;
constexpr size_t kScanBytes = sizeof(long long) * 64;
constexpr size_t kErrOff = kScanOff + kScanBytes;
constexpr size_t kScratchBytes = kErrOff + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Copies list i of the caller's CSR into padded row i of the scratch.
__global__ void k_rows_from_csr(const long long* __restrict__ off, const int* __restrict__ ids, int n,
                                int* __restrict__ rows, int* __restrict__ counts, int* __restrict__ err)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const long long s = off[i];
    const long long len = off[i + 1] - s;
    if (len < 0 || len > kNoAllocRowLen) {
        if (lane == 0) { counts[i] = 0; atomicOr(err, kErrListCapacity); }
        return;
    }
    int* row = rows + (size_t)i * kNoAllocRowLen;
    bool bad = false;
    for (long long k = lane; k < len; k += 32) {
        const int id = ids[s + k];
        bad |= id < 1;
        row[k] = id;
    }
    if (__any_sync(0xFFFFFFFFu, bad) && lane == 0) atomicOr(err, kErrBadIds);
    if (lane == 0) counts[i] = (int)len;
}

// After the size pass each row holds its list sorted descending; a repeated
// id shows up as two equal neighbours.
__global__ void k_check_distinct(int n, const int* __restrict__ rows, const int* __restrict__ counts,
                                 int* __restrict__ err)
{
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const int k = counts[i];
    const int* row = rows + (size_t)i * kNoAllocRowLen;
    bool dup = false;
    for (int j = lane + 1; j < k; j += 32) dup |= row[j] == row[j - 1];
    if (__any_sync(0xFFFFFFFFu, dup) && lane == 0) atomicOr(err, kErrBadIds);
}

std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};              // device address of the scratch, per device ordinal
unsigned long long g_ctx_id[kMaxDevices] = {};        // ...valid in the context with this id

// Unique id of the calling thread's current context (cuCtxGetId: never reused
// within a process), 0 if the driver cannot tell.
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {   // called under g_mu
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(p);
        looked_up = true;
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS) return id;
    return 0;
}

int report(int code, const char* what, cudaError_t e)
{
    char buf[256];
    std::snprintf(buf, sizeof(buf), "solar_gpu_barle_encode_noalloc: %s%s%s", what,
                  e == cudaSuccess ? "" : ": ", e == cudaSuccess ? "" : cudaGetErrorString(e));
    if (e != cudaSuccess) cudaGetLastError();
    set_last_error(buf);
    return code;
}

}  // namespace
}  // namespace sgb

extern "C" int solar_gpu_barle_encode_noalloc(const long long* csr_offsets, const int* csr_ids, int num_lists,
                                              long long* barle_offsets, unsigned char* barle_bytes,
                                              long long barle_capacity, long long* barle_total,
                                              void* stream)
{
    using namespace sgb;
    if (num_lists < 0 || num_lists > kNoAllocLists)
        return report(SOLAR_GPU_ERR_ARG, "num_lists must be in [0, 1024]", cudaSuccess);
    if (!csr_offsets || !barle_offsets || !barle_total || (num_lists > 0 && !csr_ids))
        return report(SOLAR_GPU_ERR_ARG, "a required pointer is NULL", cudaSuccess);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return report(SOLAR_GPU_ERR_NO_DEVICE, "cudaGetDevice", e);
    if (dev < 0 || dev >= kMaxDevices) return report(SOLAR_GPU_ERR_ARG, "device ordinal above 63", cudaSuccess);
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        // No context may be current yet on a first call: the lookup creates
        // the primary context, and its id is read after it.
        const unsigned long long ctx_id = current_context_id();
        if (!g_addr[dev] || ctx_id == 0 || ctx_id != g_ctx_id[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);   // this device's copy of the array
            if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "cudaGetSymbolAddress", e);
            g_addr[dev] = static_cast<unsigned char*>(p);
            g_ctx_id[dev] = current_context_id();
        }
        base = g_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    int* rows = reinterpret_cast<int*>(base);
    int* counts = reinterpret_cast<int*>(base + kCountsOff);
    int* sizes = reinterpret_cast<int*>(base + kSizesOff);
    long long* scan = reinterpret_cast<long long*>(base + kScanOff);
    int* err = reinterpret_cast<int*>(base + kErrOff);

    e = cudaMemsetAsync(err, 0, sizeof(int), st);   // the error flag must start at zero
    if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "clearing the error flag", e);
    if (num_lists > 0) {
        k_rows_from_csr<<<(num_lists * 32 + 255) / 256, 256, 0, st>>>(csr_offsets, csr_ids, num_lists, rows,
                                                                        counts, err);
        e = cudaGetLastError();
        if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "row copy", e);
        e = launch_barle_size(num_lists, kNoAllocRowLen, rows, counts, sizes, err, st);
        if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "size pass", e);
        k_check_distinct<<<(num_lists * 32 + 255) / 256, 256, 0, st>>>(num_lists, rows, counts, err);
        e = cudaGetLastError();
        if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "id check", e);
    }
    e = launch_scan_counts(sizes, num_lists, 0, barle_offsets, scan, nullptr, st);
    if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "offset scan", e);
    long long total = 0;
    int flag = 0;
    e = cudaMemcpyAsync(&total, barle_offsets + num_lists, sizeof(long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "reading the stream size", e);
    *barle_total = total;
    if (flag & kErrListCapacity)
        return report(SOLAR_GPU_ERR_ARG, "a list is longer than 2592 ids (or its offsets decrease)", cudaSuccess);
    if (flag & kErrBadIds)
        return report(SOLAR_GPU_ERR_ARG, "a list holds an id below 1 or the same id twice", cudaSuccess);
    if (flag) return report(SOLAR_GPU_ERR_DEVICE_CHECK, "device check failed in the size pass", cudaSuccess);
    if (total > barle_capacity || (total > 0 && !barle_bytes))
        return report(SOLAR_GPU_ERR_ARG, "barle_capacity is smaller than *barle_total", cudaSuccess);
    if (num_lists > 0 && total > 0) {
        e = launch_barle_write(num_lists, kNoAllocRowLen, rows, counts, barle_offsets, barle_bytes, err, st);
        if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "write pass", e);
        e = cudaMemcpyAsync(&flag, err, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "write pass", e);
        if (flag) return report(SOLAR_GPU_ERR_DEVICE_CHECK, "device check failed while writing", cudaSuccess);
    }
    return SOLAR_GPU_OK;
}
