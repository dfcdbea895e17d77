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
//     cudaGetSymbolAddress (with that device current) and keeps it; make that
//     first call before any stream capture on the device.
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
    for (long long k = lane; k < len; k += 32) row[k] = ids[s + k];
    if (lane == 0) counts[i] = (int)len;
}

std::mutex g_mu;
unsigned char* g_addr[kMaxDevices] = {};   // device address of the scratch, per device ordinal

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
        if (!g_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);   // this device's copy of the array
            if (e != cudaSuccess) return report(SOLAR_GPU_ERR_CUDA, "cudaGetSymbolAddress", e);
            g_addr[dev] = static_cast<unsigned char*>(p);
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
    if (flag) return report(SOLAR_GPU_ERR_ARG, "a list is longer than 2592 ids", cudaSuccess);
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
