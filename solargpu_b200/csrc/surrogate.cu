// BF16 GEMM on the 5th-generation tensor cores (tcgen05), for the sky-bin
// visibility surrogate:   C[M][N] (f32) = A[M][K] (bf16) x B[N][K]^T (bf16)
// (+ bias[N], optional ReLU, optional bf16 copy of the result).
//
// One CTA of 128 threads per 128 x 128 output tile.  Per K step of 64:
//   * the 4 warps copy the A and B tiles (128 x 64 bf16 each) from global
//     memory into shared memory in the canonical K-major layout without
//     swizzle: core matrices of 8 rows x 16 bytes (8 bf16), core matrix
//     (row group g, K block b) at byte (b * 16 + g) * 128, so the leading
//     (K-direction) byte offset is 2048 and the stride (row-direction) one
//     is 128;
//   * a proxy fence makes the generic-proxy stores visible to the tensor
//     core, and one elected thread issues 4 tcgen05.mma (K = 16 each,
//     M = 128, N = 128, f32 accumulator in 128 TMEM columns), then
//     tcgen05.commit arrives on an mbarrier that all threads wait on
//     (bounded by the global timer, like every wait in this library).
// Epilogue: each warp reads its 32 TMEM lanes (rows) with tcgen05.ld
// 32x32b.x8, adds the bias, applies ReLU and stores rows of C.
// The TMEM columns are allocated by warp 0 at the start and freed at the end.
// M and N must be multiples of 128, K a multiple of 64 (the caller pads).
#include "sgb_internal.cuh"

#include <cuda_bf16.h>

namespace sgb {
namespace {

constexpr int kTm = 128, kTn = 128, kTk = 64;
constexpr int kGemmThreads = 128;
// Each CTA holds 128 TMEM columns; 14 KB of (unused) dynamic shared memory on
// top of the 33 KB of tiles keeps at most 4 CTAs on an SM, so the 512
// columns always suffice and tcgen05.alloc never waits.
constexpr int kGemmSmemPad = 14 * 1024;
constexpr unsigned long long kGemmWaitNs = 1000000000ull;   // 1 s

__device__ __forceinline__ unsigned s_u32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long g_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool wait_parity(unsigned bar, unsigned parity)
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
            const unsigned long long t = g_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > kGemmWaitNs) return false;
        }
    }
}

// Shared-memory matrix descriptor, K-major, no swizzle (version 1 = sm_100).
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::f16: f32 accumulator, bf16 A and B, both
// K-major, N = 128, M = 128.
constexpr unsigned kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(kTn >> 3) << 17) |
                            ((unsigned)(kTm >> 4) << 24);

// Copies a 128 x 64 bf16 tile (rows r0.., columns k0..) of a row-major
// matrix with `ld` elements per row into the canonical layout.
__device__ __forceinline__ void load_tile(unsigned char* dst, const __nv_bfloat16* __restrict__ src, int ld,
                                          int r0, int k0)
{
#pragma unroll
    for (int i = 0; i < (kTm * kTk / 8) / kGemmThreads; ++i) {
        const int c = threadIdx.x + kGemmThreads * i;   // 16-byte chunk: row c / 8, K block c % 8
        const int row = c >> 3, kb = c & 7;
        const uint4 v = *reinterpret_cast<const uint4*>(src + (size_t)(r0 + row) * ld + k0 + 8 * kb);
        *reinterpret_cast<uint4*>(dst + (kb * (kTm / 8) + (row >> 3)) * 128 + (row & 7) * 16) = v;
    }
}

__global__ void __launch_bounds__(kGemmThreads)
k_gemm_bf16(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B, float* __restrict__ C,
            __nv_bfloat16* __restrict__ Cb, const float* __restrict__ bias, int M, int N, int K, int relu,
            int* __restrict__ err)
{
    __shared__ __align__(128) unsigned char sa[kTm * kTk * 2];
    __shared__ __align__(128) unsigned char sb[kTn * kTk * 2];
    __shared__ __align__(8) unsigned long long mma_bar;
    __shared__ unsigned tmem_base;
    __shared__ int s_fail;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * kTm, n0 = blockIdx.x * kTn;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_u32(&tmem_base)),
                     "r"(kTn));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&mma_bar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_base;

    const unsigned a0 = s_u32(sa), b0 = s_u32(sb);
    constexpr unsigned kLbo = (kTm / 8) * 128, kSbo = 128;
    unsigned phase = 0;
    for (int k0 = 0; k0 < K; k0 += kTk) {
        load_tile(sa, A, K, m0, k0);
        load_tile(sb, B, K, n0, k0);
        // generic-proxy shared stores -> visible to the tensor core's async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int s = 0; s < kTk / 16; ++s) {
                const unsigned long long da = smem_desc(a0 + 2 * s * kLbo, kLbo, kSbo);
                const unsigned long long db = smem_desc(b0 + 2 * s * kLbo, kLbo, kSbo);
                const unsigned acc = (k0 > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(s_u32(&mma_bar)) : "memory");
        }
        // the MMAs read shared memory: wait for them before the next copy
        if (!wait_parity(s_u32(&mma_bar), phase)) s_fail = 1;   // bounded
        phase ^= 1u;
        __syncthreads();
        if (s_fail) break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (!s_fail) {
        // epilogue: warp w holds rows 32w.. of the tile (TMEM lanes 32w..)
        const int row = m0 + 32 * warp + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < kTn; c0 += 8) {
            unsigned r[8];
            const unsigned taddr = tmem + ((unsigned)(32 * warp) << 16) + (unsigned)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                v[j] = __uint_as_float(r[j]) + (bias ? bias[n0 + c0 + j] : 0.0f);
                if (relu) v[j] = fmaxf(v[j], 0.0f);
            }
            if (C) {
                float4* dst = reinterpret_cast<float4*>(C + (size_t)row * N + n0 + c0);
                dst[0] = make_float4(v[0], v[1], v[2], v[3]);
                dst[1] = make_float4(v[4], v[5], v[6], v[7]);
            }
            if (Cb) {
                __nv_bfloat162 h[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                *reinterpret_cast<uint4*>(Cb + (size_t)row * N + n0 + c0) = *reinterpret_cast<uint4*>(h);
            }
        }
    } else if (threadIdx.x == 0) {
        atomicOr(err, kErrWaitTimeout);
        wait_parity(s_u32(&mma_bar), phase ^ 1u);   // once more (bounded) before the TMEM is freed
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTn));
}

}  // namespace

cudaError_t launch_gemm_bf16(const void* A, const void* B, float* C, void* Cb, const float* bias, int M, int N,
                             int K, int relu, int* err, cudaStream_t st)
{
    if (M <= 0 || N <= 0 || K <= 0 || M % kTm || N % kTn || K % kTk) return cudaErrorInvalidValue;
    const dim3 grid(N / kTn, M / kTm);
    k_gemm_bf16<<<grid, kGemmThreads, kGemmSmemPad, st>>>(static_cast<const __nv_bfloat16*>(A),
                                                static_cast<const __nv_bfloat16*>(B), C,
                                                static_cast<__nv_bfloat16*>(Cb), bias, M, N, K, relu, err);
    return cudaGetLastError();
}

}  // namespace sgb

extern "C" {

int solar_gpu_gemm_bf16(const void* A, const void* B, float* C, void* C_bf16, const float* bias, int M, int N,
                        int K, int relu, void* stream)
{
    if (!A || !B || (!C && !C_bf16) || ((uintptr_t)A | (uintptr_t)B | (uintptr_t)C | (uintptr_t)C_bf16) % 16) {
        sgb::set_last_error("gemm: null or misaligned (16-byte) pointers");
        return -1;
    }
    int* err = nullptr;
    cudaError_t e = cudaMallocAsync(&err, sizeof(int), (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), (cudaStream_t)stream);
    if (e == cudaSuccess) e = sgb::launch_gemm_bf16(A, B, C, C_bf16, bias, M, N, K, relu, err, (cudaStream_t)stream);
    int flag = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (err) cudaFreeAsync(err, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        sgb::set_last_error(cudaGetErrorString(e));
        return e == cudaErrorInvalidValue ? -1 : -2;
    }
    if (flag) {
        sgb::set_last_error("tensor-core GEMM: a bounded wait expired");
        return -5;
    }
    return 0;
}

}  // extern "C"
