// BF16 GEMM on the 5th-generation tensor cores (tcgen05), for the sky-bin
// visibility surrogate:   C[M][N] (f32) = A[M][K] (bf16) x B[N][K]^T (bf16)
// (+ bias[N], optional ReLU, optional bf16 copy of the result).
//
// One CTA of 128 threads per 128 x BN output tile (BN = 256 when N allows,
// 64 for 64-wide outputs, else 128), K in steps of 64 through a ring of kGemmStages shared-memory
// stages:
//   * thread 0 (producer) loads each stage with tensor-map TMA, one box of
//     64 bf16 (128 bytes) x rows per operand, 128-byte swizzle: this is the
//     canonical K-major SWIZZLE_128B layout the tensor core reads (8-row
//     atoms of 1024 bytes, 16-byte chunks XOR-ed with the row within the
//     atom); completion is counted in bytes on the stage's full mbarrier;
//   * thread 32 (MMA issuer) waits for a stage, issues 4 tcgen05.mma (K = 16
//     each, 32 bytes further along the swizzled rows; M = 128, N = BN, f32
//     accumulator in BN TMEM columns) and tcgen05.commit frees the stage
//     (empty mbarrier) when they complete; a last commit signals the
//     epilogue;
//   * epilogue: each warp reads its 32 TMEM lanes (rows) with tcgen05.ld
//     32x32b.x8, adds the bias, applies ReLU and stores rows of C.
// Every wait is bounded by the global timer; on expiry the kernel flags the
// error, lets its TMA copies and MMAs finish (bounded), frees TMEM and exits.
// M and N must be multiples of 128, K a multiple of 64 (the caller pads).
#include "sgb_internal.cuh"

#include <atomic>

#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>

namespace sgb {
namespace {

constexpr int kTm = 128, kTk = 64;
constexpr int kGemmThreads = 128;
constexpr int kGemmStages = 4;
constexpr unsigned long long kGemmWaitNs = 1000000000ull;   // 1 s

template <int BN>
struct GemmShape {
    static constexpr int kStageA = kTm * kTk * 2, kStageB = BN * kTk * 2;     // 16 KB, 16/32 KB
    static constexpr int kStage = kStageA + kStageB;
    static constexpr int kSmem = kGemmStages * kStage + 1024;              // + alignment slack
    // Instruction descriptor, kind::f16: f32 accumulator, bf16 A and B,
    // both K-major, N = BN, M = 128.
    static constexpr unsigned kIdesc =
        (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(BN >> 3) << 17) | ((unsigned)(kTm >> 4) << 24);
};

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

__device__ __forceinline__ bool wait_parity(unsigned bar, unsigned parity, const volatile int* fail,
                                            unsigned long long limit_ns = kGemmWaitNs)
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
            const unsigned long long t = g_ns();
            if (t0 == 0) t0 = t;
            else if (t - t0 > limit_ns) return false;
        }
    }
}

// Shared-memory matrix descriptor, K-major, 128-byte swizzle (layout type 2,
// version 1 = sm_100): stride between 8-row atoms 1024 bytes, leading offset
// unused (16 bytes), atoms 1024-byte aligned so the base offset is 0.
__device__ __forceinline__ unsigned long long smem_desc_sw128(unsigned addr)
{
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | (1ull << 16) | ((unsigned long long)(1024 >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}

__device__ __forceinline__ void tma_box(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(dst), "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(bar)
                 : "memory");
}

template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1)
k_gemm_bf16(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
            float* __restrict__ C, __nv_bfloat16* __restrict__ Cb, const float* __restrict__ bias, int M, int N, int K,
            int relu, int* __restrict__ err, int stall)
{
    extern __shared__ __align__(1024) unsigned char gsm[];
    __shared__ __align__(8) unsigned long long full[kGemmStages], empty[kGemmStages], done;
    __shared__ unsigned tmem_base;
    __shared__ volatile int s_fail;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    using S = GemmShape<BN>;
    const int m0 = blockIdx.y * kTm, n0 = blockIdx.x * BN;
    // 1024-byte aligned stage ring
    const unsigned base = (s_u32(gsm) + 1023u) & ~1023u;
    const int nk = K / kTk;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_u32(&tmem_base)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kGemmStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&full[s])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&empty[s])), "r"(1));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&done)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_base;

    int issued = 0;   // producer: stages loaded
    if (threadIdx.x == 0) {
        // ---- producer (stall: issues nothing, so the MMA thread's bounded
        // wait runs out; the self-test of the error path)
        for (int k = 0; k < (stall ? 0 : nk); ++k) {
            const int s = k % kGemmStages;
            if (k >= kGemmStages &&
                !wait_parity(s_u32(&empty[s]), (unsigned)(((k / kGemmStages) - 1) & 1), &s_fail)) {
                s_fail = 1;
                break;
            }
            const unsigned sa = base + (unsigned)(s * S::kStage), sb = sa + S::kStageA;
            const unsigned fb = s_u32(&full[s]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                         "r"((unsigned)S::kStage) : "memory");
            tma_box(sa, &mapA, k * kTk, m0, fb);
            tma_box(sb, &mapB, k * kTk, n0, fb);
            ++issued;
        }
    } else if (threadIdx.x == 32) {
        // ---- MMA issuer
        int k = 0;
        for (; k < nk; ++k) {
            const int s = k % kGemmStages;
            if (!wait_parity(s_u32(&full[s]), (unsigned)((k / kGemmStages) & 1), &s_fail)) {
                s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned sa = base + (unsigned)(s * S::kStage), sb = sa + S::kStageA;
#pragma unroll
            for (int j = 0; j < kTk / 16; ++j) {
                const unsigned long long da = smem_desc_sw128(sa + 32u * j);
                const unsigned long long db = smem_desc_sw128(sb + 32u * j);
                const unsigned acc = (k > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(S::kIdesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
            }
            // the stage is free once these MMAs have read it
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(s_u32(&empty[s])) : "memory");
        }
        // all MMAs issued so far complete -> epilogue
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     ::"r"(s_u32(&done)) : "memory");
    }
    // everyone: the accumulator is ready (or the run failed)
    // longer than the pipeline's waits, so a failed pipeline always signals first
    if (!wait_parity(s_u32(&done), 0u, nullptr, 2 * kGemmWaitNs)) s_fail = 1;
    __syncthreads();
    const bool ok = !s_fail;   // uniform over the CTA
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (ok) {
        // epilogue: warp w holds rows 32w.. of the tile (TMEM lanes 32w..)
        const int row = m0 + 32 * warp + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 8) {
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
        // let the TMA copies this thread issued land before the CTA exits
        for (int k = (issued > kGemmStages ? issued - kGemmStages : 0); k < issued; ++k)
            wait_parity(s_u32(&full[k % kGemmStages]), (unsigned)((k / kGemmStages) & 1), nullptr);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

// Persistent form for grids of more than one wave: one CTA per SM walks the
// tiles blockIdx.x, blockIdx.x + gridDim.x, ... with 6 warps:
//   * warp 0 (one thread) loads the shared-memory ring by TMA, its stage
//     counter running on across tiles;
//   * warp 1 allocates two accumulators of BN TMEM columns and one thread
//     issues the MMAs of tile i into accumulator i % 2, then commits to that
//     accumulator's full barrier;
//   * warps 2..5 are the epilogue: warp w reads TMEM lanes 32 (w % 4) ..
//     (rows of the tile), stores them and arrives on the accumulator's empty
//     barrier, so tile i's epilogue overlaps tile i + 1's MMAs.
// Every wait is bounded and checks a shared failure flag, so all roles leave
// their loops once one wait runs out; a last commit lets the MMAs in flight
// finish and the TMA thread waits for its copies before TMEM is freed.
constexpr int kPersThreads = 192;

template <int BN>
__global__ void __launch_bounds__(kPersThreads, 1)
k_gemm_bf16_pers(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                 float* __restrict__ C, __nv_bfloat16* __restrict__ Cb, const float* __restrict__ bias, int M, int N,
                 int K, int relu, int* __restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char gsm[];
    __shared__ __align__(8) unsigned long long full[kGemmStages], empty[kGemmStages], tfull[2], tempty[2], done;
    __shared__ unsigned tmem_base;
    __shared__ volatile int s_fail;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    using S = GemmShape<BN>;
    const unsigned base = (s_u32(gsm) + 1023u) & ~1023u;
    const int nk = K / kTk;
    const int ntn = N / BN;
    const int ntiles = (M / kTm) * ntn;
    const int my_tiles = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s_u32(&tmem_base)),
                     "r"(2 * BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kGemmStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&full[s])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&empty[s])), "r"(1));
        }
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&tfull[b])), "r"(1));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&tempty[b])), "r"(4));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_u32(&done)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_fail = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_base;

    long long issued = 0;   // TMA thread: stages loaded
    if (threadIdx.x == 0) {
        // ---- TMA
        long long g = 0;
        for (int i = 0; i < my_tiles && !s_fail; ++i) {
            const int t = (int)blockIdx.x + i * (int)gridDim.x;
            const int m0 = (t / ntn) * kTm, n0 = (t % ntn) * BN;
            for (int k = 0; k < nk; ++k, ++g) {
                const int s = (int)(g % kGemmStages);
                if (g >= kGemmStages &&
                    !wait_parity(s_u32(&empty[s]), (unsigned)(((g / kGemmStages) - 1) & 1), &s_fail)) {
                    s_fail = 1;
                    break;
                }
                const unsigned sa = base + (unsigned)(s * S::kStage), sb = sa + S::kStageA;
                const unsigned fb = s_u32(&full[s]);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb),
                             "r"((unsigned)S::kStage) : "memory");
                tma_box(sa, &mapA, k * kTk, m0, fb);
                tma_box(sb, &mapB, k * kTk, n0, fb);
                ++issued;
            }
        }
    } else if (threadIdx.x == 32) {
        // ---- MMA
        long long g = 0;
        for (int i = 0; i < my_tiles; ++i) {
            const int b = i & 1;
            if (i >= 2 && !wait_parity(s_u32(&tempty[b]), (unsigned)(((i >> 1) - 1) & 1), &s_fail)) {
                s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned acc_cols = tmem + (unsigned)(b * BN);
            bool bad = false;
            for (int k = 0; k < nk; ++k, ++g) {
                const int s = (int)(g % kGemmStages);
                if (!wait_parity(s_u32(&full[s]), (unsigned)((g / kGemmStages) & 1), &s_fail)) {
                    bad = true;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned sa = base + (unsigned)(s * S::kStage), sb = sa + S::kStageA;
#pragma unroll
                for (int j = 0; j < kTk / 16; ++j) {
                    const unsigned long long da = smem_desc_sw128(sa + 32u * j);
                    const unsigned long long db = smem_desc_sw128(sb + 32u * j);
                    const unsigned acc = (k > 0 || j > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                        ::"r"(acc_cols), "l"(da), "l"(db), "r"(S::kIdesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(s_u32(&empty[s])) : "memory");
            }
            if (bad) {
                s_fail = 1;
                break;
            }
            // accumulator b holds tile i once these MMAs complete
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(s_u32(&tfull[b])) : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     ::"r"(s_u32(&done)) : "memory");
    } else if (warp >= 2) {
        // ---- epilogue: this warp's TMEM lanes are rows 32q .. 32q + 31 of the tile
        const int q = warp & 3;
        for (int i = 0; i < my_tiles; ++i) {
            const int b = i & 1;
            if (!wait_parity(s_u32(&tfull[b]), (unsigned)((i >> 1) & 1), &s_fail)) {
                s_fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int t = (int)blockIdx.x + i * (int)gridDim.x;
            const int m0 = (t / ntn) * kTm, n0 = (t % ntn) * BN;
            const int row = m0 + 32 * q + lane;
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 8) {
                unsigned r[8];
                const unsigned taddr = tmem + ((unsigned)(32 * q) << 16) + (unsigned)(b * BN + c0);
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
            // the accumulator may be overwritten once all four warps have read it
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(s_u32(&tempty[b])) : "memory");
        }
    }
    // every MMA issued has completed (or the wait gave up after twice the pipeline's limit)
    if (!wait_parity(s_u32(&done), 0u, nullptr, 2 * kGemmWaitNs)) s_fail = 1;
    __syncthreads();
    if (s_fail && threadIdx.x == 0) {
        atomicOr(err, kErrWaitTimeout);
        // let this thread's TMA copies land before the CTA exits
        for (long long g = (issued > kGemmStages ? issued - kGemmStages : 0); g < issued; ++g)
            wait_parity(s_u32(&full[g % kGemmStages]), (unsigned)((g / kGemmStages) & 1), nullptr);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
}

// ---- surrogate training and inference kernels ------------------------------

constexpr int kPatch = 64;             // height patch side (cells) around the voxel's pixel
constexpr float kPatchScale = 1.0f / 50.0f;

// Features of voxel voxels[i]: the 64 x 64 heights around its pixel relative
// to the voxel's base height, / 50 m, clipped to [-2, 2] (outside the grid:
// ground at 0 m), then the voxel normal; zero padding up to `feat`.
__global__ void k_sg_features(const float* __restrict__ grid, int W, int H, int T, const int* __restrict__ pp,
                              const float* __restrict__ wall_z, const float* __restrict__ slopes,
                              const float* __restrict__ aspects, const int* __restrict__ voxels, int M, int feat,
                              __nv_bfloat16* __restrict__ out)
{
    const int i = blockIdx.y;
    if (i >= M) return;
    const int v = voxels[i];
    const int top = pp[v];
    const int gx = top % W, gy = top / W;
    const float z = v < T ? grid[top] : wall_z[v - T];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < feat; j += gridDim.x * blockDim.x) {
        float f = 0.0f;
        if (j < kPatch * kPatch) {
            const int x = gx + (j % kPatch) - kPatch / 2, y = gy + (j / kPatch) - kPatch / 2;
            const float h = (x >= 0 && x < W && y >= 0 && y < H) ? grid[y * W + x] : 0.0f;
            f = fminf(2.0f, fmaxf(-2.0f, (h - z) * kPatchScale));
        } else if (j < kPatch * kPatch + 3) {
            const float sl = slopes[v] * 0.017453292f, as = aspects[v] * 0.017453292f;
            const int c = j - kPatch * kPatch;
            f = c == 0 ? sinf(sl) * sinf(as) : c == 1 ? -sinf(sl) * cosf(as) : cosf(sl);
        }
        out[(size_t)i * feat + j] = __float2bfloat16_rn(f);
    }
}

// Labels: bit b (< active) of voxels[i]'s shadow words -> 1.0 (shadowed) / 0.0.
__global__ void k_sg_labels(const uint32_t* __restrict__ shadow, int words32, const int* __restrict__ voxels, int M,
                            int active, int outw, float* __restrict__ y)
{
    const int i = blockIdx.x, b = threadIdx.x;
    if (i >= M) return;
    const int v = voxels[i];
    for (int k = b; k < outw; k += blockDim.x)
        y[(size_t)i * outw + k] = k < active ? (float)((shadow[(size_t)v * words32 + (k >> 5)] >> (k & 31)) & 1u) : 0.0f;
}

// Mean binary cross-entropy with logits over the first `active` outputs:
// dZ = (sigmoid(Z) - Y) / (M * active) as bf16, loss sum into *loss.
__global__ void k_sg_bce(const float* __restrict__ Z, const float* __restrict__ Y, int M, int outw, int active,
                         __nv_bfloat16* __restrict__ dZ, float* __restrict__ loss)
{
    const long long n = (long long)M * outw;
    const float inv = 1.0f / ((float)M * (float)active);
    float part = 0.0f;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % outw);
        float g = 0.0f;
        if (k < active) {
            const float z = Z[t], y = Y[t];
            const float p = 1.0f / (1.0f + expf(-z));
            g = (p - y) * inv;
            part += fmaxf(z, 0.0f) - z * y + log1pf(expf(-fabsf(z)));
        }
        dZ[t] = __float2bfloat16_rn(g);
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, part * inv);
}

// dX = dY * (H > 0) as bf16 (ReLU backward through a stored activation).
__global__ void k_sg_relu_grad(const float* __restrict__ dY, const __nv_bfloat16* __restrict__ H, long long n,
                               __nv_bfloat16* __restrict__ dX)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        dX[t] = __float2bfloat16_rn(__bfloat162float(H[t]) > 0.0f ? dY[t] : 0.0f);
}

// out[c][r] = in[r][c] (bf16, 32 x 32 tiles through shared memory).
__global__ void k_sg_transpose(const __nv_bfloat16* __restrict__ in, int R, int C, __nv_bfloat16* __restrict__ out)
{
    __shared__ __nv_bfloat16 t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;   // row tiles on x (up to 2^31 - 1)
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < R && c < C) t[k][threadIdx.x] = in[(size_t)r * C + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < R && c < C) out[(size_t)c * R + r] = t[threadIdx.x][k];
    }
}

// out[c] += sum over the rows r0 .. r0 + rows_per_block of in[r][c] (bias
// gradients; out zeroed first, one atomic add per column and block).
__global__ void k_sg_colsum(const __nv_bfloat16* __restrict__ in, int R, int C, int rows_per_block,
                            float* __restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const int r0 = blockIdx.y * rows_per_block, r1 = min(R, r0 + rows_per_block);
    float s = 0.0f;
    for (int r = r0; r < r1; ++r) s += __bfloat162float(in[(size_t)r * C + c]);
    atomicAdd(out + c, s);
}

// Adam on FP32 master parameters; the bf16 copy feeds the GEMMs.
__global__ void k_sg_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                          float c2, __nv_bfloat16* __restrict__ pb)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const float gt = g[t];
        const float mt = b1 * m[t] + (1.0f - b1) * gt;
        const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
        m[t] = mt;
        v[t] = vt;
        const float q = p[t] - lr * (mt / c1) / (sqrtf(vt / c2) + eps);
        p[t] = q;
        if (pb) pb[t] = __float2bfloat16_rn(q);
    }
}

// ---- convolutional front end (4 x 4 kernels, stride 2, padding 1, NHWC) ----

constexpr int kCoarse = 8;   // cells per side of one context (max-pooled) cell

// out[cy][cx] = max of grid over the kCoarse x kCoarse cells of (cx, cy).
__global__ void k_sg_coarse(const float* __restrict__ grid, int W, int H, int Wc, int Hc, float* __restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Wc * Hc) return;
    const int cx = c % Wc, cy = c / Wc;
    float m = -3.0e38f;
    for (int y = cy * kCoarse; y < min(H, (cy + 1) * kCoarse); ++y)
        for (int x = cx * kCoarse; x < min(W, (cx + 1) * kCoarse); ++x) m = fmaxf(m, grid[y * W + x]);
    out[c] = m;
}

// Two-channel image of voxel voxels[i], NHWC [64][64][2]: channel 0 the
// heights of the 64 x 64 cells around its pixel, channel 1 the maxima of the
// 64 x 64 context cells (kCoarse x kCoarse cells each) around its context
// cell, both relative to the voxel's base height, / 50 m, clipped to [-2, 2]
// (outside the grid: 0 m).  nrm[i] = the voxel normal, zero-padded to 64.
__global__ void k_sg_image(const float* __restrict__ grid, const float* __restrict__ coarse, int W, int H, int T,
                           const int* __restrict__ pp, const float* __restrict__ wall_z,
                           const float* __restrict__ slopes, const float* __restrict__ aspects,
                           const int* __restrict__ voxels, int M, __nv_bfloat162* __restrict__ img,
                           __nv_bfloat16* __restrict__ nrm)
{
    const int i = blockIdx.y;
    if (i >= M) return;
    const int v = voxels[i];
    const int top = pp[v];
    const int gx = top % W, gy = top / W;
    const float z = v < T ? grid[top] : wall_z[v - T];
    const int Wc = (W + kCoarse - 1) / kCoarse, Hc = (H + kCoarse - 1) / kCoarse;
    const int cgx = gx / kCoarse, cgy = gy / kCoarse;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < kPatch * kPatch; j += gridDim.x * blockDim.x) {
        const int dx = (j % kPatch) - kPatch / 2, dy = (j / kPatch) - kPatch / 2;
        const int x = gx + dx, y = gy + dy, cx = cgx + dx, cy = cgy + dy;
        const float h = (x >= 0 && x < W && y >= 0 && y < H) ? grid[y * W + x] : 0.0f;
        const float hc = (cx >= 0 && cx < Wc && cy >= 0 && cy < Hc) ? coarse[cy * Wc + cx] : 0.0f;
        img[(size_t)i * kPatch * kPatch + j] = __floats2bfloat162_rn(fminf(2.0f, fmaxf(-2.0f, (h - z) * kPatchScale)),
                                                                     fminf(2.0f, fmaxf(-2.0f, (hc - z) * kPatchScale)));
    }
    if (blockIdx.x == 0 && threadIdx.x < 64) {
        const int c = threadIdx.x;
        float f = 0.0f;
        if (c < 3) {
            const float sl = slopes[v] * 0.017453292f, as = aspects[v] * 0.017453292f;
            f = c == 0 ? sinf(sl) * sinf(as) : c == 1 ? -sinf(sl) * cosf(as) : cosf(sl);
        }
        nrm[(size_t)i * 64 + c] = __float2bfloat16_rn(f);
    }
}

// im2col for a 4 x 4, stride-2, padding-1 convolution over X [B][Hi][Wi][Cin]:
// cols[(b * Ho + oy) * Wo + ox][(ky * 4 + kx) * Cin + c] = X[b][2oy-1+ky][2ox-1+kx][c]
// (0 outside the image), columns 16 * Cin .. Kp - 1 zero.  One thread per 8
// consecutive columns (Cin % 8 == 0: one 16-byte load and store).
__global__ void k_sg_im2col(const __nv_bfloat16* __restrict__ X, int B, int Hi, int Wi, int Cin, int Kp,
                            __nv_bfloat16* __restrict__ cols)
{
    const int Ho = Hi / 2, Wo = Wi / 2, K = 16 * Cin, g8 = Kp / 8;
    const long long n = (long long)B * Ho * Wo * g8;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long row = t / g8;
        const int k0 = (int)(t % g8) * 8;
        const int ox = (int)(row % Wo), oy = (int)((row / Wo) % Ho);
        const long long b = row / ((long long)Wo * Ho);
        uint4 out = make_uint4(0u, 0u, 0u, 0u);
        if (Cin % 8 == 0) {
            if (k0 < K) {
                const int tap = k0 / Cin, c = k0 % Cin;
                const int y = 2 * oy - 1 + tap / 4, x = 2 * ox - 1 + tap % 4;
                if (y >= 0 && y < Hi && x >= 0 && x < Wi)
                    out = *reinterpret_cast<const uint4*>(X + (((size_t)b * Hi + y) * Wi + x) * Cin + c);
            }
        } else {
            __nv_bfloat16 e[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = k0 + q;
                e[q] = __float2bfloat16_rn(0.0f);
                if (k < K) {
                    const int tap = k / Cin, c = k % Cin;
                    const int y = 2 * oy - 1 + tap / 4, x = 2 * ox - 1 + tap % 4;
                    if (y >= 0 && y < Hi && x >= 0 && x < Wi) e[q] = X[(((size_t)b * Hi + y) * Wi + x) * Cin + c];
                }
            }
            out = *reinterpret_cast<uint4*>(e);
        }
        *reinterpret_cast<uint4*>(cols + row * Kp + k0) = out;
    }
}

// Backward of k_sg_im2col fused with the ReLU of the layer below:
// g[b][y][x][c] = bf16( (X[b][y][x][c] > 0) * sum over the (<= 2 x 2) output
// positions whose 4 x 4 window covers (y, x) of dcols[row][tap * Cin + c] ).
// One thread per 8 channels (Cin % 8 == 0).
__global__ void k_sg_col2im_relu(const float* __restrict__ dcols, const __nv_bfloat16* __restrict__ X, int B, int Hi,
                                 int Wi, int Cin, int Kp, __nv_bfloat16* __restrict__ g)
{
    const int Ho = Hi / 2, Wo = Wi / 2, g8 = Cin / 8;
    const long long n = (long long)B * Hi * Wi * g8;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long pix = t / g8;
        const int c0 = (int)(t % g8) * 8;
        const int x = (int)(pix % Wi), y = (int)((pix / Wi) % Hi);
        const long long b = pix / ((long long)Wi * Hi);
        float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            const int oy = ((y + 1) >> 1) - a, ky = y + 1 - 2 * oy;
            if (oy < 0 || oy >= Ho) continue;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int ox = ((x + 1) >> 1) - e, kx = x + 1 - 2 * ox;
                if (ox < 0 || ox >= Wo) continue;
                const float4* src = reinterpret_cast<const float4*>(
                    dcols + (((size_t)b * Ho + oy) * Wo + ox) * Kp + (ky * 4 + kx) * Cin + c0);
                const float4 u = src[0], w = src[1];
                acc[0] += u.x; acc[1] += u.y; acc[2] += u.z; acc[3] += u.w;
                acc[4] += w.x; acc[5] += w.y; acc[6] += w.z; acc[7] += w.w;
            }
        }
        const uint4 xv = *reinterpret_cast<const uint4*>(X + (size_t)pix * Cin + c0);
        const __nv_bfloat16* xe = reinterpret_cast<const __nv_bfloat16*>(&xv);
        __nv_bfloat16 o[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) o[q] = __float2bfloat16_rn(__bfloat162float(xe[q]) > 0.0f ? acc[q] : 0.0f);
        *reinterpret_cast<uint4*>(g + (size_t)pix * Cin + c0) = *reinterpret_cast<uint4*>(o);
    }
}

// out[r] = [ a[r][0 .. wa) | b[r][0 .. wb) ]  (bf16 rows side by side).
__global__ void k_sg_hcat(const __nv_bfloat16* __restrict__ a, int wa, const __nv_bfloat16* __restrict__ b, int wb,
                          int rows, __nv_bfloat16* __restrict__ out)
{
    const int w = wa + wb;
    const long long n = (long long)rows * w;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long r = t / w;
        const int c = (int)(t % w);
        out[t] = c < wa ? a[r * wa + c] : b[r * wb + c - wa];
    }
}

// out[r][c] = bf16(dY[r][c] * (H[r][c] > 0)) for c < cols, with row strides
// (ReLU backward through the leading columns of a wider gradient).
__global__ void k_sg_relu_grad_cols(const float* __restrict__ dY, int ldy, const __nv_bfloat16* __restrict__ H,
                                    int ldh, int rows, int cols, __nv_bfloat16* __restrict__ out)
{
    const long long n = (long long)rows * cols;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long r = t / cols;
        const int c = (int)(t % cols);
        out[t] = __float2bfloat16_rn(__bfloat162float(H[r * ldh + c]) > 0.0f ? dY[r * ldy + c] : 0.0f);
    }
}

// out[c][r] = in[r][c] (f32, 32 x 32 tiles through shared memory).
__global__ void k_sg_transpose_f32(const float* __restrict__ in, int R, int C, float* __restrict__ out)
{
    __shared__ float t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;   // row tiles on x (up to 2^31 - 1)
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < R && c < C) t[k][threadIdx.x] = in[(size_t)r * C + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < R && c < C) out[(size_t)c * R + r] = t[threadIdx.x][k];
    }
}

}  // namespace

namespace {
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn()
{
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// Row-major [rows][K] bf16 matrix, boxes of 64 elements (128 bytes) x box_rows
// rows with 128-byte swizzle.
bool make_map(CUtensorMap* map, const void* ptr, int rows, int K, int box_rows)
{
    EncodeTiled fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kTk, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN>
cudaError_t launch_gemm_tiles(const void* A, const void* B, float* C, void* Cb, const float* bias, int M, int N,
                              int K, int relu, int* err, cudaStream_t st, int stall)
{
    CUtensorMap mapA, mapB;
    if (!make_map(&mapA, A, M, K, kTm) || !make_map(&mapB, B, N, K, BN)) return cudaErrorInvalidValue;
    static std::atomic<bool> attr[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev].load(std::memory_order_acquire)) {
        e = cudaFuncSetAttribute(k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, GemmShape<BN>::kSmem);
        if (e != cudaSuccess) return e;
        attr[dev].store(true, std::memory_order_release);
    }
    const int tiles = (M / kTm) * (N / BN);
    static std::atomic<int> sms_cached{0};
    int sms = sms_cached.load(std::memory_order_relaxed);
    if (!sms) {
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
        sms_cached.store(sms, std::memory_order_relaxed);
    }
    if (!stall && tiles > sms && !getenv("SGB_GEMM_ONE_TILE_PER_CTA")) {
        // more than one wave: persistent CTAs with two TMEM accumulators
        static std::atomic<bool> pattr[64];
        if (!pattr[dev].load(std::memory_order_acquire)) {
            e = cudaFuncSetAttribute(k_gemm_bf16_pers<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     GemmShape<BN>::kSmem);
            if (e != cudaSuccess) return e;
            pattr[dev].store(true, std::memory_order_release);
        }
        k_gemm_bf16_pers<BN><<<sms, kPersThreads, GemmShape<BN>::kSmem, st>>>(
            mapA, mapB, C, static_cast<__nv_bfloat16*>(Cb), bias, M, N, K, relu, err);
        return cudaGetLastError();
    }
    const dim3 grid(N / BN, M / kTm);
    k_gemm_bf16<BN><<<grid, kGemmThreads, GemmShape<BN>::kSmem, st>>>(
        mapA, mapB, C, static_cast<__nv_bfloat16*>(Cb), bias, M, N, K, relu, err, stall);
    return cudaGetLastError();
}
}  // namespace

// Tile width: 256 columns when N allows it and the grid still covers the
// SMs (148 on B200) at least once, 64 when N is not a multiple of 128,
// else 128.  SGB_GEMM_BN (64, 128, 256) forces a width that divides N.
cudaError_t launch_gemm_bf16(const void* A, const void* B, float* C, void* Cb, const float* bias, int M, int N,
                             int K, int relu, int* err, cudaStream_t st, int stall)
{
    if (M <= 0 || N <= 0 || K <= 0 || M % kTm || N % 64 || K % kTk) return cudaErrorInvalidValue;
    int bn = N % 128 ? 64 : (N % 256 == 0 && (long long)(M / kTm) * (N / 256) >= 148) ? 256 : 128;
    if (const char* force = getenv("SGB_GEMM_BN")) {
        const int f = atoi(force);
        if ((f == 64 || f == 128 || f == 256) && N % f == 0) bn = f;
    }
    switch (bn) {
    case 256: return launch_gemm_tiles<256>(A, B, C, Cb, bias, M, N, K, relu, err, st, stall);
    case 128: return launch_gemm_tiles<128>(A, B, C, Cb, bias, M, N, K, relu, err, st, stall);
    default: return launch_gemm_tiles<64>(A, B, C, Cb, bias, M, N, K, relu, err, st, stall);
    }
}

}  // namespace sgb

extern "C" {

namespace {
int sg_status(cudaError_t e)
{
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        sgb::set_last_error(cudaGetErrorString(e));
        return -2;
    }
    return 0;
}
unsigned sg_blocks(long long n) { return (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16); }
}  // namespace

int solar_gpu_sg_features(const float* grid, int W, int H, int T, const int* pixel_parent, const float* wall_z,
                          const float* slopes, const float* aspects, const int* voxels, int M, int feat,
                          void* out_bf16, void* stream)
{
    if (M <= 0) return 0;
    if (feat < 4096 + 3 || M > 65535) { sgb::set_last_error("features: feat >= 4099, M <= 65535"); return -1; }
    sgb::k_sg_features<<<dim3(4, M), 256, 0, (cudaStream_t)stream>>>(grid, W, H, T, pixel_parent, wall_z, slopes,
                                                                     aspects, voxels, M, feat,
                                                                     (__nv_bfloat16*)out_bf16);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_labels(const uint32_t* shadow, int words32, const int* voxels, int M, int active, int outw,
                        float* y, void* stream)
{
    if (M <= 0) return 0;
    if (active > outw || active > 32 * words32) { sgb::set_last_error("labels: active bins"); return -1; }
    sgb::k_sg_labels<<<M, 128, 0, (cudaStream_t)stream>>>(shadow, words32, voxels, M, active, outw, y);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_bce(const float* Z, const float* Y, int M, int outw, int active, void* dZ_bf16, float* loss,
                     void* stream)
{
    const long long n = (long long)M * outw;
    if (n <= 0) return 0;
    sgb::k_sg_bce<<<sg_blocks(n), 256, 0, (cudaStream_t)stream>>>(Z, Y, M, outw, active, (__nv_bfloat16*)dZ_bf16, loss);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_relu_grad(const float* dY, const void* H_bf16, long long n, void* dX_bf16, void* stream)
{
    if (n <= 0) return 0;
    sgb::k_sg_relu_grad<<<sg_blocks(n), 256, 0, (cudaStream_t)stream>>>(dY, (const __nv_bfloat16*)H_bf16, n,
                                                                        (__nv_bfloat16*)dX_bf16);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_transpose(const void* in_bf16, int R, int C, void* out_bf16, void* stream)
{
    if (R <= 0 || C <= 0) return 0;
    if ((C + 31) / 32 > 65535) { sgb::set_last_error("transpose: C < 2^21"); return -1; }
    sgb::k_sg_transpose<<<dim3((R + 31) / 32, (C + 31) / 32), dim3(32, 8), 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)in_bf16, R, C, (__nv_bfloat16*)out_bf16);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_colsum(const void* in_bf16, int R, int C, float* out, void* stream)
{
    if (R <= 0 || C <= 0) return 0;
    const int rpb = std::max(64, (R + 1023) / 1024);
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * (size_t)C, (cudaStream_t)stream);
    if (e != cudaSuccess) return sg_status(e);
    sgb::k_sg_colsum<<<dim3((C + 127) / 128, (R + rpb - 1) / rpb), 128, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)in_bf16, R, C, rpb, out);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                      float eps, int step, void* p_bf16, void* stream)
{
    if (n <= 0) return 0;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    sgb::k_sg_adam<<<sg_blocks(n), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2,
                                                                  (__nv_bfloat16*)p_bf16);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_coarse(const float* grid, int W, int H, float* out, void* stream)
{
    if (W <= 0 || H <= 0) return 0;
    const int Wc = (W + sgb::kCoarse - 1) / sgb::kCoarse, Hc = (H + sgb::kCoarse - 1) / sgb::kCoarse;
    sgb::k_sg_coarse<<<(Wc * Hc + 255) / 256, 256, 0, (cudaStream_t)stream>>>(grid, W, H, Wc, Hc, out);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_image(const float* grid, const float* coarse, int W, int H, int T, const int* pixel_parent,
                       const float* wall_z, const float* slopes, const float* aspects, const int* voxels, int M,
                       void* img_bf16, void* nrm_bf16, void* stream)
{
    if (M <= 0) return 0;
    if (M > 65535) { sgb::set_last_error("image: M <= 65535"); return -1; }
    sgb::k_sg_image<<<dim3(4, M), 256, 0, (cudaStream_t)stream>>>(grid, coarse, W, H, T, pixel_parent, wall_z, slopes,
                                                                  aspects, voxels, M, (__nv_bfloat162*)img_bf16,
                                                                  (__nv_bfloat16*)nrm_bf16);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_im2col(const void* X_bf16, int B, int Hi, int Wi, int Cin, int Kp, void* cols_bf16, void* stream)
{
    if (B <= 0) return 0;
    if (Hi % 2 || Wi % 2 || Cin <= 0 || Kp % 64 || Kp < 16 * Cin || (Cin % 8 && Cin > 4)) {
        sgb::set_last_error("im2col: even sides, Kp % 64 == 0, Kp >= 16 Cin, Cin % 8 == 0 or Cin <= 4");
        return -1;
    }
    const long long n = (long long)B * (Hi / 2) * (Wi / 2) * (Kp / 8);
    sgb::k_sg_im2col<<<sg_blocks(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)X_bf16, B, Hi, Wi, Cin, Kp,
                                                                     (__nv_bfloat16*)cols_bf16);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_col2im_relu(const float* dcols, const void* X_bf16, int B, int Hi, int Wi, int Cin, int Kp,
                             void* g_bf16, void* stream)
{
    if (B <= 0) return 0;
    if (Hi % 2 || Wi % 2 || Cin % 8 || Kp % 64 || Kp < 16 * Cin) {
        sgb::set_last_error("col2im: even sides, Cin % 8 == 0, Kp % 64 == 0, Kp >= 16 Cin");
        return -1;
    }
    const long long n = (long long)B * Hi * Wi * (Cin / 8);
    sgb::k_sg_col2im_relu<<<sg_blocks(n), 256, 0, (cudaStream_t)stream>>>(dcols, (const __nv_bfloat16*)X_bf16, B, Hi,
                                                                          Wi, Cin, Kp, (__nv_bfloat16*)g_bf16);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_hcat(const void* a_bf16, int wa, const void* b_bf16, int wb, int rows, void* out_bf16, void* stream)
{
    const long long n = (long long)rows * (wa + wb);
    if (n <= 0) return 0;
    sgb::k_sg_hcat<<<sg_blocks(n), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)a_bf16, wa,
                                                                   (const __nv_bfloat16*)b_bf16, wb, rows,
                                                                   (__nv_bfloat16*)out_bf16);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_relu_grad_cols(const float* dY, int ldy, const void* H_bf16, int ldh, int rows, int cols,
                                void* out_bf16, void* stream)
{
    const long long n = (long long)rows * cols;
    if (n <= 0) return 0;
    if (cols > ldy || cols > ldh) { sgb::set_last_error("relu_grad_cols: cols > stride"); return -1; }
    sgb::k_sg_relu_grad_cols<<<sg_blocks(n), 256, 0, (cudaStream_t)stream>>>(dY, ldy, (const __nv_bfloat16*)H_bf16,
                                                                             ldh, rows, cols,
                                                                             (__nv_bfloat16*)out_bf16);
    return sg_status(cudaSuccess);
}

int solar_gpu_sg_transpose_f32(const float* in, int R, int C, float* out, void* stream)
{
    if (R <= 0 || C <= 0) return 0;
    if ((C + 31) / 32 > 65535) { sgb::set_last_error("transpose: C < 2^21"); return -1; }
    sgb::k_sg_transpose_f32<<<dim3((R + 31) / 32, (C + 31) / 32), dim3(32, 8), 0, (cudaStream_t)stream>>>(in, R, C,
                                                                                                        out);
    return sg_status(cudaSuccess);
}

namespace {
int gemm_call(const void* A, const void* B, float* C, void* C_bf16, const float* bias, int M, int N, int K, int relu,
              cudaStream_t st, int stall)
{
    if (!A || !B || (!C && !C_bf16) || ((uintptr_t)A | (uintptr_t)B | (uintptr_t)C | (uintptr_t)C_bf16) % 16) {
        sgb::set_last_error("gemm: null or misaligned (16-byte) pointers");
        return -1;
    }
    int* err = nullptr;
    cudaError_t e = cudaMallocAsync(&err, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) e = sgb::launch_gemm_bf16(A, B, C, C_bf16, bias, M, N, K, relu, err, st, stall);
    int flag = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (err) cudaFreeAsync(err, st);
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
}  // namespace

int solar_gpu_gemm_bf16(const void* A, const void* B, float* C, void* C_bf16, const float* bias, int M, int N,
                        int K, int relu, void* stream)
{
    return gemm_call(A, B, C, C_bf16, bias, M, N, K, relu, (cudaStream_t)stream, 0);
}

int solar_gpu_selftest_bounded_wait(void* stream)
{
    // One 128 x 64 x 64 tile whose operand loads are never issued: the MMA
    // thread's wait for them runs out after about a second, the kernel flags
    // the error, frees its TMEM and exits; the call reports it like any
    // expired wait.
    cudaStream_t st = (cudaStream_t)stream;
    void* buf = nullptr;
    const size_t a_bytes = 128 * 64 * 2, b_bytes = 64 * 64 * 2, c_bytes = 128 * 64 * 4;
    cudaError_t e = cudaMallocAsync(&buf, a_bytes + b_bytes + c_bytes, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(buf, 0, a_bytes + b_bytes + c_bytes, st);
    if (e != cudaSuccess) {
        sgb::set_last_error(cudaGetErrorString(e));
        return -2;
    }
    char* p = static_cast<char*>(buf);
    const int rc = gemm_call(p, p + a_bytes, reinterpret_cast<float*>(p + a_bytes + b_bytes), nullptr, nullptr, 128,
                             64, 64, 0, st, 1);
    cudaFreeAsync(buf, st);
    cudaStreamSynchronize(st);
    return rc;
}

}  // extern "C"
