/*
 * solargpu_b200.h -- C ABI of libsolargpu_b200.so, a B200 (sm_100a) build of
 * SolarGPU's annual DSM irradiance path: DDA viewshed tracer, shadowed
 * direct + Perez diffuse pass, and the inter-reflection pass over CSR or
 * ba-RLE neighbor lists.
 *
 * Reference interfaces replaced (paths relative to the SolarGPU tree):
 *   solar_gpu_uncompressed_gpu_irradiance  <- solar_gpu::uncompressed_gpu_irradiance,
 *                                             include/solar_gpu_api.h:37-42
 *   solar_gpu_compressed_gpu_irradiance    <- solar_gpu::compressed_gpu_irradiance,
 *                                             include/solar_gpu_api.h:49-54
 * The library also exports those two C++ symbols themselves (namespace
 * solar_gpu, identical signatures), so the reference CLI links against it
 * unchanged; they forward to the C functions below.
 *
 * Plain C: pointers, sizes and ints only.  All functions return 0 on success
 * and a negative SOLAR_GPU_ERR_* code otherwise (the reference exits the
 * process on a CUDA error instead); solar_gpu_last_error() describes the
 * last failure of the calling thread.
 */
#ifndef SOLARGPU_B200_H
#define SOLARGPU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SOLAR_GPU_HOURS_PER_YEAR 8760   /* include/pipeline_constants.h:10 */

enum {
    SOLAR_GPU_OK = 0,
    SOLAR_GPU_ERR_ARG = -1,          /* bad argument: null pointer, size, option, index range */
    SOLAR_GPU_ERR_CUDA = -2,         /* a CUDA runtime call or kernel launch failed */
    SOLAR_GPU_ERR_NO_DEVICE = -3,    /* no usable CUDA device */
    SOLAR_GPU_ERR_OOM = -4,          /* device allocation failed */
    SOLAR_GPU_ERR_DEVICE_CHECK = -5  /* a kernel flagged malformed data (e.g. a ba-RLE stream) */
};

/* Neighbor list storage (reference: the two pipeline instances). */
enum { SOLAR_GPU_CSR = 0, SOLAR_GPU_BARLE = 1, SOLAR_GPU_BOTH = 2 };
/* Annual accumulation. */
enum { SOLAR_GPU_ACC_FP64 = 0, SOLAR_GPU_ACC_KAHAN = 1, SOLAR_GPU_ACC_FP32 = 2 };
/* Reflection evaluation. */
enum { SOLAR_GPU_REFL_HOURLY = 0, SOLAR_GPU_REFL_ANNUAL = 1, SOLAR_GPU_REFL_NONE = 2 };

typedef struct solar_gpu_options {
    int neighbor_format;     /* SOLAR_GPU_CSR / SOLAR_GPU_BARLE (SOLAR_GPU_BOTH: trace only) */
    int hour_block;          /* 1 = plain per-hour path; 32..512 = hour-block width (powers of 2); 0 = 128 */
    int accumulation;        /* SOLAR_GPU_ACC_* */
    int reflection;          /* SOLAR_GPU_REFL_HOURLY (reflection per hour, reference semantics),
                                SOLAR_GPU_REFL_ANNUAL (sum over hours first, one sparse product) or
                                SOLAR_GPU_REFL_NONE (each voxel's own direct + diffuse only, FP64
                                sums: the reflected share is 1 - none / hourly) */
    long long chunk_voxels;  /* tracer chunk in voxels (bounds the raw hit buffer); 0 = from free memory */
    int use_graph;           /* capture the hour-block loop in a CUDA graph */
    int time_kernels;        /* record CUDA events around every kernel group (no graph); see
                                solar_gpu_kernel_times */
    int group_size;          /* hour-block reflection kernel: 0 = one warp per voxel, list decoded
                                and weights computed in every block (B 32..256); 1 = weights computed
                                once per run (B 64..512); 2, 4, 8 = that many voxels share one warp,
                                their weighted lists merged once per run into union entries
                                (B 64..512, 32..256, 32..128); 64 = groups of up to 64 voxels
                                whose union rows are staged through shared memory, one CTA
                                per group (B 64..256); 128 = groups of 128 voxels as a dense
                                product on the tcgen05 tensor cores (fp16 slab, weights split
                                into two fp16 parts, FP32 accumulation; B 256) */
} solar_gpu_options;

/* CSR lists, hour block 256, FP64 block sums, hourly reflection, chunk from
   free memory, CUDA graph on, no kernel timing, group size 128 (the
   tensor-core kernel).  The drop-in entry points run with these, format
   aside. */
void solar_gpu_default_options(solar_gpu_options* opt);

/* ---- drop-in entry points (synchronous, host buffers, device 0) -------- */

/* Same arguments as the reference (include/solar_gpu_api.h:15-36); the
   std::vector arguments become pointer + count.  As in the reference only
   the first 8760 entries of each series are used; a count below 8760 is
   SOLAR_GPU_ERR_ARG.  sun_positions is [8760][2] (azimuth_deg, altitude_deg).  wall_z may
   be NULL when num_total_voxels == num_top_voxels.  irradiance_out receives
   num_total_voxels annual sums (Wh/m^2). */
int solar_gpu_uncompressed_gpu_irradiance(
    const float* grid_data, int grid_width, int grid_height,
    int num_total_voxels, int num_top_voxels,
    const int* pixel_parent, const float* wall_z, float max_height,
    const float* sun_positions, int num_sun_positions,
    const float* direct_irradiance, int num_direct,
    const float* diffuse_irradiance, int num_diffuse,
    const float* slopes, const float* aspects, float* irradiance_out);

int solar_gpu_compressed_gpu_irradiance(
    const float* grid_data, int grid_width, int grid_height,
    int num_total_voxels, int num_top_voxels,
    const int* pixel_parent, const float* wall_z, float max_height,
    const float* sun_positions, int num_sun_positions,
    const float* direct_irradiance, int num_direct,
    const float* diffuse_irradiance, int num_diffuse,
    const float* slopes, const float* aspects, float* irradiance_out);

/* ---- context API: persistent device workspace and stream --------------- */

typedef struct solar_gpu_context solar_gpu_context;

int solar_gpu_create(int device, solar_gpu_context** out);
void solar_gpu_destroy(solar_gpu_context* ctx);
/* Frees the context's device buffers (they are grow-only and otherwise kept
   for the next call); the context stays usable.  Results of the last trace
   are no longer available afterwards. */
int solar_gpu_release(solar_gpu_context* ctx);

/* No counterpart in the reference.  Caps the device bytes the context's
   buffers may hold (0: no cap; the default), e.g. for several contexts
   sharing one GPU.  A call that would pass the cap returns SOLAR_GPU_ERR_OOM
   before allocating, and the context stays usable; the tracer's automatic
   chunk is sized within the cap.  memory_held: bytes held now. */
int solar_gpu_set_memory_limit(solar_gpu_context* ctx, long long bytes);
long long solar_gpu_memory_held(solar_gpu_context* ctx);

/* Scene description.  For solar_gpu_run_host the array pointers are host
   pointers; for solar_gpu_run_device and solar_gpu_trace the per-cell and
   per-voxel arrays (grid, pixel_parent, wall_z, slopes, aspects) are device
   pointers while the 8760-entry series (sun_positions, direct, diffuse)
   stay host pointers. */
typedef struct solar_gpu_scene {
    const float* grid;
    int grid_width, grid_height;
    int num_total_voxels, num_top_voxels;
    const int* pixel_parent;
    const float* wall_z;
    float max_height;
    const float* sun_positions;     /* [8760][2] host */
    const float* direct_irradiance; /* [8760] host */
    const float* diffuse_irradiance;/* [8760] host */
    const float* slopes;
    const float* aspects;
} solar_gpu_scene;

/* Host buffers in and out; copies, compute and the read-back are inside. */
int solar_gpu_run_host(solar_gpu_context* ctx, const solar_gpu_options* opt,
                       const solar_gpu_scene* scene, float* irradiance_out);

/* Device-resident inputs and output, enqueued on `stream` (cudaStream_t or
   NULL for the context's own stream).  Returns after the work is enqueued
   except for the small host synchronisations Stage 1 needs to size its
   output buffers. */
int solar_gpu_run_device(solar_gpu_context* ctx, const solar_gpu_options* opt,
                         const solar_gpu_scene* scene, float* irradiance_out_device,
                         void* stream);

/* No counterpart in the reference (it runs one DSM per call).  Runs n
   scenes -- uneven DSM tiles, each with its own site and hourly series -- in
   n contexts (one per tile, same device, device-resident scenes as for
   solar_gpu_run_device): Stage 1 and the once-per-run list builds tile by
   tile, then the hour-block loops of all tiles as parallel branches of one
   CUDA graph, launched once on `stream` (NULL: the first context's stream),
   so that the small tiles' persistent reflection kernels share the SMs.
   opts[i] are tile i's options (e.g. an autotuner's choice for its size)
   and outs[i] receives its annual irradiance.  Needs hour_block > 1 and
   hourly reflection; time_kernels is ignored.  Synchronous. */
int solar_gpu_run_batch(solar_gpu_context* const* ctxs, int n, const solar_gpu_options* opts,
                        const solar_gpu_scene* scenes, float* const* outs, void* stream);

/* Voxelization of a heightmap on the GPU, replacing the reference's host
   code (src/voxelization.cpp:10-97, detect_wall_voxels and
   compute_top_slope_aspect, packed as src/main.cpp:112-127 packs them): one
   top voxel per cell in raster order (pixel_parent i = i, slope and aspect
   from central differences over cells of voxel_size), then the column-drop
   wall voxels in raster order of their cell, from the top of the drop
   downwards (wall_z, slope pi/2, aspect from the open sides).  grid is a
   device array [H][W]; *num_total (host) receives T + walls.  With all
   output pointers NULL only the count is made; otherwise pixel_parent,
   slopes, aspects are device arrays of capacity >= *num_total voxels and
   wall_z of *num_total - T (may be NULL without walls).  Wall counts and
   heights are identical to the reference's; angles may differ from the host
   library's atan2f in the last bits.  Synchronous on `stream`. */
int solar_gpu_voxelize(solar_gpu_context* ctx, const float* grid, int W, int H, float voxel_size,
                       long long* num_total, int* pixel_parent, float* wall_z, float* slopes, float* aspects,
                       long long capacity, void* stream);

/* ---- stage access (parity checks, tools) ------------------------------- */

/* Runs Stage 1 only (device scene), building the lists opt->neighbor_format
   asks for (SOLAR_GPU_BOTH builds both).  Synchronous. */
int solar_gpu_trace(solar_gpu_context* ctx, const solar_gpu_options* opt,
                    const solar_gpu_scene* scene, void* stream);

/* Sizes of the last Stage 1 result. */
int solar_gpu_trace_sizes(solar_gpu_context* ctx, long long* csr_entries, long long* barle_bytes,
                          int* shadow_words, int* active_bins, int* num_voxels);

/* Copies the last Stage 1 result to host buffers (any may be NULL):
   csr_offsets [N+1] int64, csr_ids [csr_entries] (1-based cell ids in
   first-hit direction order, as the reference CSR), barle_offsets [N+1],
   barle_bytes [barle_bytes] (byte-identical to the reference encoder),
   shadow [N][shadow_words] uint32 (bit b of word w set = dense sun bin 32w+b
   is blocked for that voxel). */
/* Stage 1 products handed back to the library (host arrays), e.g. read from
   an on-disk cache: one list format plus the shadow words, laid out as
   solar_gpu_trace_copy returns them. */
typedef struct solar_gpu_lists {
    int format;                  /* SOLAR_GPU_CSR or SOLAR_GPU_BARLE */
    const long long* offsets;    /* [N + 1], offsets[0] = 0, offsets[N] = data_size */
    const void* data;            /* CSR ids (int32, 1-based cells) or ba-RLE bytes */
    long long data_size;         /* ids (CSR) or bytes (ba-RLE) */
    const uint32_t* shadow;      /* [N][shadow_words] */
    int shadow_words;            /* must match the sky bins of the scene's sun positions */
    int active_bins;
} solar_gpu_lists;

/* No counterpart in the reference (it always traces).  Stage 2/3 only: the
   solar and reflection passes over caller-provided neighbor lists and shadow
   words, for re-runs of a traced scene with new hourly irradiance (the sun
   positions, and so the sky bins, must be the ones the lists were traced
   with; shadow_words and active_bins are checked against them).  Scene
   arrays are device pointers as for solar_gpu_run_device; lists are host
   arrays.  opt->neighbor_format is ignored (lists->format is used).
   Malformed lists cannot fault: offsets are checked on the host, ids outside
   the top cells get weight 0, and ba-RLE decoding is bounds-checked
   (SOLAR_GPU_ERR_DEVICE_CHECK). */
int solar_gpu_run_lists(solar_gpu_context* ctx, const solar_gpu_options* opt, const solar_gpu_scene* scene,
                        const solar_gpu_lists* lists, float* irradiance_out, void* stream);

int solar_gpu_trace_copy(solar_gpu_context* ctx, long long* csr_offsets, int* csr_ids,
                         long long* barle_offsets, unsigned char* barle_bytes, uint32_t* shadow);

/* No counterpart in the reference.  Copies the part of the last Stage 1
   result that belongs to voxels [v0, v1) (scenes whose full lists are too
   large to copy): csr_offsets / barle_offsets [v1-v0+1] are the absolute
   offsets offsets[v0..v1]; csr_ids and barle_bytes receive the entries
   between offsets[v0] and offsets[v1] (size them from a first call that
   passes NULL for them); shadow [v1-v0][shadow_words].  Any may be NULL. */
/* After a full run (solar_gpu_run_device / solar_gpu_run_host) of a scene so
   large that Stage 1's raw hit rows exceed a quarter of the device memory,
   the lists are released once the weighted lists are built, to make room for
   the hour loop; solar_gpu_trace (Stage 1 alone) always keeps them. */
int solar_gpu_trace_copy_range(solar_gpu_context* ctx, int v0, int v1, long long* csr_offsets, int* csr_ids,
                               long long* barle_offsets, unsigned char* barle_bytes, uint32_t* shadow);

/* Stage times of the last run, milliseconds, from CUDA events:
   [0] setup (tables, geometry), [1] Stage 1 (trace + lists),
   [2] Stage 2/3 (solar + reflection + accumulation), [3] total.
   Returns the number of values written. */
int solar_gpu_last_timings(solar_gpu_context* ctx, double* ms, int n);

/* Per kernel group device time of the last run with time_kernels set:
   ms[i] and launches[i] for i < SOLAR_GPU_KT_COUNT.  Returns the count. */
enum {
    SOLAR_GPU_KT_SETUP = 0,      /* hour table, voxel geometry, input check */
    SOLAR_GPU_KT_TRACE = 1,      /* DDA tracer */
    SOLAR_GPU_KT_DEDUPE = 2,     /* first-occurrence dedupe */
    SOLAR_GPU_KT_CSR = 3,        /* offsets scan + CSR gather */
    SOLAR_GPU_KT_BARLE = 4,      /* ba-RLE size, scan, write */
    SOLAR_GPU_KT_SOLAR = 5,      /* solar slab / hourly / annual-sum kernels */
    SOLAR_GPU_KT_REFLECT = 6,    /* reflection + accumulation kernels */
    SOLAR_GPU_KT_FINALIZE = 7,
    SOLAR_GPU_KT_GROUP = 8,      /* grouped-reflection build (once per run) */
    SOLAR_GPU_KT_COUNT = 9
};
int solar_gpu_kernel_times(solar_gpu_context* ctx, double* ms, long long* launches, int n);

/* Entries the hour-block reflection streamed per block in the last run
   (weighted or merged union entries; 0 for group_size 0). */
long long solar_gpu_last_reflection_entries(solar_gpu_context* ctx);

/* Slab rows the shared-memory tile kernel (group_size 64) staged per hour
   block in the last run: the sum over groups of their union sizes; 0 for
   other kernels. */
long long solar_gpu_last_staged_rows(solar_gpu_context* ctx);

/* Nonzero reflection weights (receiver, neighbor pairs) of the last run with
   group_size >= 1: each contributes one FMA per daylight hour; 0 otherwise. */
long long solar_gpu_last_weighted_entries(solar_gpu_context* ctx);

/* Number of kernel launches the library issued in the last run. */
long long solar_gpu_last_launch_count(solar_gpu_context* ctx);

/* No counterpart in the reference.  The sun-bin shadow words of the listed
   voxels only (device int32 ids, at most 2^20), traced exactly as the full
   pass traces them; out is device [n][*shadow_words].  Used to spot-check
   and to fall back from the visibility surrogate. */
int solar_gpu_trace_shadow_subset(solar_gpu_context* ctx, const solar_gpu_scene* scene, const int* voxels, int n,
                                  uint32_t* shadow_out, int* shadow_words, void* stream);

/* ---- tensor-core GEMM (sky-bin visibility surrogate) ------------------- */

/* No counterpart in the reference.  C[M][N] = A[M][K] x B[N][K]^T (+ bias[N],
   ReLU if relu != 0) on the tcgen05 tensor cores: A, B bf16 row-major (K
   contiguous), f32 accumulation in TMEM, output f32 (C) and/or bf16 (C_bf16),
   row-major; device pointers, 16-byte aligned.  M a multiple of 128, N of 64,
   K of 64.  Synchronous on `stream`. */
int solar_gpu_gemm_bf16(const void* A, const void* B, float* C, void* C_bf16, const float* bias, int M, int N,
                        int K, int relu, void* stream);

/* No counterpart in the reference.  Self-test of the device-side bounded
   waits: one GEMM tile whose operand loads are withheld, so that its MMA
   thread's wait for them runs out (about 1 s); the kernel records the error
   and exits normally.  Returns what any expired wait returns,
   SOLAR_GPU_ERR_DEVICE_CHECK with "a bounded wait expired" as the last
   error; the device stays usable. */
int solar_gpu_selftest_bounded_wait(void* stream);

/* Surrogate training/inference kernels (device pointers, bf16 = 2-byte
   bfloat16, row-major).  features: per voxel the 64 x 64 heights around its
   pixel relative to its base height / 50 m (clipped to +-2) and its normal,
   zero-padded to feat (>= 4099) columns.  labels: the first `active` shadow
   bits of each voxel as 0/1 floats over outw columns.  bce: mean binary
   cross-entropy with logits over the first `active` columns (adds to *loss),
   dZ = (sigmoid(Z) - Y) / (M active) as bf16.  relu_grad: dX = dY (H > 0).
   transpose: out[C][R] = in[R][C].  colsum: out[c] = sum_r in[r][c] (out
   overwritten).  adam:
   one Adam step on FP32 parameters (bias-corrected, step >= 1), optional
   bf16 copy. */
int solar_gpu_sg_features(const float* grid, int W, int H, int T, const int* pixel_parent, const float* wall_z,
                          const float* slopes, const float* aspects, const int* voxels, int M, int feat,
                          void* out_bf16, void* stream);
int solar_gpu_sg_labels(const uint32_t* shadow, int words32, const int* voxels, int M, int active, int outw,
                        float* y, void* stream);
int solar_gpu_sg_bce(const float* Z, const float* Y, int M, int outw, int active, void* dZ_bf16, float* loss,
                     void* stream);
int solar_gpu_sg_relu_grad(const float* dY, const void* H_bf16, long long n, void* dX_bf16, void* stream);
int solar_gpu_sg_transpose(const void* in_bf16, int R, int C, void* out_bf16, void* stream);
int solar_gpu_sg_colsum(const void* in_bf16, int R, int C, float* out, void* stream);
int solar_gpu_sg_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                      float eps, int step, void* p_bf16, void* stream);

/* Convolutional front end of the surrogate (4 x 4 kernels, stride 2,
   padding 1, NHWC bf16 activations).  coarse: out[cy][cx] = max of grid over
   the 8 x 8 cells of context cell (cx, cy), ceil(H/8) x ceil(W/8).  image:
   per voxel a [64][64][2] image, channel 0 the heights of the 64 x 64 cells
   around its pixel, channel 1 the context maxima of the 64 x 64 context cells
   around its context cell, both relative to its base height / 50 m (clipped
   to +-2), and nrm [M][64] its normal zero-padded.  im2col: cols[(b Ho + oy)
   Wo + ox][(ky 4 + kx) Cin + c] = X[b][2oy-1+ky][2ox-1+kx][c] (0 outside),
   zero columns up to Kp.  col2im_relu: the gradient of X through im2col,
   times (X > 0), as bf16.  hcat: rows of a and b side by side.
   relu_grad_cols: out[r][c] = dY[r][c] (H[r][c] > 0) for c < cols, strided
   inputs.  transpose_f32: out[C][R] = in[R][C]. */
int solar_gpu_sg_coarse(const float* grid, int W, int H, float* out, void* stream);
int solar_gpu_sg_image(const float* grid, const float* coarse, int W, int H, int T, const int* pixel_parent,
                       const float* wall_z, const float* slopes, const float* aspects, const int* voxels, int M,
                       void* img_bf16, void* nrm_bf16, void* stream);
int solar_gpu_sg_im2col(const void* X_bf16, int B, int Hi, int Wi, int Cin, int Kp, void* cols_bf16, void* stream);
int solar_gpu_sg_col2im_relu(const float* dcols, const void* X_bf16, int B, int Hi, int Wi, int Cin, int Kp,
                             void* g_bf16, void* stream);
int solar_gpu_sg_hcat(const void* a_bf16, int wa, const void* b_bf16, int wb, int rows, void* out_bf16, void* stream);
int solar_gpu_sg_relu_grad_cols(const float* dY, int ldy, const void* H_bf16, int ldh, int rows, int cols,
                                void* out_bf16, void* stream);
int solar_gpu_sg_transpose_f32(const float* in, int R, int C, float* out, void* stream);

/* ---- encoding without device allocation -------------------------------- */

/* No counterpart in the reference.  ba-RLE-encodes num_lists CSR neighbor
   lists (device csr_offsets [num_lists+1] int64 from 0, device csr_ids
   int32) into device barle_offsets [num_lists+1] and device barle_bytes
   (capacity barle_capacity bytes); *barle_total (host) receives the byte
   count, also when the capacity is too small (barle_offsets is filled then,
   barle_bytes is left untouched).  Each list must hold distinct ids >= 1, as
   the tracer's lists do; other lists are rejected (SOLAR_GPU_ERR_ARG).
   Bytes are identical to the library's own ba-RLE lists and to the reference
   encoder.  For callers that may not allocate device memory (their GPU memory
   is owned by a host framework's pool, or cudaMalloc/cudaFree stalls are not
   acceptable): it allocates nothing; its scratch is one fixed static device
   array of about 10.6 MB per device, so num_lists <= 1024 and each list
   <= 2592 ids.  Calls share that array: calls that overlap on the GPU race
   and must be serialised.  The first call on a device (and the first after
   the device's context was reset) looks up the array's address; make it
   before any stream capture.  Runs on `stream` (NULL = the
   legacy default stream) and synchronises it. */
int solar_gpu_barle_encode_noalloc(const long long* csr_offsets, const int* csr_ids, int num_lists,
                                   long long* barle_offsets, unsigned char* barle_bytes,
                                   long long barle_capacity, long long* barle_total, void* stream);

/* Message of the calling thread's last failure ("" if none). */
const char* solar_gpu_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SOLARGPU_B200_H */
