// Internal types and launchers shared by the translation units of
// libsolargpu_b200.so.  Nothing here is part of the public C ABI
// (include/solargpu_b200.h).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace sgb {

constexpr int kHoursPerYear = 8760;   // include/pipeline_constants.h:10 of the reference
constexpr int kMaxDirs = 72 * 36;     // 5 deg x 5 deg bins over both hemispheres
constexpr int kRawGroup = 16;         // directions buffered per tracer store

// Device error flag bits (set by kernels, read back by the host).
enum DeviceError : int {
    kErrBarleStream = 1,   // a ba-RLE stream ran past its byte range or had a bad width code
    kErrHashFull = 2,      // a dedupe hash probe exceeded its bound
    kErrListCapacity = 4,  // a neighbor list exceeded the buffer capacity
    kErrWaitTimeout = 8,   // a bounded wait on a shared-memory barrier expired
    kErrTraceBounds = 16,  // a ray passed the tracer's border (its clamped index ended it)
};

// One traced direction; host-computed exactly as the reference computes Cdir
// (include/cuda/viewshed_stage.cuh:64-80), plus the per-direction constants of
// the DDA (viewshed_kernels.cu:32-40), which are direction-only.
struct DirEntry {
    float cx, cy, cz;
    float ax, ay;      // fmaxf(fabsf(c), 1e-8f)
    float dX, dY;      // 1.0f / ax, 1.0f / ay (IEEE)
    int meta;          // bits 0..15: dense sun bin + 1 (0 = none); bit 16: upper hemisphere;
                       // bits 17..26: early-exit table of an upper direction (cone.cu)
};

// The integer cone of one early-exit table (cone.cu): directions of quadrant
// (sx, sy) whose unsigned step vector (1/dX, 1/dY) lies between the
// primitive vectors a = (ax, ay) and b = (bx, by), det(a, b) = 1.
struct ConeSpec {
    int sx, sy;
    int ax, ay, bx, by;
};
constexpr int kConeOrder = 8;        // cone vectors have components <= 8
constexpr int kMaxConeTables = 1024; // 10 bits of DirEntry::meta

// Per daylight hour, FP32 values of the FP64-evaluated solar geometry.
//   cos_aoi(v) = dot(n_v, s)
//   direct     = (cos_aoi > 0 && dense >= 0 && !shadow) ? dni_eff * cos_aoi : 0
//   diffuse    = max(0, c0 * (1 + cos s) + c1 * max(0, cos_aoi) + c2 * sin s)
struct HourEntry {
    float sx, sy, sz;
    float dni_eff;
    float c0, c1, c2;
    int dense;         // sun bin (dense index) or -1; padding entries have dense = -1 and zeros
};

struct DevScene {
    const float* grid;        // [T]
    const float* gpad;        // [H + 2][W + 2]: grid inside a border of +inf (the tracer's copy)
    const int* pix_parent;    // [N]
    const float* wall_z;      // [N - T] or nullptr
    const float* slopes;      // [N]
    const float* aspects;     // [N]
    int W, H, N, T;
    float maxz;
    // [tables][H + 2][W + 2] early-exit bounds of upper rays (cone.cu), or
    // nullptr (no early exit: the reference's range test alone)
    const float* cone;
    size_t cone_stride;
};

// Per-voxel geometry derived once per call.
//   geo_n[v] = (nx, ny, nz, sin slope) with n as in reflection_kernels.cu:59-64
//   geo_p[v] = (gx, gy, z, 0)
struct DevGeom {
    float4* geo_n;
    float4* geo_p;
};

// Sets the calling thread's message returned by solar_gpu_last_error().
void set_last_error(const char* msg);

// ------------------------------------------------------------------ launchers

// tracer (trace.cu)
// Stage 1 kernels address rows of the raw hit buffer of a chunk of voxels
// [voxel_offset, voxel_offset + chunk_count).  Row lv holds chunk voxel
// perm[lv] when a permutation is given (counts, sizes indexed by chunk
// voxel), else chunk voxel lv; kernels that iterate voxels take the inverse.
// gpad [(H + 2) * (W + 2)] = grid inside a one-cell border of +inf.
cudaError_t launch_pad_grid(const float* grid, int W, int H, float* gpad, cudaStream_t st);
// Early-exit tables (cone.cu): n_specs bordered tables of `stride` floats in
// tabs; tmp holds as many (scratch).
cudaError_t launch_cone_tables(const float* grid, int W, int H, float maxz, const ConeSpec* specs, int n_specs,
                               float* tabs, float* tmp, size_t stride, cudaStream_t st);
int cone_window_radius(int W, int H);
// s.gpad must be set (launch_pad_grid); s.cone may be nullptr.
cudaError_t launch_trace(const DevScene& s, const DirEntry* dirs, int D, int words32,
                         int voxel_offset, int chunk_count, int* raw, uint32_t* shadow,
                         const int* perm, int* err, cudaStream_t st);
// ovf: chunk_count + 1 ints of scratch (rows the small-table pass hands on).
cudaError_t launch_dedupe(int chunk_count, int D, int* raw, int* counts, int* err, const int* perm, int* ovf,
                          cudaStream_t st);
cudaError_t launch_invert(const int* perm, int n, int* inv, cudaStream_t st);
// perm = the chunk voxels [v0, v0 + n) (as v - v0) in visiting order;
// flag [N] and pos [N + 1] scratch.
cudaError_t launch_chunk_order(const int* order, int N, int v0, int n, int* flag, long long* pos,
                               long long* scan_tmp, int* perm, cudaStream_t st);
cudaError_t launch_scan_counts(const int* counts, int n, long long base, long long* offsets,
                               long long* block_sums, int* block_tmp, cudaStream_t st);
size_t scan_scratch_elems(int n);
cudaError_t launch_gather_csr(int chunk_count, int D, const int* raw, const long long* offsets,
                              int* csr_ids, const int* inv, cudaStream_t st);

// ba-RLE encoder (barle.cu)
cudaError_t launch_barle_size(int chunk_count, int D, int* raw, const int* counts,
                              int* sizes, int* err, cudaStream_t st);
cudaError_t launch_barle_size(int chunk_count, int D, int* raw, const int* counts, int* sizes, int* err,
                              const int* perm, cudaStream_t st);
cudaError_t launch_barle_write(int chunk_count, int D, const int* raw, const int* counts,
                               const long long* offsets, unsigned char* out, int* err, const int* inv,
                               cudaStream_t st);
cudaError_t launch_barle_write(int chunk_count, int D, const int* raw, const int* counts,
                               const long long* offsets, unsigned char* out, int* err,
                               cudaStream_t st);

// solar (solar.cu)
cudaError_t launch_hour_table(const float* nudged, const float* dni, const float* dhi,
                              const int* sun_dense, const int* hour_index, int n_hours,
                              int n_padded, HourEntry* table, cudaStream_t st);
cudaError_t launch_voxel_geom(const DevScene& s, DevGeom g, cudaStream_t st);
cudaError_t launch_solar_slab(const DevGeom& g, int T, const uint32_t* shadow, int words32,
                              const HourEntry* table, int j0, int B, float* slab, cudaStream_t st);
cudaError_t launch_solar_hour(const DevGeom& g, int N, const uint32_t* shadow, int words32,
                              const HourEntry* table, int j, float* hourly, cudaStream_t st);
cudaError_t launch_solar_sum(const DevGeom& g, int N, const uint32_t* shadow, int words32,
                             const HourEntry* table, int n_hours, double* sums, cudaStream_t st);

// reflection (reflect.cu)
struct NeighborLists {
    int format;                  // 0 = CSR, 1 = ba-RLE
    const long long* offsets;    // [N + 1] (ids for CSR, bytes for ba-RLE)
    const int* ids;              // CSR ids, 1-based
    const unsigned char* bytes;  // ba-RLE stream
};
struct Accum {
    int mode;        // 0 = FP64 sums, 1 = Kahan-compensated FP32, 2 = plain FP32
    double* f64;     // [N]
    float* f32;      // [N] (sum) for modes 1, 2
    float* comp;     // [N] Kahan compensation for mode 1
};
cudaError_t launch_reflect_block(const DevGeom& g, int N, int T, const uint32_t* shadow,
                                 int words32, const HourEntry* table, int j0, int B,
                                 const float* slab, const NeighborLists& nl, const Accum& acc,
                                 const int* order, int* err, cudaStream_t st);
// Visiting order of the reflection pass (32 x 32 cell tiles, Morton inside).
long long order_positions(int W, int H);
cudaError_t launch_voxel_order(const int* pix_parent, int N, int T, int W, int H, int* counts,
                               int* first_wall, long long* cursor, long long* scan_tmp, int* order,
                               cudaStream_t st);
cudaError_t launch_reflect_hour(const DevGeom& g, int N, int T, const float* hourly,
                                const NeighborLists& nl, const Accum& acc, int* err,
                                cudaStream_t st);
cudaError_t launch_reflect_annual(const DevGeom& g, int N, int T, const double* sums,
                                  const NeighborLists& nl, double* out, int* err,
                                  cudaStream_t st);
cudaError_t launch_finalize(const Accum& acc, int N, float* out, cudaStream_t st);

// grouped reflection (group.cu)
struct GroupLists {
    int V;                       // voxels per group (1, 2, 4 or 8)
    const long long* offsets;    // [G + 1] union entries per group
    const int* cells;            // [E] neighbor cell of each union entry, ascending per group
    const float* weights;        // [E][V] weight of that cell for each voxel of the group
};
int group_count(int N, int V);
// Weighted lists in visiting order: pass 0 counts nonzero weights per
// position, pass 1 writes (cell, w) at woff[p].
cudaError_t launch_weight_lists(int pass, const DevGeom& g, int N, int T, const NeighborLists& nl,
                                const int* order, int* counts, const long long* woff, int* cells,
                                float* wts, int* err, cudaStream_t st);
// Merges the weighted lists of V consecutive positions into union entries.
cudaError_t launch_group_merge(int pass, int V, int N, const long long* woff, const int* wcell,
                               const float* wts, int* counts, const long long* goff, int* cell, float* w,
                               cudaStream_t st);
// slab: [N][B] rows of every voxel (neighbor values and each voxel's own term).
cudaError_t launch_reflect_group(int N, int B, const float* slab, const GroupLists& gl, const int* order,
                                 const Accum& acc, cudaStream_t st);
cudaError_t launch_finalize_f64(const double* in, int N, float* out, cudaStream_t st);

// tiled reflection (tile.cu)
struct TileLists {
    int G;                         // voxels per group at most (64 = 16 quads)
    int NG;                        // groups
    const int* start;              // [NG + 1] first visiting position of each group
    const int* unions;             // [NG] union rows of each group
    const long long* woff;         // [N + 1] entry offsets per visiting position
    const int* cells;              // union cells of group q at woff[start[q]] (descending)
    int R;                         // union rows per chunk (rows one shared-memory stage holds)
    const long long* gbase;        // [NG + 1] first merged entry of each group
    const long long* tbase;        // [NG + 1] first chunk table of each group
    const int* table;              // [chunks][20] per chunk: quad offsets, block start, padded count
    const unsigned short* erow;    // [Em] row of each merged entry inside its chunk
    const float4* ew;              // [Em] the quad's 4 weights for that row (0 where a voxel lacks it)
};
// Group boundaries: flag/pos scratch [N] / [N + 1]; start [N + 1].
cudaError_t launch_tile_groups(int N, int G, const long long* woff, int* flag, long long* pos,
                               long long* scan_tmp, int* start, cudaStream_t st);
// Union rows per chunk of the tile kernel for hour block B (0 if not built).
int tile_rows_per_stage(int B);
// Per group: the union of its cells (descending) written over the start of
// the group's cells, and each entry's slot in it; rows_total = sum of the
// unions (slab rows staged per hour block).
cudaError_t launch_tile_build(int NG, const int* start, const long long* woff, int* cells, unsigned short* slots,
                              int* unions, long long* rows_total, int* err, cudaStream_t st);
// Merges the slot lists of each quad and lays them out chunk by chunk:
// pass 0 counts (gcnt: padded merged entries, gnch: chunks, per group),
// pass 1 writes at gbase / tbase (scans of gcnt / gnch); ew must be zero.
cudaError_t launch_tile_layout(int pass, int NG, int R, const int* start, const int* unions, const long long* woff,
                               const unsigned short* slots, const float* wts, int* gcnt, int* gnch,
                               const long long* gbase, const long long* tbase, int* table,
                               unsigned short* erow, float4* ew, cudaStream_t st);
// BF16 tensor-core GEMM (surrogate.cu): C = A x B^T (+bias, ReLU); M a
// multiple of 128, N and K of 64; C and/or Cb (bf16 copy) may be null.
// stall != 0 withholds the operand loads (self-test of the bounded waits).
cudaError_t launch_gemm_bf16(const void* A, const void* B, float* C, void* Cb, const float* bias, int M, int N,
                             int K, int relu, int* err, cudaStream_t st, int stall = 0);
// slab: [N][B] rows of every voxel (neighbor values and each voxel's own term).
cudaError_t launch_reflect_tile(int B, const float* slab, const TileLists& tl, const int* order, const Accum& acc,
                                int* err, cudaStream_t st);

// tensor-core reflection (mma.cu): groups of 128 visiting positions, hour
// blocks of 256, fp16 slab of the top cells.
struct MmaLists {
    int N;
    const int* order;          // [N] voxel at each visiting position
    const long long* woff;     // [N + 1] weighted-list offsets; the union of group q starts at woff[128 q]
    const int* cells;          // union cells per group (written over the weighted cells)
    const int* unions;         // [groups] union size
    const long long* cbase;    // [groups + 1] first chunk of each group
    const long long* coff;     // [chunks + 1] first entry of each chunk
    const void* ent;           // [entries] 8 bytes: W-tile byte offset, fp16 hi, fp16 lo
    const float* scale;        // [N] per visiting position: 2^e undoing the weight scaling
    const int* sched;          // [mma_grid + 1 + groups]: per-CTA offsets, then the groups of each CTA
};
constexpr int kMmaGroup = 128;
constexpr int kMmaHours = 256;
constexpr int kMmaChunk = 64;
int mma_group_count(int N);
// CTAs of the hour-block kernel for N voxels (the schedule is made for them).
int mma_grid(int N);
// Balanced static schedule of the groups over mma_grid(N) CTAs: in visiting
// order, each group goes to the CTA with the least work so far (its chunks
// plus a per-group cost), as a dynamic scheduler would hand them out, so
// neighbouring groups still run at the same time.  cbase [groups + 1] on the
// host; sched receives mma_grid + 1 offsets followed by the groups.
void mma_schedule(int N, const long long* cbase, int* sched);
// Union of each group (cells rewritten in place, slots per entry, union size
// and chunk count per group); *over counts groups above the union cap.
// retry: groups + 1 ints of scratch (groups the small first pass hands on).
cudaError_t launch_mma_union(int N, const long long* woff, int* cells, unsigned short* slots, int* unions, int* nch,
                             int* over, int* retry, cudaStream_t st);
// pass 0: entries per chunk (ccnt at cbase) and the per-position scale;
// pass 1: the entries at coff (the scan of ccnt).
cudaError_t launch_mma_layout(int pass, int N, const long long* woff, const unsigned short* slots, const float* wts,
                              const int* nch, const long long* cbase, int* ccnt, const long long* coff, uint2* ent,
                              float* scale, cudaStream_t st);
cudaError_t launch_solar_slab16(const DevGeom& g, int T, const uint32_t* shadow, int words32, const HourEntry* table,
                                int j0, void* slab16, cudaStream_t st);
cudaError_t launch_reflect_mma(const void* slab16, const MmaLists& ml, const DevGeom& g, const uint32_t* shadow,
                               int words32, const HourEntry* table, int j0, const Accum& acc, int* err,
                               cudaStream_t st);

// voxelization (voxel.cu): wall voxels per cell, then the packed arrays
// (tops [0, T), walls after them at T + off[cell] + v).
cudaError_t launch_vox_count(const float* grid, int W, int H, float voxel_size, int* counts, cudaStream_t st);
cudaError_t launch_vox_write(const float* grid, int W, int H, float voxel_size, float scale, const long long* off,
                             int* parent, float* wall_z, float* slopes, float* aspects, cudaStream_t st);

}  // namespace sgb
