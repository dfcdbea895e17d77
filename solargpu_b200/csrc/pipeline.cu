// Host orchestration and the C ABI (include/solargpu_b200.h).
//
// Replaces the reference pipeline hosts (src/cuda/gpu_irradiance_uncompressed.cu,
// src/cuda/gpu_irradiance_compressed.cu) and the out-of-core viewshed driver
// (include/cuda/viewshed_stage.cuh:37-125):
//   * all state lives in a context (no __constant__ globals), so calls are
//     reentrant per context and run on the caller's stream;
//   * device buffers are grow-only and reused across calls;
//   * Stage 1 runs in voxel chunks bounded by a memory budget, and builds the
//     CSR and/or ba-RLE lists on the device (no host round trip of the raw
//     hit buffer, no host encoder);
//   * errors come back as return codes, never exit().
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "solargpu_b200.h"
#include "sgb_internal.cuh"
#include "sky.h"

using namespace sgb;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what, int line)
{
    const int code = (e == cudaErrorMemoryAllocation) ? SOLAR_GPU_ERR_OOM
                   : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? SOLAR_GPU_ERR_NO_DEVICE
                   : SOLAR_GPU_ERR_CUDA;
    cudaGetLastError();   // clear a sticky launch error so the context stays usable
    return fail(code, "%s failed (pipeline.cu:%d): %s", what, line, cudaGetErrorString(e));
}

#define CK(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return cuda_fail(e_, #call, __LINE__); } while (0)
#define RK(call) do { int r_ = (call); if (r_ != SOLAR_GPU_OK) return r_; } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

template <typename T> T* as(DevBuf& b) { return static_cast<T*>(b.p); }


__global__ void k_check_ids(const int* __restrict__ ids, int n, int N, int* __restrict__ bad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && (unsigned)ids[i] >= (unsigned)N) atomicOr(bad, 1);
}

__global__ void k_validate_parents(const int* __restrict__ pp, int N, int T, int* __restrict__ bad)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= N) return;
    const int p = pp[v];
    // Layout contract of src/main.cpp:112-127: tops are cells in raster order.
    if ((v < T && p != v) || p < 0 || p >= T) atomicOr(bad, 1);
}

}  // namespace

namespace sgb {
// Lets other translation units report through solar_gpu_last_error().
void set_last_error(const char* msg) { g_err = msg; }
}  // namespace sgb

// Everything the hour-block loop of one run needs, built by stage23; kept in
// the context when the loop is enqueued later (solar_gpu_run_batch).
struct HourLoop {
    bool mma = false, tiled = false;
    int group_size = 0, N = 0, T = 0, Hd = 0, B = 0, slab_rows = 0, words32 = 0;
    sgb::DevGeom g{};
    const uint32_t* sh = nullptr;
    const sgb::HourEntry* tab = nullptr;
    float* slab = nullptr;
    void* slab16 = nullptr;
    sgb::MmaLists ml{};
    sgb::TileLists tl{};
    sgb::GroupLists gl{};
    sgb::NeighborLists nl{};
    sgb::Accum acc{};
    int* err = nullptr;
    const int* order = nullptr;
    float* out = nullptr;
};

struct solar_gpu_context {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaEvent_t ev[4] = {};
    DevBuf dirs, nudged, dni, dhi, sun_dense, hour_index, table, geo_n, geo_p, shadow, raw,
        counts, csr_off, csr_ids, barle_off, barle_sizes, barle_bytes, scan_tmp, slab, hourly,
        acc_f64, acc_f32, acc_comp, sums, out_f64, err, in_grid, in_pp, in_wz, in_slopes,
        in_aspects, out_f32, order, order_cnt, order_cur, order_tmp, grp_cnt, grp_off, grp_tmp,
        grp_cell, grp_w, w_cnt, w_off, w_tmp, w_cell, w_val, order_first, order_inv, tile_flag, tile_pos,
        tile_start, tile_union, tile_slot, tile_rows, tile_gcnt, tile_gnch, tile_gbase, tile_tbase, tile_table,
        tile_erow, tile_ew, chunk_perm, chunk_flag, chunk_pos, chunk_tmp, mma_union, mma_nch, mma_cbase,
        mma_ccnt, mma_coff, mma_ent, mma_scale, mma_over, slab16, dd_ovf, vox_cnt, vox_off, vox_tmp, gpad, mma_sched, mma_retry, cone, cone_tmp, cone_specs;
    int* h_scalars = nullptr;   // pinned host scratch for small read-backs
    long long mem_limit = 0;    // device bytes the buffers may hold (0: no limit)
    size_t dev_total = 0;       // device memory size, read once at creation
    // last Stage 1 result
    int N = 0, T = 0, words32 = 0, active = 0;
    long long csr_total = 0, barle_total = 0;
    bool have_csr = false, have_barle = false;
    double timings[4] = {0, 0, 0, 0};
    long long launches = 0;
    long long group_entries = 0;
    long long staged_rows = 0;   // slab rows the tile kernel stages per hour block
    long long weighted_entries = 0;   // nonzero reflection weights of the last run
    bool timed = false;
    // a run released buffers to make room (scenes of tens of millions of
    // voxels): the next run starts by releasing the Stage 2/3 buffers too
    bool squeezed = false;
    // solar_gpu_run_batch: stage23 stops before the hour loop and leaves it here
    bool defer_hours = false;
    // solar_gpu_run_batch: the early-exit tables of every tile are built in
    // one buffer (the first context's), tile after tile on one stream
    DevBuf* cone_shared = nullptr;
    HourLoop hours;
    // per kernel-group event log (time_kernels)
    bool ktime = false;
    std::vector<cudaEvent_t> kt_pool;
    std::vector<int> kt_ids;   // group of event pair i
    int kt_used = 0;
    cudaStream_t kt_stream = nullptr;
};

static constexpr int kNumBufs = 84;
extern "C" {
static void all_bufs(solar_gpu_context* c, DevBuf** out);   // defined with the exports below
}

namespace {

// Device bytes held by the context's buffers.
size_t held_bytes(solar_gpu_context* c)
{
    DevBuf* bufs[kNumBufs];
    all_bufs(c, bufs);
    size_t h = 0;
    for (DevBuf* b : bufs) h += b->cap;
    return h;
}

// Refuses (SOLAR_GPU_ERR_OOM, nothing allocated) when holding `extra` more
// bytes would pass the context's memory limit.
int check_limit(solar_gpu_context* c, size_t extra)
{
    if (c->mem_limit <= 0) return SOLAR_GPU_OK;
    const size_t held = held_bytes(c);
    if (held + extra > (size_t)c->mem_limit)
        return fail(SOLAR_GPU_ERR_OOM, "device memory limit of %lld bytes: %zu held, %zu more needed", c->mem_limit,
                    held, extra);
    return SOLAR_GPU_OK;
}

int ensure(solar_gpu_context* c, DevBuf& b, size_t bytes)
{
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return SOLAR_GPU_OK;
    const size_t cap = (bytes + 255) & ~(size_t)255;
    RK(check_limit(c, cap - b.cap));
    if (b.p) CK(cudaFree(b.p));
    b.p = nullptr;
    b.cap = 0;
    CK(cudaMalloc(&b.p, cap));
    b.cap = cap;
    return SOLAR_GPU_OK;
}

// Grows `b` to at least `bytes`, keeping the first `used` bytes (old and new
// buffers are both held during the copy).
int ensure_keep(solar_gpu_context* c, DevBuf& b, size_t bytes, size_t used, cudaStream_t st)
{
    if (b.cap >= bytes) return SOLAR_GPU_OK;
    void* np = nullptr;
    const size_t cap = ((bytes + bytes / 8) + 255) & ~(size_t)255;
    RK(check_limit(c, cap));
    CK(cudaMalloc(&np, cap));
    if (used && b.p) CK(cudaMemcpyAsync(np, b.p, used, cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    if (b.p) CK(cudaFree(b.p));
    b.p = np;
    b.cap = cap;
    return SOLAR_GPU_OK;
}

int read_ll(solar_gpu_context* c, const long long* dev, long long* out, cudaStream_t st)
{
    CK(cudaMemcpyAsync(c->h_scalars, dev, sizeof(long long), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::memcpy(out, c->h_scalars, sizeof(long long));
    return SOLAR_GPU_OK;
}

// Event pair around a kernel group when time_kernels is set.
struct KScope {
    solar_gpu_context* c;
    int idx = -1;
    KScope(solar_gpu_context* ctx, int group) : c(ctx)
    {
        if (!c->ktime) return;
        if ((size_t)(2 * c->kt_used + 2) > c->kt_pool.size()) {
            for (int i = 0; i < 256; ++i) {
                cudaEvent_t e;
                if (cudaEventCreate(&e) != cudaSuccess) return;
                c->kt_pool.push_back(e);
            }
        }
        idx = c->kt_used++;
        c->kt_ids.push_back(group);
        cudaEventRecord(c->kt_pool[2 * idx], c->kt_stream);
    }
    ~KScope()
    {
        if (idx >= 0) cudaEventRecord(c->kt_pool[2 * idx + 1], c->kt_stream);
    }
};

int check_scene(const solar_gpu_scene* s)
{
    if (!s) return fail(SOLAR_GPU_ERR_ARG, "scene is NULL");
    if (s->grid_width <= 0 || s->grid_height <= 0)
        return fail(SOLAR_GPU_ERR_ARG, "grid size %dx%d", s->grid_width, s->grid_height);
    if ((long long)s->grid_width * s->grid_height != (long long)s->num_top_voxels)
        return fail(SOLAR_GPU_ERR_ARG, "num_top_voxels %d != grid_width * grid_height", s->num_top_voxels);
    // the tracer's bordered copy of the grid is indexed with int
    if ((long long)(s->grid_width + 2) * (s->grid_height + 2) > 0x7FFFFFFFLL)
        return fail(SOLAR_GPU_ERR_ARG, "grid %dx%d: (width + 2) * (height + 2) must stay below 2^31",
                    s->grid_width, s->grid_height);
    if (s->num_total_voxels < s->num_top_voxels)
        return fail(SOLAR_GPU_ERR_ARG, "num_total_voxels %d < num_top_voxels", s->num_total_voxels);
    if (!s->grid || !s->pixel_parent || !s->slopes || !s->aspects)
        return fail(SOLAR_GPU_ERR_ARG, "a voxel array pointer is NULL");
    if (s->num_total_voxels > s->num_top_voxels && !s->wall_z)
        return fail(SOLAR_GPU_ERR_ARG, "wall_z is NULL but there are %d wall voxels",
                    s->num_total_voxels - s->num_top_voxels);
    if (!s->sun_positions || !s->direct_irradiance || !s->diffuse_irradiance)
        return fail(SOLAR_GPU_ERR_ARG, "an hourly series pointer is NULL");
    return SOLAR_GPU_OK;
}

int check_options(const solar_gpu_options* o, bool trace_only)
{
    if (!o) return fail(SOLAR_GPU_ERR_ARG, "options is NULL");
    if (o->neighbor_format < 0 || o->neighbor_format > 2 || (!trace_only && o->neighbor_format == 2))
        return fail(SOLAR_GPU_ERR_ARG, "neighbor_format %d", o->neighbor_format);
    const int B = o->hour_block;
    if (!(B == 0 || B == 1 || B == 32 || B == 64 || B == 128 || B == 256 || B == 512))
        return fail(SOLAR_GPU_ERR_ARG, "hour_block %d (1, 32, 64, 128, 256 or 512)", B);
    if (o->accumulation < 0 || o->accumulation > 2) return fail(SOLAR_GPU_ERR_ARG, "accumulation %d", o->accumulation);
    if (o->reflection < 0 || o->reflection > 2) return fail(SOLAR_GPU_ERR_ARG, "reflection %d", o->reflection);
    if (o->chunk_voxels < 0) return fail(SOLAR_GPU_ERR_ARG, "chunk_voxels %lld", o->chunk_voxels);
    // hour-block widths each reflection kernel is built for
    const int V = o->group_size;
    const int Bq = B == 0 ? 128 : B;
    bool ok = false;
    switch (V) {
    case 0: case 4: ok = Bq >= 32 && Bq <= 256; break;
    case 8: ok = Bq >= 32 && Bq <= 128; break;
    case 1: case 2: ok = Bq >= 64 && Bq <= 512; break;
    case 64: ok = Bq >= 64 && Bq <= 256; break;
    case 128: ok = Bq == kMmaHours; break;
    default: return fail(SOLAR_GPU_ERR_ARG, "group_size %d (0, 1, 2, 4, 8, 64 or 128)", V);
    }
    if (Bq > 1 && !ok)
        return fail(SOLAR_GPU_ERR_ARG, "hour_block %d is not built for group_size %d", Bq, V);
    return SOLAR_GPU_OK;
}

DevScene dev_scene(const solar_gpu_scene* s)
{
    DevScene d;
    d.grid = s->grid;
    d.gpad = nullptr;
    d.pix_parent = s->pixel_parent;
    d.wall_z = s->wall_z;
    d.slopes = s->slopes;
    d.aspects = s->aspects;
    d.W = s->grid_width;
    d.H = s->grid_height;
    d.N = s->num_total_voxels;
    d.T = s->num_top_voxels;
    d.maxz = s->max_height;
    d.cone = nullptr;
    d.cone_stride = 0;
    return d;
}

// Tables, geometry and input validation.
int prepare(solar_gpu_context* c, const solar_gpu_scene* s, SkyTables& sky, cudaStream_t st)
{
    sky = make_sky_tables(s->sun_positions);
    const int D = (int)sky.dirs.size();
    const int Hd = (int)sky.hour_index.size();
    const int n_padded = ((Hd + 511) / 512) * 512 + 512;   // room for the widest hour block
    RK(ensure(c, c->dirs, sizeof(DirEntry) * D));
    RK(ensure(c, c->nudged, sizeof(float) * 2 * kHoursPerYear));
    RK(ensure(c, c->dni, sizeof(float) * kHoursPerYear));
    RK(ensure(c, c->dhi, sizeof(float) * kHoursPerYear));
    RK(ensure(c, c->sun_dense, sizeof(int) * kHoursPerYear));
    RK(ensure(c, c->hour_index, sizeof(int) * (Hd + 1)));
    RK(ensure(c, c->table, sizeof(HourEntry) * n_padded));
    RK(ensure(c, c->err, sizeof(int)));
    CK(cudaMemcpyAsync(c->dirs.p, sky.dirs.data(), sizeof(DirEntry) * D, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->nudged.p, sky.nudged.data(), sizeof(float) * 2 * kHoursPerYear, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->dni.p, s->direct_irradiance, sizeof(float) * kHoursPerYear, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->dhi.p, s->diffuse_irradiance, sizeof(float) * kHoursPerYear, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->sun_dense.p, sky.sun_dense.data(), sizeof(int) * kHoursPerYear, cudaMemcpyHostToDevice, st));
    if (Hd) CK(cudaMemcpyAsync(c->hour_index.p, sky.hour_index.data(), sizeof(int) * Hd, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(c->err.p, 0, sizeof(int), st));
    {
        KScope k(c, SOLAR_GPU_KT_SETUP);
        CK(launch_hour_table(as<float>(c->nudged), as<float>(c->dni), as<float>(c->dhi), as<int>(c->sun_dense),
                             as<int>(c->hour_index), Hd, n_padded, as<HourEntry>(c->table), st));
    }
    const int N = s->num_total_voxels;
    RK(ensure(c, c->geo_n, sizeof(float4) * (size_t)N));
    RK(ensure(c, c->geo_p, sizeof(float4) * (size_t)N));
    {
        KScope k(c, SOLAR_GPU_KT_SETUP);
        k_validate_parents<<<(N + 255) / 256, 256, 0, st>>>(s->pixel_parent, N, s->num_top_voxels, as<int>(c->err));
        CK(cudaGetLastError());
    }
    int bad = 0;
    CK(cudaMemcpyAsync(c->h_scalars, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::memcpy(&bad, c->h_scalars, sizeof(int));
    if (bad) return fail(SOLAR_GPU_ERR_ARG, "pixel_parent violates the voxel layout (tops i -> i, walls in [0, T))");
    DevGeom g{as<float4>(c->geo_n), as<float4>(c->geo_p)};
    {
        KScope k(c, SOLAR_GPU_KT_SETUP);
        CK(launch_voxel_geom(dev_scene(s), g, st));
    }
    {
        const long long npos = order_positions(s->grid_width, s->grid_height);
        RK(ensure(c, c->order, sizeof(int) * (size_t)N));
        RK(ensure(c, c->order_cnt, sizeof(int) * (size_t)npos));
        RK(ensure(c, c->order_first, sizeof(int) * ((size_t)npos + 1)));
        RK(ensure(c, c->order_cur, sizeof(long long) * ((size_t)npos + 1)));
        RK(ensure(c, c->order_tmp, sizeof(long long) * scan_scratch_elems((int)npos)));
        KScope k(c, SOLAR_GPU_KT_SETUP);
        CK(launch_voxel_order(s->pixel_parent, N, s->num_top_voxels, s->grid_width, s->grid_height,
                              as<int>(c->order_cnt), as<int>(c->order_first), as<long long>(c->order_cur),
                              as<long long>(c->order_tmp), as<int>(c->order), st));
    }
    c->launches += 8;
    return SOLAR_GPU_OK;
}

long long auto_chunk(solar_gpu_context* c, int N, int D)
{
    // A raw buffer kept from an earlier call that holds the whole scene is
    // reused without asking the driver for free memory (that query can wait
    // behind other processes' driver calls, e.g. monitoring tools).
    if (c->raw.cap >= sizeof(int) * (size_t)N * D) return N;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = (size_t)8 << 30;
    if (c->mem_limit > 0) {
        // under a memory limit: what the limit leaves, counting the raw buffer's current size as free
        const size_t held = held_bytes(c) - c->raw.cap;
        const size_t room = (size_t)c->mem_limit > held ? (size_t)c->mem_limit - held : 0;
        if (room < free_b) free_b = room;
    }
    // The raw hit rows (D ints per voxel) get at most 35 % of free memory.
    const double budget = 0.35 * (double)free_b;
    long long chunk = (long long)(budget / ((double)D * sizeof(int)));
    if (chunk < 1024) chunk = 1024;
    if (chunk > N) chunk = N;
    return chunk;
}

// The tracer's copy of the heightmap inside a border of +inf and the
// early-exit tables of the upper directions (cone.cu), rebuilt each call (the
// caller may change heights between calls).  The tables' build scratch is the
// raw hit buffer (not yet written: the tracer runs after the build) when it
// is large enough.  New table memory may take a sixteenth of the free device
// memory (and of what a memory limit leaves): the tables only save time, and
// contexts of many tiles held at once leave little room; past that, or with
// SGB_CONE=0, the tracer runs without them (the reference's range test
// alone).
int padded_grid(solar_gpu_context* c, const solar_gpu_scene* s, const SkyTables& sky, DevScene& ds,
                cudaStream_t st)
{
    const int W = s->grid_width, H = s->grid_height;
    const size_t cells = (size_t)(W + 2) * (size_t)(H + 2);
    RK(ensure(c, c->gpad, sizeof(float) * cells));
    CK(launch_pad_grid(s->grid, W, H, as<float>(c->gpad), st));
    int nt = (int)sky.cones.size();
    if (const char* env = std::getenv("SGB_CONE"))
        if (std::atoi(env) == 0) nt = 0;
    DevBuf& tabs = c->cone_shared ? *c->cone_shared : c->cone;
    const size_t bytes = sizeof(float) * cells * (size_t)nt;
    const bool scratch_in_raw = c->raw.cap >= bytes;
    // device memory these tables would add to what the context holds
    const size_t grow = (bytes > tabs.cap ? bytes - tabs.cap : 0) +
                        (!scratch_in_raw && bytes > c->cone_tmp.cap ? bytes - c->cone_tmp.cap : 0);
    if (nt > 0 && grow > 0) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
        size_t room = free_b;
        if (c->mem_limit > 0) {
            const size_t held = held_bytes(c);
            room = std::min(room, (size_t)c->mem_limit > held ? (size_t)c->mem_limit - held : (size_t)0);
        }
        if (grow > room / 16) nt = 0;
    }
    ds.gpad = as<float>(c->gpad);
    ds.cone = nullptr;
    ds.cone_stride = 0;
    c->launches += 1;
    if (nt == 0) return SOLAR_GPU_OK;
    if (ensure(c, tabs, bytes) != SOLAR_GPU_OK ||
        (!scratch_in_raw && ensure(c, c->cone_tmp, bytes) != SOLAR_GPU_OK)) {
        (void)cudaGetLastError();   // no room after all: the tracer runs without the tables
        return SOLAR_GPU_OK;
    }
    RK(ensure(c, c->cone_specs, sizeof(ConeSpec) * nt));
    CK(cudaMemcpyAsync(c->cone_specs.p, sky.cones.data(), sizeof(ConeSpec) * nt, cudaMemcpyHostToDevice, st));
    CK(launch_cone_tables(s->grid, W, H, s->max_height, as<ConeSpec>(c->cone_specs), nt, as<float>(tabs),
                          scratch_in_raw ? as<float>(c->raw) : as<float>(c->cone_tmp), cells, st));
    c->launches += 5;
    ds.cone = as<float>(tabs);
    ds.cone_stride = cells;
    return SOLAR_GPU_OK;
}

int stage1(solar_gpu_context* c, const solar_gpu_options* o, const solar_gpu_scene* s,
           const SkyTables& sky, cudaStream_t st, bool want_csr, bool want_barle)
{
    const int N = s->num_total_voxels;
    const int D = (int)sky.dirs.size();
    const long long chunk = o->chunk_voxels > 0 ? (o->chunk_voxels < N ? o->chunk_voxels : N) : auto_chunk(c, N, D);
    c->N = N;
    c->T = s->num_top_voxels;
    c->words32 = sky.words32 > 0 ? sky.words32 : 1;
    c->active = sky.active;
    c->have_csr = want_csr;
    c->have_barle = want_barle;
    c->csr_total = c->barle_total = 0;
    RK(ensure(c, c->shadow, sizeof(uint32_t) * (size_t)N * c->words32));
    CK(cudaMemsetAsync(c->shadow.p, 0, sizeof(uint32_t) * (size_t)N * c->words32, st));
    RK(ensure(c, c->raw, sizeof(int) * (size_t)chunk * D));
    RK(ensure(c, c->counts, sizeof(int) * (size_t)N));
    RK(ensure(c, c->dd_ovf, sizeof(int) * ((size_t)chunk + 1)));
    RK(ensure(c, c->scan_tmp, sizeof(long long) * scan_scratch_elems((int)chunk)));
    if (want_csr) {
        RK(ensure(c, c->csr_off, sizeof(long long) * ((size_t)N + 1)));
        RK(ensure(c, c->csr_ids, sizeof(int) * (size_t)N * 96));
    }
    if (want_barle) {
        RK(ensure(c, c->barle_off, sizeof(long long) * ((size_t)N + 1)));
        RK(ensure(c, c->barle_sizes, sizeof(int) * (size_t)N));
        RK(ensure(c, c->barle_bytes, (size_t)N * 160));
    }
    DevScene ds = dev_scene(s);
    {
        KScope k(c, SOLAR_GPU_KT_TRACE);   // the tracer's inputs count with the tracer
        RK(padded_grid(c, s, sky, ds, st));
    }
    // Rows follow the visiting order (Morton-adjacent voxels share a warp, so
    // their rays have similar lengths); with several chunks, each chunk (a
    // range of voxel indices) is traced in the visiting order of its voxels.
    const int* perm = nullptr;
    const int* inv = nullptr;
    RK(ensure(c, c->order_inv, sizeof(int) * (size_t)N));
    if (chunk >= N) {
        CK(launch_invert(as<int>(c->order), N, as<int>(c->order_inv), st));
        perm = as<int>(c->order);
        inv = as<int>(c->order_inv);
        c->launches += 1;
    } else {
        RK(ensure(c, c->chunk_perm, sizeof(int) * (size_t)chunk));
        RK(ensure(c, c->chunk_flag, sizeof(int) * (size_t)N));
        RK(ensure(c, c->chunk_pos, sizeof(long long) * ((size_t)N + 1)));
        RK(ensure(c, c->chunk_tmp, sizeof(long long) * scan_scratch_elems(N)));
        perm = as<int>(c->chunk_perm);
        inv = as<int>(c->order_inv);
    }
    long long csr_total = 0, barle_total = 0;
    for (long long v0 = 0; v0 < N; v0 += chunk) {
        const int n = (int)((N - v0) < chunk ? (N - v0) : chunk);
        if (chunk < N) {
            KScope k(c, SOLAR_GPU_KT_SETUP);
            CK(launch_chunk_order(as<int>(c->order), N, (int)v0, n, as<int>(c->chunk_flag),
                                  as<long long>(c->chunk_pos), as<long long>(c->chunk_tmp),
                                  as<int>(c->chunk_perm), st));
            CK(launch_invert(as<int>(c->chunk_perm), n, as<int>(c->order_inv), st));
            c->launches += 6;
        }
        {
            KScope k(c, SOLAR_GPU_KT_TRACE);
            CK(launch_trace(ds, as<DirEntry>(c->dirs), D, c->words32, (int)v0, n, as<int>(c->raw),
                            as<uint32_t>(c->shadow), perm, as<int>(c->err), st));
        }
        {
            KScope k(c, SOLAR_GPU_KT_DEDUPE);
            CK(launch_dedupe(n, D, as<int>(c->raw), as<int>(c->counts) + v0, as<int>(c->err), perm,
                             as<int>(c->dd_ovf), st));
        }
        c->launches += 2;
        const double frac_left = (double)N / (double)(v0 + n);
        if (want_csr) {
            long long* off = as<long long>(c->csr_off) + v0;
            {
                KScope k(c, SOLAR_GPU_KT_CSR);
                CK(launch_scan_counts(as<int>(c->counts) + v0, n, csr_total, off, as<long long>(c->scan_tmp), nullptr, st));
            }
            long long total = 0;
            RK(read_ll(c, off + n, &total, st));
            const long long est = (long long)(total * frac_left * 1.05);
            RK(ensure_keep(c, c->csr_ids, sizeof(int) * (size_t)(est > total ? est : total), sizeof(int) * (size_t)csr_total, st));
            {
                KScope k(c, SOLAR_GPU_KT_CSR);
                CK(launch_gather_csr(n, D, as<int>(c->raw), off, as<int>(c->csr_ids), inv, st));
            }
            csr_total = total;
            c->launches += 4;
        }
        if (want_barle) {
            long long* off = as<long long>(c->barle_off) + v0;
            {
                KScope k(c, SOLAR_GPU_KT_BARLE);
                CK(launch_barle_size(n, D, as<int>(c->raw), as<int>(c->counts) + v0, as<int>(c->barle_sizes) + v0,
                                     as<int>(c->err), perm, st));
                CK(launch_scan_counts(as<int>(c->barle_sizes) + v0, n, barle_total, off, as<long long>(c->scan_tmp), nullptr, st));
            }
            long long total = 0;
            RK(read_ll(c, off + n, &total, st));
            const long long est = (long long)(total * frac_left * 1.05);
            RK(ensure_keep(c, c->barle_bytes, (size_t)(est > total ? est : total), (size_t)barle_total, st));
            {
                KScope k(c, SOLAR_GPU_KT_BARLE);
                CK(launch_barle_write(n, D, as<int>(c->raw), as<int>(c->counts) + v0, off,
                                      as<unsigned char>(c->barle_bytes), as<int>(c->err), inv, st));
            }
            barle_total = total;
            c->launches += 5;
        }
    }
    c->csr_total = csr_total;
    c->barle_total = barle_total;
    // A raw hit buffer above a quarter of the device (scenes of tens of
    // millions of voxels) is released here to leave room for Stage 2/3;
    // smaller ones are kept for the next call.
    if (c->raw.cap > c->dev_total / 4) {
        c->squeezed = true;
        for (DevBuf* b : {&c->raw, &c->cone, &c->cone_tmp}) {
            CK(cudaFree(b->p));
            b->p = nullptr;
            b->cap = 0;
        }
    }
    return SOLAR_GPU_OK;
}

// The hour-block loop of one run (solar slab + reflection per block of B
// hours) and the final conversion of the accumulators into the output.
cudaError_t enqueue_hours(solar_gpu_context* c, const HourLoop& h, cudaStream_t st)
{
    cudaError_t le = cudaSuccess;
    for (int j0 = 0; j0 < h.Hd && le == cudaSuccess; j0 += h.B) {
        {
            KScope k(c, SOLAR_GPU_KT_SOLAR);
            le = h.mma ? launch_solar_slab16(h.g, h.T, h.sh, h.words32, h.tab, j0, h.slab16, st)
                       : launch_solar_slab(h.g, h.slab_rows, h.sh, h.words32, h.tab, j0, h.B, h.slab, st);
        }
        if (le == cudaSuccess) {
            KScope k(c, SOLAR_GPU_KT_REFLECT);
            if (h.mma)
                le = launch_reflect_mma(h.slab16, h.ml, h.g, h.sh, h.words32, h.tab, j0, h.acc, h.err, st);
            else if (h.tiled)
                le = launch_reflect_tile(h.B, h.slab, h.tl, h.order, h.acc, h.err, st);
            else if (h.group_size > 0)
                le = launch_reflect_group(h.N, h.B, h.slab, h.gl, h.order, h.acc, st);
            else
                le = launch_reflect_block(h.g, h.N, h.T, h.sh, h.words32, h.tab, j0, h.B, h.slab, h.nl, h.acc,
                                          h.order, h.err, st);
        }
        c->launches += 2;
    }
    if (le == cudaSuccess) {
        KScope k(c, SOLAR_GPU_KT_FINALIZE);
        le = launch_finalize(h.acc, h.N, h.out, st);
        c->launches += 1;
    }
    return le;
}

int stage23(solar_gpu_context* c, const solar_gpu_options* o, const solar_gpu_scene* s,
            const SkyTables& sky, float* out, cudaStream_t st)
{
    const int N = s->num_total_voxels, T = s->num_top_voxels;
    const int Hd = (int)sky.hour_index.size();
    const int B = o->hour_block == 0 ? 128 : o->hour_block;
    DevGeom g{as<float4>(c->geo_n), as<float4>(c->geo_p)};
    NeighborLists nl;
    nl.format = o->neighbor_format;
    if (nl.format == SOLAR_GPU_CSR) {
        nl.offsets = as<long long>(c->csr_off);
        nl.ids = as<int>(c->csr_ids);
        nl.bytes = nullptr;
    } else {
        nl.offsets = as<long long>(c->barle_off);
        nl.ids = nullptr;
        nl.bytes = as<unsigned char>(c->barle_bytes);
    }
    const uint32_t* sh = as<uint32_t>(c->shadow);
    const HourEntry* tab = as<HourEntry>(c->table);
    int* err = as<int>(c->err);
    if (o->reflection == SOLAR_GPU_REFL_NONE) {
        // own direct + diffuse only: the annual form's FP64 sums, no reflection
        RK(ensure(c, c->sums, sizeof(double) * (size_t)N));
        {
            KScope k(c, SOLAR_GPU_KT_SOLAR);
            CK(launch_solar_sum(g, N, sh, c->words32, tab, Hd, as<double>(c->sums), st));
        }
        {
            KScope k(c, SOLAR_GPU_KT_FINALIZE);
            CK(launch_finalize_f64(as<double>(c->sums), N, out, st));
        }
        c->launches += 2;
        return SOLAR_GPU_OK;
    }
    if (o->reflection == SOLAR_GPU_REFL_ANNUAL) {
        RK(ensure(c, c->sums, sizeof(double) * (size_t)N));
        RK(ensure(c, c->out_f64, sizeof(double) * (size_t)N));
        {
            KScope k(c, SOLAR_GPU_KT_SOLAR);
            CK(launch_solar_sum(g, N, sh, c->words32, tab, Hd, as<double>(c->sums), st));
        }
        {
            KScope k(c, SOLAR_GPU_KT_REFLECT);
            CK(launch_reflect_annual(g, N, T, as<double>(c->sums), nl, as<double>(c->out_f64), err, st));
        }
        {
            KScope k(c, SOLAR_GPU_KT_FINALIZE);
            CK(launch_finalize_f64(as<double>(c->out_f64), N, out, st));
        }
        c->launches += 3;
        return SOLAR_GPU_OK;
    }
    Accum acc;
    acc.mode = o->accumulation;
    acc.f64 = nullptr;
    acc.f32 = acc.comp = nullptr;
    if (acc.mode == SOLAR_GPU_ACC_FP64) {
        RK(ensure(c, c->acc_f64, sizeof(double) * (size_t)N));
        acc.f64 = as<double>(c->acc_f64);
        CK(cudaMemsetAsync(acc.f64, 0, sizeof(double) * (size_t)N, st));
    } else {
        RK(ensure(c, c->acc_f32, sizeof(float) * (size_t)N));
        RK(ensure(c, c->acc_comp, sizeof(float) * (size_t)N));
        acc.f32 = as<float>(c->acc_f32);
        acc.comp = as<float>(c->acc_comp);
        CK(cudaMemsetAsync(acc.f32, 0, sizeof(float) * (size_t)N, st));
        CK(cudaMemsetAsync(acc.comp, 0, sizeof(float) * (size_t)N, st));
    }
    if (B == 1) {
        RK(ensure(c, c->hourly, sizeof(float) * (size_t)N));
        for (int j = 0; j < Hd; ++j) {
            {
                KScope k(c, SOLAR_GPU_KT_SOLAR);
                CK(launch_solar_hour(g, N, sh, c->words32, tab, j, as<float>(c->hourly), st));
            }
            {
                KScope k(c, SOLAR_GPU_KT_REFLECT);
                CK(launch_reflect_hour(g, N, T, as<float>(c->hourly), nl, acc, err, st));
            }
        }
        c->launches += 2LL * Hd;
    } else {
        // Rows for the top cells (neighbor values); the weighted-list kernels
        // also read each voxel's own row, so there the slab covers all voxels.
        const int slab_rows = o->group_size > 0 ? N : T;
        GroupLists gl{o->group_size, nullptr, nullptr, nullptr};
        TileLists tl{};
        MmaLists ml{};
        // group_size 128: the tensor-core kernel; a scene with a group whose
        // union of neighbor cells exceeds the build's cap runs the shared-
        // memory tile kernel (group_size 64) instead.
        bool mma = o->group_size == kMmaGroup;
        bool tiled = o->group_size >= 64;
        if (o->group_size > 0) {
            // Once per run: the nonzero weights of every list in visiting order,
            // then (V > 1) the merged union entries of each group of V voxels.
            int V = o->group_size;
            RK(ensure(c, c->w_cnt, sizeof(int) * (size_t)N));
            RK(ensure(c, c->w_off, sizeof(long long) * ((size_t)N + 1)));
            RK(ensure(c, c->w_tmp, sizeof(long long) * scan_scratch_elems(N)));
            {
                KScope k(c, SOLAR_GPU_KT_GROUP);
                CK(launch_weight_lists(0, g, N, T, nl, as<int>(c->order), as<int>(c->w_cnt), nullptr, nullptr,
                                       nullptr, err, st));
                CK(launch_scan_counts(as<int>(c->w_cnt), N, 0, as<long long>(c->w_off), as<long long>(c->w_tmp),
                                      nullptr, st));
            }
            long long Ew = 0;
            RK(read_ll(c, as<long long>(c->w_off) + N, &Ew, st));
            c->weighted_entries = Ew;
            RK(ensure(c, c->w_cell, sizeof(int) * (size_t)(Ew + 1)));
            RK(ensure(c, c->w_val, sizeof(float) * (size_t)(Ew + 1)));
            {
                KScope k(c, SOLAR_GPU_KT_GROUP);
                CK(launch_weight_lists(1, g, N, T, nl, as<int>(c->order), nullptr, as<long long>(c->w_off),
                                       as<int>(c->w_cell), as<float>(c->w_val), err, st));
            }
            c->launches += 5;
            if (mma) {
                const int NG = mma_group_count(N);
                RK(ensure(c, c->tile_slot, sizeof(unsigned short) * (size_t)(Ew + 1)));
                RK(ensure(c, c->mma_union, sizeof(int) * (size_t)NG));
                RK(ensure(c, c->mma_nch, sizeof(int) * (size_t)NG));
                RK(ensure(c, c->mma_cbase, sizeof(long long) * ((size_t)NG + 1)));
                RK(ensure(c, c->mma_over, sizeof(long long)));
                RK(ensure(c, c->mma_retry, sizeof(int) * ((size_t)NG + 1)));
                {
                    KScope k(c, SOLAR_GPU_KT_GROUP);
                    CK(cudaMemsetAsync(c->mma_over.p, 0, sizeof(long long), st));
                    CK(launch_mma_union(N, as<long long>(c->w_off), as<int>(c->w_cell),
                                        as<unsigned short>(c->tile_slot), as<int>(c->mma_union), as<int>(c->mma_nch),
                                        as<int>(c->mma_over), as<int>(c->mma_retry), st));
                    CK(launch_scan_counts(as<int>(c->mma_nch), NG, 0, as<long long>(c->mma_cbase),
                                          as<long long>(c->w_tmp), nullptr, st));
                }
                long long over = 0, C = 0;
                RK(read_ll(c, as<long long>(c->mma_over), &over, st));
                RK(read_ll(c, as<long long>(c->mma_cbase) + NG, &C, st));
                c->launches += 4;
                if (over != 0) {
                    // the union build rewrote the cells of the groups it kept: rebuild the lists
                    mma = false;
                    V = 64;
                    KScope k(c, SOLAR_GPU_KT_GROUP);
                    CK(launch_weight_lists(1, g, N, T, nl, as<int>(c->order), nullptr, as<long long>(c->w_off),
                                           as<int>(c->w_cell), as<float>(c->w_val), err, st));
                    c->launches += 1;
                } else {
                    RK(ensure(c, c->mma_ccnt, sizeof(int) * (size_t)(C + 1)));
                    RK(ensure(c, c->mma_coff, sizeof(long long) * ((size_t)C + 1)));
                    RK(ensure(c, c->mma_scale, sizeof(float) * (size_t)N));
                    RK(ensure(c, c->mma_ent, 8 * (size_t)(Ew + 1)));
                    {
                        KScope k(c, SOLAR_GPU_KT_GROUP);
                        CK(launch_mma_layout(0, N, as<long long>(c->w_off), as<unsigned short>(c->tile_slot),
                                             as<float>(c->w_val), as<int>(c->mma_nch), as<long long>(c->mma_cbase),
                                             as<int>(c->mma_ccnt), nullptr, nullptr, as<float>(c->mma_scale), st));
                        RK(ensure(c, c->chunk_tmp, sizeof(long long) * scan_scratch_elems((int)C)));
                        CK(launch_scan_counts(as<int>(c->mma_ccnt), (int)C, 0, as<long long>(c->mma_coff),
                                              as<long long>(c->chunk_tmp), nullptr, st));
                        CK(launch_mma_layout(1, N, as<long long>(c->w_off), as<unsigned short>(c->tile_slot),
                                             as<float>(c->w_val), as<int>(c->mma_nch), as<long long>(c->mma_cbase),
                                             as<int>(c->mma_ccnt), as<long long>(c->mma_coff),
                                             static_cast<uint2*>(c->mma_ent.p), as<float>(c->mma_scale), st));
                    }
                    c->launches += 3;
                    c->group_entries = Ew;
                    c->staged_rows = C * kMmaChunk;
                    // weights and slots are dead now (see the tile path below)
                    if (c->w_val.cap + c->tile_slot.cap > c->dev_total / 16) {
                        c->squeezed = true;
                        CK(cudaFree(c->w_val.p));
                        CK(cudaFree(c->tile_slot.p));
                        c->w_val.p = c->tile_slot.p = nullptr;
                        c->w_val.cap = c->tile_slot.cap = 0;
                    }
                    ml.N = N;
                    ml.order = as<int>(c->order);
                    ml.woff = as<long long>(c->w_off);
                    ml.cells = as<int>(c->w_cell);
                    ml.unions = as<int>(c->mma_union);
                    ml.cbase = as<long long>(c->mma_cbase);
                    ml.coff = as<long long>(c->mma_coff);
                    ml.ent = c->mma_ent.p;
                    ml.scale = as<float>(c->mma_scale);
                    // balanced group order over the CTAs of the hour-block kernel
                    std::vector<long long> cb((size_t)NG + 1);
                    CK(cudaMemcpyAsync(cb.data(), c->mma_cbase.p, sizeof(long long) * ((size_t)NG + 1),
                                       cudaMemcpyDeviceToHost, st));
                    CK(cudaStreamSynchronize(st));
                    std::vector<int> sched((size_t)mma_grid(N) + 1 + NG);
                    mma_schedule(N, cb.data(), sched.data());
                    RK(ensure(c, c->mma_sched, sizeof(int) * sched.size()));
                    CK(cudaMemcpyAsync(c->mma_sched.p, sched.data(), sizeof(int) * sched.size(), cudaMemcpyHostToDevice,
                                       st));
                    ml.sched = as<int>(c->mma_sched);
                }
            }
            if (mma) {
                // built above
            } else if (V == 1) {
                c->group_entries = Ew;
                gl.offsets = as<long long>(c->w_off);
                gl.cells = as<int>(c->w_cell);
                gl.weights = as<float>(c->w_val);
            } else if (tiled) {
                // Groups of up to V visiting positions; the weighted lists of
                // each group are rewritten in place into union cells + slots,
                // then the slot lists of each 4 consecutive voxels are merged
                // and laid out chunk by chunk.
                RK(ensure(c, c->tile_flag, sizeof(int) * (size_t)N));
                RK(ensure(c, c->tile_pos, sizeof(long long) * ((size_t)N + 1)));
                RK(ensure(c, c->tile_start, sizeof(int) * ((size_t)N + 1)));
                RK(ensure(c, c->tile_slot, sizeof(unsigned short) * (size_t)(Ew + 1)));
                {
                    KScope k(c, SOLAR_GPU_KT_GROUP);
                    CK(launch_tile_groups(N, V, as<long long>(c->w_off), as<int>(c->tile_flag),
                                          as<long long>(c->tile_pos), as<long long>(c->w_tmp),
                                          as<int>(c->tile_start), st));
                }
                long long NG = 0;
                RK(read_ll(c, as<long long>(c->tile_pos) + N, &NG, st));
                RK(ensure(c, c->tile_union, sizeof(int) * (size_t)(NG + 1)));
                RK(ensure(c, c->tile_rows, sizeof(long long)));
                {
                    KScope k(c, SOLAR_GPU_KT_GROUP);
                    CK(launch_tile_build((int)NG, as<int>(c->tile_start), as<long long>(c->w_off),
                                         as<int>(c->w_cell), as<unsigned short>(c->tile_slot),
                                         as<int>(c->tile_union), as<long long>(c->tile_rows), err, st));
                }
                RK(read_ll(c, as<long long>(c->tile_rows), &c->staged_rows, st));
                const int R = tile_rows_per_stage(B);
                RK(ensure(c, c->tile_gcnt, sizeof(int) * (size_t)NG));
                RK(ensure(c, c->tile_gnch, sizeof(int) * (size_t)NG));
                RK(ensure(c, c->tile_gbase, sizeof(long long) * ((size_t)NG + 1)));
                RK(ensure(c, c->tile_tbase, sizeof(long long) * ((size_t)NG + 1)));
                {
                    KScope k(c, SOLAR_GPU_KT_GROUP);
                    CK(launch_tile_layout(0, (int)NG, R, as<int>(c->tile_start), as<int>(c->tile_union),
                                          as<long long>(c->w_off), as<unsigned short>(c->tile_slot),
                                          as<float>(c->w_val), as<int>(c->tile_gcnt), as<int>(c->tile_gnch),
                                          nullptr, nullptr, nullptr, nullptr, nullptr, st));
                    CK(launch_scan_counts(as<int>(c->tile_gcnt), (int)NG, 0, as<long long>(c->tile_gbase),
                                          as<long long>(c->w_tmp), nullptr, st));
                    CK(launch_scan_counts(as<int>(c->tile_gnch), (int)NG, 0, as<long long>(c->tile_tbase),
                                          as<long long>(c->w_tmp), nullptr, st));
                }
                long long Em = 0, TC = 0;
                RK(read_ll(c, as<long long>(c->tile_gbase) + NG, &Em, st));
                RK(read_ll(c, as<long long>(c->tile_tbase) + NG, &TC, st));
                RK(ensure(c, c->tile_erow, sizeof(unsigned short) * (size_t)(Em + 8)));
                RK(ensure(c, c->tile_ew, sizeof(float4) * (size_t)(Em + 8)));
                RK(ensure(c, c->tile_table, sizeof(int) * 20 * (size_t)(TC + 1)));
                {
                    KScope k(c, SOLAR_GPU_KT_GROUP);
                    CK(cudaMemsetAsync(c->tile_ew.p, 0, sizeof(float4) * (size_t)(Em + 8), st));
                    CK(launch_tile_layout(1, (int)NG, R, as<int>(c->tile_start), as<int>(c->tile_union),
                                          as<long long>(c->w_off), as<unsigned short>(c->tile_slot),
                                          as<float>(c->w_val), nullptr, nullptr, as<long long>(c->tile_gbase),
                                          as<long long>(c->tile_tbase), as<int>(c->tile_table),
                                          as<unsigned short>(c->tile_erow), as<float4>(c->tile_ew), st));
                }
                c->launches += 10;
                c->group_entries = Em;
                // Per-voxel weights and slots are dead now; above 1/16 of the
                // device (scenes of tens of millions of voxels) they are
                // released to make room for the slab.
                if (c->w_val.cap + c->tile_slot.cap > c->dev_total / 16) {
                    c->squeezed = true;
                    CK(cudaFree(c->w_val.p));
                    CK(cudaFree(c->tile_slot.p));
                    c->w_val.p = c->tile_slot.p = nullptr;
                    c->w_val.cap = c->tile_slot.cap = 0;
                }
                tl.G = V;
                tl.NG = (int)NG;
                tl.start = as<int>(c->tile_start);
                tl.unions = as<int>(c->tile_union);
                tl.woff = as<long long>(c->w_off);
                tl.cells = as<int>(c->w_cell);
                tl.R = R;
                tl.gbase = as<long long>(c->tile_gbase);
                tl.tbase = as<long long>(c->tile_tbase);
                tl.table = as<int>(c->tile_table);
                tl.erow = as<unsigned short>(c->tile_erow);
                tl.ew = as<float4>(c->tile_ew);
            } else {
                const int G = group_count(N, V);
                RK(ensure(c, c->grp_cnt, sizeof(int) * (size_t)G));
                RK(ensure(c, c->grp_off, sizeof(long long) * ((size_t)G + 1)));
                RK(ensure(c, c->grp_tmp, sizeof(long long) * scan_scratch_elems(G)));
                {
                    KScope k(c, SOLAR_GPU_KT_GROUP);
                    CK(launch_group_merge(0, V, N, as<long long>(c->w_off), as<int>(c->w_cell), as<float>(c->w_val),
                                          as<int>(c->grp_cnt), nullptr, nullptr, nullptr, st));
                    CK(launch_scan_counts(as<int>(c->grp_cnt), G, 0, as<long long>(c->grp_off),
                                          as<long long>(c->grp_tmp), nullptr, st));
                }
                long long E = 0;
                RK(read_ll(c, as<long long>(c->grp_off) + G, &E, st));
                RK(ensure(c, c->grp_cell, sizeof(int) * (size_t)(E + 1)));
                RK(ensure(c, c->grp_w, sizeof(float) * (size_t)(E + 1) * V));
                {
                    KScope k(c, SOLAR_GPU_KT_GROUP);
                    CK(launch_group_merge(1, V, N, as<long long>(c->w_off), as<int>(c->w_cell), as<float>(c->w_val),
                                          as<int>(c->grp_cnt), as<long long>(c->grp_off), as<int>(c->grp_cell),
                                          as<float>(c->grp_w), st));
                }
                c->group_entries = E;
                c->launches += 5;
                gl.offsets = as<long long>(c->grp_off);
                gl.cells = as<int>(c->grp_cell);
                gl.weights = as<float>(c->grp_w);
            }
        }
        if (o->group_size > 0 && c->squeezed) {
            // Very large scenes: the hour loop reads only the weighted lists
            // (or the group layouts built from them), so the CSR / ba-RLE
            // lists are released to make room for the slab; solar_gpu_trace
            // (Stage 1 alone) keeps them.
            CK(cudaStreamSynchronize(st));
            for (DevBuf* b : {&c->csr_ids, &c->barle_bytes}) {
                if (b->p) CK(cudaFree(b->p));
                b->p = nullptr;
                b->cap = 0;
            }
            c->have_csr = c->have_barle = false;
        }
        // allocated after the once-per-run builds, whose intermediates may
        // have been released to make room (very large scenes); the tensor-core
        // kernel reads an fp16 slab of the top cells only
        float* slab = nullptr;
        if (mma) {
            RK(ensure(c, c->slab16, 2 * (size_t)T * kMmaHours));
        } else {
            RK(ensure(c, c->slab, sizeof(float) * (size_t)slab_rows * B));
            slab = as<float>(c->slab);
        }
        HourLoop& h = c->hours;
        h = HourLoop{};
        h.mma = mma;
        h.tiled = tiled;
        h.group_size = o->group_size;
        h.N = N;
        h.T = T;
        h.Hd = Hd;
        h.B = B;
        h.slab_rows = slab_rows;
        h.words32 = c->words32;
        h.g = g;
        h.sh = sh;
        h.tab = tab;
        h.slab = slab;
        h.slab16 = c->slab16.p;
        h.ml = ml;
        h.tl = tl;
        h.gl = gl;
        h.nl = nl;
        h.acc = acc;
        h.err = err;
        h.order = as<int>(c->order);
        h.out = out;
        if (c->defer_hours) return SOLAR_GPU_OK;   // enqueued by solar_gpu_run_batch
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        const bool use_graph = o->use_graph != 0 && !c->ktime;
        if (use_graph) CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t le = enqueue_hours(c, h, st);
        if (use_graph) {
            const cudaError_t ce = cudaStreamEndCapture(st, &graph);
            if (le == cudaSuccess) le = ce;
            if (le == cudaSuccess) le = cudaGraphInstantiate(&exec, graph, 0);
            if (le == cudaSuccess) le = cudaGraphLaunch(exec, st);
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
        }
        CK(le);
        return SOLAR_GPU_OK;
    }
    {
        KScope k(c, SOLAR_GPU_KT_FINALIZE);
        CK(launch_finalize(acc, N, out, st));
    }
    c->launches += 1;
    return SOLAR_GPU_OK;
}

int check_device_flags(solar_gpu_context* c, cudaStream_t st)
{
    CK(cudaMemcpyAsync(c->h_scalars, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int f = 0;
    std::memcpy(&f, c->h_scalars, sizeof(int));
    if (f) return fail(SOLAR_GPU_ERR_DEVICE_CHECK, "device check flags 0x%x (1 = ba-RLE stream, 2 = hash, 4 = capacity, 8 = wait timeout, 16 = tracer border)", f);
    return SOLAR_GPU_OK;
}

int run_device_impl(solar_gpu_context* c, const solar_gpu_options* o, const solar_gpu_scene* s,
                    float* out, cudaStream_t st, bool trace_only)
{
    RK(check_scene(s));
    RK(check_options(o, trace_only));
    if (!trace_only && !out) return fail(SOLAR_GPU_ERR_ARG, "irradiance output is NULL");
    CK(cudaSetDevice(c->device));
    if (c->squeezed) {
        // The previous run released buffers to fit: the Stage 2/3 buffers it
        // still holds (slabs, weighted lists, group layouts) are rebuilt by
        // every run, and holding them would leave no room for Stage 1.
        CK(cudaStreamSynchronize(st));
        DevBuf* stage23[] = {&c->slab, &c->slab16, &c->w_cnt, &c->w_off, &c->w_cell, &c->w_val, &c->grp_cell,
                             &c->grp_w, &c->tile_slot, &c->tile_erow, &c->tile_ew, &c->tile_table, &c->mma_ent,
                             &c->mma_ccnt, &c->mma_coff, &c->mma_scale, &c->hourly, &c->csr_ids, &c->barle_bytes};
        for (DevBuf* b : stage23) {
            if (b->p) CK(cudaFree(b->p));
            b->p = nullptr;
            b->cap = 0;
        }
        c->squeezed = false;
        c->have_csr = c->have_barle = false;
    }
    c->launches = 0;
    c->timed = false;
    c->ktime = o->time_kernels != 0;
    c->group_entries = 0;
    c->staged_rows = 0;
    c->weighted_entries = 0;
    c->kt_used = 0;
    c->kt_ids.clear();
    c->kt_stream = st;
    CK(cudaEventRecord(c->ev[0], st));
    SkyTables sky;
    RK(prepare(c, s, sky, st));
    CK(cudaEventRecord(c->ev[1], st));
    const bool csr = o->neighbor_format == SOLAR_GPU_CSR || o->neighbor_format == SOLAR_GPU_BOTH;
    const bool barle = o->neighbor_format == SOLAR_GPU_BARLE || o->neighbor_format == SOLAR_GPU_BOTH;
    RK(stage1(c, o, s, sky, st, csr, barle));
    CK(cudaEventRecord(c->ev[2], st));
    if (!trace_only) RK(stage23(c, o, s, sky, out, st));
    CK(cudaEventRecord(c->ev[3], st));
    c->timed = true;
    return SOLAR_GPU_OK;
}

int run_lists_impl(solar_gpu_context* c, const solar_gpu_options* o_in, const solar_gpu_scene* s,
                   const solar_gpu_lists* l, float* out, cudaStream_t st)
{
    if (!o_in || !l) return fail(SOLAR_GPU_ERR_ARG, "options or lists is NULL");
    if (l->format != SOLAR_GPU_CSR && l->format != SOLAR_GPU_BARLE)
        return fail(SOLAR_GPU_ERR_ARG, "lists format %d", l->format);
    solar_gpu_options o = *o_in;
    o.neighbor_format = l->format;
    RK(check_scene(s));
    RK(check_options(&o, false));
    if (!out) return fail(SOLAR_GPU_ERR_ARG, "irradiance output is NULL");
    const int N = s->num_total_voxels;
    if (!l->offsets || !l->shadow || (l->data_size > 0 && !l->data) || l->data_size < 0)
        return fail(SOLAR_GPU_ERR_ARG, "lists arrays are NULL");
    if (l->offsets[0] != 0 || l->offsets[N] != l->data_size)
        return fail(SOLAR_GPU_ERR_ARG, "list offsets run from %lld to %lld, data has %lld", l->offsets[0],
                    l->offsets[N], l->data_size);
    for (int v = 0; v < N; ++v)
        if (l->offsets[v + 1] < l->offsets[v]) return fail(SOLAR_GPU_ERR_ARG, "list offsets decrease at voxel %d", v);
    CK(cudaSetDevice(c->device));
    c->launches = 0;
    c->timed = false;
    c->ktime = o.time_kernels != 0;
    c->group_entries = 0;
    c->staged_rows = 0;
    c->weighted_entries = 0;
    c->kt_used = 0;
    c->kt_ids.clear();
    c->kt_stream = st;
    CK(cudaEventRecord(c->ev[0], st));
    SkyTables sky;
    RK(prepare(c, s, sky, st));
    const int words32 = sky.words32 > 0 ? sky.words32 : 1;
    if (l->shadow_words != words32 || l->active_bins != sky.active)
        return fail(SOLAR_GPU_ERR_ARG, "lists were traced with %d sun bins (%d words), these sun positions give %d (%d)",
                    l->active_bins, l->shadow_words, sky.active, words32);
    CK(cudaEventRecord(c->ev[1], st));
    c->N = N;
    c->T = s->num_top_voxels;
    c->words32 = words32;
    c->active = sky.active;
    c->have_csr = l->format == SOLAR_GPU_CSR;
    c->have_barle = !c->have_csr;
    c->csr_total = c->have_csr ? l->data_size : 0;
    c->barle_total = c->have_barle ? l->data_size : 0;
    RK(ensure(c, c->shadow, sizeof(uint32_t) * (size_t)N * words32));
    CK(cudaMemcpyAsync(c->shadow.p, l->shadow, sizeof(uint32_t) * (size_t)N * words32, cudaMemcpyHostToDevice, st));
    DevBuf& off = c->have_csr ? c->csr_off : c->barle_off;
    DevBuf& dat = c->have_csr ? c->csr_ids : c->barle_bytes;
    const size_t dbytes = (size_t)l->data_size * (c->have_csr ? sizeof(int) : 1);
    RK(ensure(c, off, sizeof(long long) * ((size_t)N + 1)));
    RK(ensure(c, dat, dbytes ? dbytes : 16));
    CK(cudaMemcpyAsync(off.p, l->offsets, sizeof(long long) * ((size_t)N + 1), cudaMemcpyHostToDevice, st));
    if (dbytes) CK(cudaMemcpyAsync(dat.p, l->data, dbytes, cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(c->ev[2], st));
    RK(stage23(c, &o, s, sky, out, st));
    CK(cudaEventRecord(c->ev[3], st));
    CK(cudaStreamSynchronize(st));   // the host arrays may be released after return
    RK(check_device_flags(c, st));
    c->timed = true;
    return SOLAR_GPU_OK;
}

__global__ void k_gather_shadow(const uint32_t* __restrict__ shadow, int words32, const int* __restrict__ voxels,
                                int n, uint32_t* __restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (long long)n * words32) out[t] = shadow[(size_t)voxels[t / words32] * words32 + t % words32];
}

int trace_subset_impl(solar_gpu_context* c, const solar_gpu_scene* s, const int* voxels, int n, uint32_t* out,
                      int* words_out, cudaStream_t st)
{
    RK(check_scene(s));
    if (!voxels || !out || n < 0) return fail(SOLAR_GPU_ERR_ARG, "voxels / output is NULL");
    if (n > (1 << 20)) return fail(SOLAR_GPU_ERR_ARG, "at most %d voxels per call (got %d)", 1 << 20, n);
    CK(cudaSetDevice(c->device));
    c->launches = 0;
    c->ktime = false;
    SkyTables sky;
    RK(prepare(c, s, sky, st));
    const int N = s->num_total_voxels, D = (int)sky.dirs.size();
    const int words32 = sky.words32 > 0 ? sky.words32 : 1;
    if (words_out) *words_out = words32;
    if (n == 0) return SOLAR_GPU_OK;
    // the listed voxels must exist (the tracer reads their parents)
    RK(ensure(c, c->err, sizeof(int)));
    RK(ensure(c, c->shadow, sizeof(uint32_t) * (size_t)N * words32));
    CK(cudaMemsetAsync(c->shadow.p, 0, sizeof(uint32_t) * (size_t)N * words32, st));
    RK(ensure(c, c->raw, sizeof(int) * (size_t)n * D));
    RK(ensure(c, c->order_inv, sizeof(int) * (size_t)n));
    k_check_ids<<<(n + 255) / 256, 256, 0, st>>>(voxels, n, N, as<int>(c->err));
    CK(cudaMemcpyAsync(c->h_scalars, c->err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int bad = 0;
    std::memcpy(&bad, c->h_scalars, sizeof(int));
    if (bad) return fail(SOLAR_GPU_ERR_ARG, "voxel ids outside [0, %d)", N);
    DevScene ds = dev_scene(s);
    RK(padded_grid(c, s, sky, ds, st));
    CK(launch_trace(ds, as<DirEntry>(c->dirs), D, words32, 0, n, as<int>(c->raw),
                    as<uint32_t>(c->shadow), voxels, as<int>(c->err), st));
    const long long cells = (long long)n * words32;
    k_gather_shadow<<<(unsigned)((cells + 255) / 256), 256, 0, st>>>(as<uint32_t>(c->shadow), words32, voxels, n, out);
    CK(cudaGetLastError());
    return check_device_flags(c, st);
}

std::mutex g_default_mu;
solar_gpu_context* g_default = nullptr;

int drop_in(int fmt, const float* grid_data, int grid_width, int grid_height,
            int num_total_voxels, int num_top_voxels, const int* pixel_parent, const float* wall_z,
            float max_height, const float* sun_positions, int num_sun, const float* direct, int num_direct,
            const float* diffuse, int num_diffuse, const float* slopes, const float* aspects, float* out)
{
    // The reference reads the first 8760 entries of each series
    // (src/cuda/device_globals.cu:58-65); fewer is an error here.
    if (num_sun < kHoursPerYear || num_direct < kHoursPerYear || num_diffuse < kHoursPerYear)
        return fail(SOLAR_GPU_ERR_ARG, "hourly series need %d entries (got %d, %d, %d)",
                    kHoursPerYear, num_sun, num_direct, num_diffuse);
    std::lock_guard<std::mutex> lk(g_default_mu);
    if (!g_default) RK(solar_gpu_create(0, &g_default));
    solar_gpu_options o;
    solar_gpu_default_options(&o);
    o.neighbor_format = fmt;
    solar_gpu_scene s;
    s.grid = grid_data;
    s.grid_width = grid_width;
    s.grid_height = grid_height;
    s.num_total_voxels = num_total_voxels;
    s.num_top_voxels = num_top_voxels;
    s.pixel_parent = pixel_parent;
    s.wall_z = wall_z;
    s.max_height = max_height;
    s.sun_positions = sun_positions;
    s.direct_irradiance = direct;
    s.diffuse_irradiance = diffuse;
    s.slopes = slopes;
    s.aspects = aspects;
    return solar_gpu_run_host(g_default, &o, &s, out);
}

}  // namespace

extern "C" {

void solar_gpu_default_options(solar_gpu_options* o)
{
    if (!o) return;
    o->neighbor_format = SOLAR_GPU_CSR;
    o->hour_block = 256;
    o->accumulation = SOLAR_GPU_ACC_FP64;
    o->reflection = SOLAR_GPU_REFL_HOURLY;
    o->chunk_voxels = 0;
    o->use_graph = 1;
    o->time_kernels = 0;
    o->group_size = kMmaGroup;
}

const char* solar_gpu_last_error(void) { return g_err.c_str(); }

int solar_gpu_create(int device, solar_gpu_context** out)
{
    if (!out) return fail(SOLAR_GPU_ERR_ARG, "out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= 0) { cudaGetLastError(); return fail(SOLAR_GPU_ERR_NO_DEVICE, "no CUDA device"); }
    if (device < 0 || device >= n) return fail(SOLAR_GPU_ERR_ARG, "device %d of %d", device, n);
    CK(cudaSetDevice(device));
    solar_gpu_context* c = new solar_gpu_context();
    c->device = device;
    cudaError_t e1 = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
    for (int i = 0; i < 4 && e1 == cudaSuccess; ++i) e1 = cudaEventCreate(&c->ev[i]);
    if (e1 == cudaSuccess) e1 = cudaMallocHost((void**)&c->h_scalars, 64);
    size_t free_b = 0;
    if (e1 == cudaSuccess) e1 = cudaMemGetInfo(&free_b, &c->dev_total);
    if (e1 != cudaSuccess) { solar_gpu_destroy(c); return cuda_fail(e1, "context setup", __LINE__); }
    *out = c;
    return SOLAR_GPU_OK;
}


static void all_bufs(solar_gpu_context* c, DevBuf** out)
{
    DevBuf* bufs[kNumBufs] = {&c->dirs, &c->nudged, &c->dni, &c->dhi, &c->sun_dense, &c->hour_index, &c->table,
                      &c->geo_n, &c->geo_p, &c->shadow, &c->raw, &c->counts, &c->csr_off, &c->csr_ids,
                      &c->barle_off, &c->barle_sizes, &c->barle_bytes, &c->scan_tmp, &c->slab, &c->hourly,
                      &c->acc_f64, &c->acc_f32, &c->acc_comp, &c->sums, &c->out_f64, &c->err, &c->in_grid,
                      &c->in_pp, &c->in_wz, &c->in_slopes, &c->in_aspects, &c->out_f32, &c->order,
                      &c->order_cnt, &c->order_cur, &c->order_tmp, &c->grp_cnt, &c->grp_off,
                      &c->grp_tmp, &c->grp_cell, &c->grp_w, &c->w_cnt, &c->w_off, &c->w_tmp,
                      &c->w_cell, &c->w_val, &c->order_first, &c->order_inv,
                                &c->tile_flag, &c->tile_pos, &c->tile_start, &c->tile_union, &c->tile_slot,
                                &c->tile_rows, &c->tile_gcnt, &c->tile_gnch, &c->tile_gbase, &c->tile_tbase,
                                &c->tile_table, &c->tile_erow, &c->tile_ew, &c->chunk_perm, &c->chunk_flag,
                                &c->chunk_pos, &c->chunk_tmp, &c->mma_union, &c->mma_nch, &c->mma_cbase,
                                &c->mma_ccnt, &c->mma_coff, &c->mma_ent, &c->mma_scale, &c->mma_over, &c->slab16,
                                &c->dd_ovf, &c->vox_cnt, &c->vox_off, &c->vox_tmp, &c->gpad, &c->mma_sched, &c->mma_retry,
                                &c->cone, &c->cone_tmp, &c->cone_specs};
    for (int i = 0; i < kNumBufs; ++i) out[i] = bufs[i];
}

int solar_gpu_set_memory_limit(solar_gpu_context* c, long long bytes)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    if (bytes < 0) return fail(SOLAR_GPU_ERR_ARG, "memory limit must be >= 0");
    c->mem_limit = bytes;
    return SOLAR_GPU_OK;
}

long long solar_gpu_memory_held(solar_gpu_context* c)
{
    return c ? (long long)held_bytes(c) : 0;
}

int solar_gpu_release(solar_gpu_context* c)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    CK(cudaSetDevice(c->device));
    CK(cudaDeviceSynchronize());
    DevBuf* bufs[kNumBufs];
    all_bufs(c, bufs);
    for (DevBuf* b : bufs) {
        if (b->p) cudaFree(b->p);
        b->p = nullptr;
        b->cap = 0;
    }
    c->have_csr = c->have_barle = false;
    c->N = 0;
    c->timed = false;
    c->kt_used = 0;
    return SOLAR_GPU_OK;
}

void solar_gpu_destroy(solar_gpu_context* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->own) cudaStreamSynchronize(c->own);
    DevBuf* bufs[kNumBufs];
    all_bufs(c, bufs);
    for (DevBuf* b : bufs) if (b->p) cudaFree(b->p);
    for (int i = 0; i < 4; ++i) if (c->ev[i]) cudaEventDestroy(c->ev[i]);
    for (cudaEvent_t e : c->kt_pool) cudaEventDestroy(e);
    if (c->own) cudaStreamDestroy(c->own);
    if (c->h_scalars) cudaFreeHost(c->h_scalars);
    delete c;
}

int solar_gpu_run_device(solar_gpu_context* c, const solar_gpu_options* o, const solar_gpu_scene* s,
                         float* out, void* stream)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    cudaStream_t st = stream ? (cudaStream_t)stream : c->own;
    RK(run_device_impl(c, o, s, out, st, false));
    return check_device_flags(c, st);
}

int solar_gpu_run_batch(solar_gpu_context* const* ctxs, int n, const solar_gpu_options* opts,
                        const solar_gpu_scene* scenes, float* const* outs, void* stream)
{
    if (!ctxs || !scenes || !outs || !opts || n <= 0) return fail(SOLAR_GPU_ERR_ARG, "NULL argument or n <= 0");
    for (int i = 0; i < n; ++i) {
        if (!ctxs[i] || !outs[i]) return fail(SOLAR_GPU_ERR_ARG, "context or output %d is NULL", i);
        if (ctxs[i]->device != ctxs[0]->device) return fail(SOLAR_GPU_ERR_ARG, "contexts on different devices");
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == ctxs[i]) return fail(SOLAR_GPU_ERR_ARG, "context %d is given twice", i);
    }
    for (int i = 0; i < n; ++i)
        if (opts[i].hour_block == 1 || opts[i].reflection != SOLAR_GPU_REFL_HOURLY)
            return fail(SOLAR_GPU_ERR_ARG, "a batch runs the hour-block path (hour_block > 1, hourly reflection)");
    CK(cudaSetDevice(ctxs[0]->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : ctxs[0]->own;
    // Stage 1 and the once-per-run builds, tile after tile (each sizes its
    // buffers from its own lists); each stops before its hour loop.
    for (int i = 0; i < n; ++i) {
        solar_gpu_context* c = ctxs[i];
        solar_gpu_options ob = opts[i];
        ob.time_kernels = 0;
        c->defer_hours = true;
        c->cone_shared = &ctxs[0]->cone;   // one stream: tile i's tables are built after tile i - 1 is traced
        const int rc = run_device_impl(c, &ob, &scenes[i], outs[i], st, false);
        c->defer_hours = false;
        c->cone_shared = nullptr;
        if (rc != SOLAR_GPU_OK) return rc;
    }
    // One CUDA graph holds every tile's hour loop as a branch of its own (on
    // the tile context's stream, forked from and joined back into `st`), so
    // the small tiles' persistent kernels run side by side on the SMs.
    std::vector<cudaEvent_t> ev(n + 1, nullptr);
    cudaError_t le = cudaSuccess;
    for (int i = 0; i <= n && le == cudaSuccess; ++i) le = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool capturing = false;
    if (le == cudaSuccess) le = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (le == cudaSuccess) {
        capturing = true;
        le = cudaEventRecord(ev[n], st);
    }
    for (int i = 0; i < n && le == cudaSuccess; ++i) {
        solar_gpu_context* c = ctxs[i];
        le = cudaStreamWaitEvent(c->own, ev[n], 0);
        if (le == cudaSuccess) le = enqueue_hours(c, c->hours, c->own);
        if (le == cudaSuccess) le = cudaEventRecord(ev[i], c->own);
        if (le == cudaSuccess) le = cudaStreamWaitEvent(st, ev[i], 0);
    }
    if (capturing) {
        const cudaError_t ce = cudaStreamEndCapture(st, &graph);
        if (le == cudaSuccess) le = ce;
    }
    if (le == cudaSuccess) le = cudaGraphInstantiate(&exec, graph, 0);
    if (le == cudaSuccess) le = cudaGraphLaunch(exec, st);
    if (le == cudaSuccess) le = cudaStreamSynchronize(st);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (cudaEvent_t e : ev) if (e) cudaEventDestroy(e);
    CK(le);
    for (int i = 0; i < n; ++i) RK(check_device_flags(ctxs[i], st));
    return SOLAR_GPU_OK;
}

int solar_gpu_voxelize(solar_gpu_context* c, const float* grid, int W, int H, float voxel_size,
                       long long* num_total, int* pixel_parent, float* wall_z, float* slopes, float* aspects,
                       long long capacity, void* stream)
{
    if (!c || !grid || !num_total) return fail(SOLAR_GPU_ERR_ARG, "context, grid or num_total is NULL");
    if (W <= 0 || H <= 0 || (long long)W * H > 0x7FFFFFFFLL) return fail(SOLAR_GPU_ERR_ARG, "grid %d x %d", W, H);
    if (!(voxel_size > 0.0f)) return fail(SOLAR_GPU_ERR_ARG, "voxel_size must be > 0");
    CK(cudaSetDevice(c->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : c->own;
    const int T = W * H;
    RK(ensure(c, c->vox_cnt, sizeof(int) * (size_t)T));
    RK(ensure(c, c->vox_off, sizeof(long long) * ((size_t)T + 1)));
    RK(ensure(c, c->vox_tmp, sizeof(long long) * scan_scratch_elems(T)));
    CK(launch_vox_count(grid, W, H, voxel_size, as<int>(c->vox_cnt), st));
    CK(launch_scan_counts(as<int>(c->vox_cnt), T, 0, as<long long>(c->vox_off), as<long long>(c->vox_tmp), nullptr,
                          st));
    long long walls = 0;
    RK(read_ll(c, as<long long>(c->vox_off) + T, &walls, st));
    *num_total = (long long)T + walls;
    if (!pixel_parent && !slopes && !aspects) return SOLAR_GPU_OK;   // sizes only
    if (!pixel_parent || !slopes || !aspects || (walls > 0 && !wall_z))
        return fail(SOLAR_GPU_ERR_ARG, "an output array is NULL");
    if (capacity < *num_total) return fail(SOLAR_GPU_ERR_ARG, "capacity %lld < %lld voxels", capacity, *num_total);
    if (*num_total > 0x7FFFFFFFLL) return fail(SOLAR_GPU_ERR_ARG, "%lld voxels exceed the int32 voxel index", *num_total);
    // the cell size of the slope differences is the voxel size (src/main.cpp:103)
    CK(launch_vox_write(grid, W, H, voxel_size, voxel_size, as<long long>(c->vox_off), pixel_parent, wall_z, slopes,
                        aspects, st));
    CK(cudaStreamSynchronize(st));
    return SOLAR_GPU_OK;
}

int solar_gpu_run_lists(solar_gpu_context* c, const solar_gpu_options* o, const solar_gpu_scene* s,
                        const solar_gpu_lists* l, float* out, void* stream)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    return run_lists_impl(c, o, s, l, out, stream ? (cudaStream_t)stream : c->own);
}

int solar_gpu_trace_shadow_subset(solar_gpu_context* c, const solar_gpu_scene* s, const int* voxels, int n,
                                  uint32_t* shadow_out, int* shadow_words, void* stream)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    return trace_subset_impl(c, s, voxels, n, shadow_out, shadow_words, stream ? (cudaStream_t)stream : c->own);
}

int solar_gpu_run_host(solar_gpu_context* c, const solar_gpu_options* o, const solar_gpu_scene* s,
                       float* out)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    RK(check_scene(s));
    if (!out) return fail(SOLAR_GPU_ERR_ARG, "irradiance_out is NULL");
    CK(cudaSetDevice(c->device));
    cudaStream_t st = c->own;
    const size_t N = (size_t)s->num_total_voxels, T = (size_t)s->num_top_voxels, NW = N - T;
    RK(ensure(c, c->in_grid, sizeof(float) * T));
    RK(ensure(c, c->in_pp, sizeof(int) * N));
    RK(ensure(c, c->in_wz, sizeof(float) * (NW ? NW : 1)));
    RK(ensure(c, c->in_slopes, sizeof(float) * N));
    RK(ensure(c, c->in_aspects, sizeof(float) * N));
    RK(ensure(c, c->out_f32, sizeof(float) * N));
    CK(cudaMemcpyAsync(c->in_grid.p, s->grid, sizeof(float) * T, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->in_pp.p, s->pixel_parent, sizeof(int) * N, cudaMemcpyHostToDevice, st));
    if (NW) CK(cudaMemcpyAsync(c->in_wz.p, s->wall_z, sizeof(float) * NW, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->in_slopes.p, s->slopes, sizeof(float) * N, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->in_aspects.p, s->aspects, sizeof(float) * N, cudaMemcpyHostToDevice, st));
    solar_gpu_scene d = *s;
    d.grid = as<float>(c->in_grid);
    d.pixel_parent = as<int>(c->in_pp);
    d.wall_z = NW ? as<float>(c->in_wz) : nullptr;
    d.slopes = as<float>(c->in_slopes);
    d.aspects = as<float>(c->in_aspects);
    RK(run_device_impl(c, o, &d, as<float>(c->out_f32), st, false));
    CK(cudaMemcpyAsync(out, c->out_f32.p, sizeof(float) * N, cudaMemcpyDeviceToHost, st));
    return check_device_flags(c, st);
}

int solar_gpu_trace(solar_gpu_context* c, const solar_gpu_options* o, const solar_gpu_scene* s, void* stream)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    cudaStream_t st = stream ? (cudaStream_t)stream : c->own;
    RK(run_device_impl(c, o, s, nullptr, st, true));
    return check_device_flags(c, st);
}

int solar_gpu_trace_sizes(solar_gpu_context* c, long long* csr_entries, long long* barle_bytes,
                          int* shadow_words, int* active_bins, int* num_voxels)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    if (csr_entries) *csr_entries = c->have_csr ? c->csr_total : -1;
    if (barle_bytes) *barle_bytes = c->have_barle ? c->barle_total : -1;
    if (shadow_words) *shadow_words = c->words32;
    if (active_bins) *active_bins = c->active;
    if (num_voxels) *num_voxels = c->N;
    return SOLAR_GPU_OK;
}

int solar_gpu_trace_copy(solar_gpu_context* c, long long* csr_offsets, int* csr_ids,
                         long long* barle_offsets, unsigned char* barle_bytes, uint32_t* shadow)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    CK(cudaSetDevice(c->device));
    const size_t N = (size_t)c->N;
    if ((csr_offsets || csr_ids) && !c->have_csr) return fail(SOLAR_GPU_ERR_ARG, "no CSR lists in the last trace");
    if ((barle_offsets || barle_bytes) && !c->have_barle) return fail(SOLAR_GPU_ERR_ARG, "no ba-RLE lists in the last trace");
    CK(cudaStreamSynchronize(c->own));
    CK(cudaDeviceSynchronize());
    if (csr_offsets) CK(cudaMemcpy(csr_offsets, c->csr_off.p, sizeof(long long) * (N + 1), cudaMemcpyDeviceToHost));
    if (csr_ids && c->csr_total) CK(cudaMemcpy(csr_ids, c->csr_ids.p, sizeof(int) * (size_t)c->csr_total, cudaMemcpyDeviceToHost));
    if (barle_offsets) CK(cudaMemcpy(barle_offsets, c->barle_off.p, sizeof(long long) * (N + 1), cudaMemcpyDeviceToHost));
    if (barle_bytes && c->barle_total) CK(cudaMemcpy(barle_bytes, c->barle_bytes.p, (size_t)c->barle_total, cudaMemcpyDeviceToHost));
    if (shadow) CK(cudaMemcpy(shadow, c->shadow.p, sizeof(uint32_t) * N * c->words32, cudaMemcpyDeviceToHost));
    return SOLAR_GPU_OK;
}

int solar_gpu_trace_copy_range(solar_gpu_context* c, int v0, int v1, long long* csr_offsets, int* csr_ids,
                               long long* barle_offsets, unsigned char* barle_bytes, uint32_t* shadow)
{
    if (!c) return fail(SOLAR_GPU_ERR_ARG, "context is NULL");
    if (v0 < 0 || v1 < v0 || v1 > c->N) return fail(SOLAR_GPU_ERR_ARG, "voxel range outside [0, num_voxels]");
    CK(cudaSetDevice(c->device));
    if ((csr_offsets || csr_ids) && !c->have_csr) return fail(SOLAR_GPU_ERR_ARG, "no CSR lists in the last trace");
    if ((barle_offsets || barle_bytes) && !c->have_barle) return fail(SOLAR_GPU_ERR_ARG, "no ba-RLE lists in the last trace");
    CK(cudaStreamSynchronize(c->own));
    CK(cudaDeviceSynchronize());
    const size_t n = (size_t)(v1 - v0);
    long long a = 0, b = 0;
    if (csr_offsets || csr_ids) {
        CK(cudaMemcpy(&a, as<long long>(c->csr_off) + v0, sizeof(long long), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&b, as<long long>(c->csr_off) + v1, sizeof(long long), cudaMemcpyDeviceToHost));
        if (csr_offsets)
            CK(cudaMemcpy(csr_offsets, as<long long>(c->csr_off) + v0, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost));
        if (csr_ids && b > a)
            CK(cudaMemcpy(csr_ids, as<int>(c->csr_ids) + a, sizeof(int) * (size_t)(b - a), cudaMemcpyDeviceToHost));
    }
    if (barle_offsets || barle_bytes) {
        CK(cudaMemcpy(&a, as<long long>(c->barle_off) + v0, sizeof(long long), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&b, as<long long>(c->barle_off) + v1, sizeof(long long), cudaMemcpyDeviceToHost));
        if (barle_offsets)
            CK(cudaMemcpy(barle_offsets, as<long long>(c->barle_off) + v0, sizeof(long long) * (n + 1), cudaMemcpyDeviceToHost));
        if (barle_bytes && b > a)
            CK(cudaMemcpy(barle_bytes, as<unsigned char>(c->barle_bytes) + a, (size_t)(b - a), cudaMemcpyDeviceToHost));
    }
    if (shadow && n)
        CK(cudaMemcpy(shadow, as<uint32_t>(c->shadow) + (size_t)v0 * c->words32, sizeof(uint32_t) * n * c->words32,
                      cudaMemcpyDeviceToHost));
    return SOLAR_GPU_OK;
}

int solar_gpu_last_timings(solar_gpu_context* c, double* ms, int n)
{
    if (!c || !ms) return fail(SOLAR_GPU_ERR_ARG, "NULL argument");
    if (!c->timed) return 0;
    CK(cudaEventSynchronize(c->ev[3]));
    float t[4] = {0, 0, 0, 0};
    CK(cudaEventElapsedTime(&t[0], c->ev[0], c->ev[1]));
    CK(cudaEventElapsedTime(&t[1], c->ev[1], c->ev[2]));
    CK(cudaEventElapsedTime(&t[2], c->ev[2], c->ev[3]));
    CK(cudaEventElapsedTime(&t[3], c->ev[0], c->ev[3]));
    int k = n < 4 ? n : 4;
    for (int i = 0; i < k; ++i) ms[i] = t[i];
    return k;
}

long long solar_gpu_last_launch_count(solar_gpu_context* c) { return c ? c->launches : -1; }

long long solar_gpu_last_reflection_entries(solar_gpu_context* c) { return c ? c->group_entries : -1; }

long long solar_gpu_last_staged_rows(solar_gpu_context* c) { return c ? c->staged_rows : -1; }

long long solar_gpu_last_weighted_entries(solar_gpu_context* c) { return c ? c->weighted_entries : -1; }

int solar_gpu_kernel_times(solar_gpu_context* c, double* ms, long long* launches, int n)
{
    if (!c || !ms || !launches) return fail(SOLAR_GPU_ERR_ARG, "NULL argument");
    const int k = n < SOLAR_GPU_KT_COUNT ? n : SOLAR_GPU_KT_COUNT;
    for (int i = 0; i < k; ++i) { ms[i] = 0.0; launches[i] = 0; }
    if (c->kt_used == 0) return k;
    CK(cudaEventSynchronize(c->kt_pool[2 * (c->kt_used - 1) + 1]));
    for (int i = 0; i < c->kt_used; ++i) {
        float t = 0.0f;
        CK(cudaEventElapsedTime(&t, c->kt_pool[2 * i], c->kt_pool[2 * i + 1]));
        const int g = c->kt_ids[i];
        if (g < k) { ms[g] += t; launches[g] += 1; }
    }
    return k;
}

int solar_gpu_uncompressed_gpu_irradiance(
    const float* grid_data, int grid_width, int grid_height, int num_total_voxels, int num_top_voxels,
    const int* pixel_parent, const float* wall_z, float max_height,
    const float* sun_positions, int num_sun_positions, const float* direct_irradiance, int num_direct,
    const float* diffuse_irradiance, int num_diffuse, const float* slopes, const float* aspects,
    float* irradiance_out)
{
    return drop_in(SOLAR_GPU_CSR, grid_data, grid_width, grid_height, num_total_voxels, num_top_voxels,
                   pixel_parent, wall_z, max_height, sun_positions, num_sun_positions, direct_irradiance,
                   num_direct, diffuse_irradiance, num_diffuse, slopes, aspects, irradiance_out);
}

int solar_gpu_compressed_gpu_irradiance(
    const float* grid_data, int grid_width, int grid_height, int num_total_voxels, int num_top_voxels,
    const int* pixel_parent, const float* wall_z, float max_height,
    const float* sun_positions, int num_sun_positions, const float* direct_irradiance, int num_direct,
    const float* diffuse_irradiance, int num_diffuse, const float* slopes, const float* aspects,
    float* irradiance_out)
{
    return drop_in(SOLAR_GPU_BARLE, grid_data, grid_width, grid_height, num_total_voxels, num_top_voxels,
                   pixel_parent, wall_z, max_height, sun_positions, num_sun_positions, direct_irradiance,
                   num_direct, diffuse_irradiance, num_diffuse, slopes, aspects, irradiance_out);
}

}  // extern "C"
