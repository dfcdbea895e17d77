/*
 * CPU oracle for the SolarGPU annual irradiance path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the algorithm
 * of the reference pipeline so the CUDA product can be checked against it.
 * Only the test suite, the smoke check and the CPU-baseline leg of the
 * benchmark load it; the product library never links or calls it.
 *
 * Restated pieces (reference paths are relative to the SolarGPU tree):
 *   - sky bins                      src/sky_bins.cpp:9-52
 *   - hemisphere direction set      include/cuda/viewshed_stage.cuh:64-80
 *   - DDA viewshed + shadow bits    src/cuda/kernels/viewshed_kernels.cu:7-59
 *   - first-occurrence neighbor     viewshed_kernels.cu:49-55 with the CSR
 *     lists (CSR order)             consumer of gpu_irradiance_uncompressed.cu:84-94
 *   - ba-RLE encoder                src/barle_compression.cpp:12-187
 *   - ba-RLE decoder                src/cuda/kernels/reflection_kernels.cu:103-183
 *   - solar (direct + Perez)        src/cuda/kernels/solar_kernel.cu:8-77
 *   - reflection weights            reflection_kernels.cu:18-65
 *   - annual accumulation           solar_kernel.cu:79-85 (here in FP64)
 *
 * Float work that must be bit-exact (sky bins, directions, DDA) is done in
 * float with -ffp-contract=off; the one product that the CUDA build of the
 * reference fuses into an FMA (the ray height oz + Cdir.z * t) is selectable
 * by `fma_mode` so the choice can be checked against the reference kernel's
 * own output.  Irradiance is evaluated in double precision from the same
 * float inputs, with the reference's float constants taken at their float
 * values.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_HOURS 8760

/* ------------------------------------------------------------------ */
/* Sky bins: src/sky_bins.cpp:9-52                                     */
/* ------------------------------------------------------------------ */

/* sun_az_alt: [8760][2] float.  Outputs: full_to_dense [hsize*vsize],
   sun_dense_idx [8760], nudged [8760][2].  meta = {hsize, vsize,
   vsize_full, active_bin_count, hgrid_size_s (8-bit words per voxel)}. */
int orc_sky_bins(const float* sun_az_alt, float h_res, float v_res,
                 int* full_to_dense, int* sun_dense_idx, float* nudged, int* meta)
{
    unsigned hsize = (unsigned)ceilf(360.0f / h_res);
    unsigned vsize = (unsigned)ceilf(90.0f / v_res);
    unsigned char* used = (unsigned char*)calloc((size_t)hsize * vsize, 1);
    if (!used) return -1;
    for (int k = 0; k < ORC_HOURS; ++k) {
        float az = sun_az_alt[2 * k] - 1e-8f;
        float alt = sun_az_alt[2 * k + 1] - 1e-8f;
        nudged[2 * k] = az;
        nudged[2 * k + 1] = alt;
        if (alt < 1.0f) continue;
        unsigned bi = (unsigned)(az / h_res);
        unsigned bj = (unsigned)(alt / v_res);
        if (bi < hsize && bj < vsize) used[bi * vsize + bj] = 1;
    }
    int active = 0;
    for (unsigned i = 0; i < hsize; ++i)
        for (unsigned j = 0; j < vsize; ++j)
            full_to_dense[i * vsize + j] = used[i * vsize + j] ? active++ : -1;
    for (int k = 0; k < ORC_HOURS; ++k) {
        float az = nudged[2 * k], alt = nudged[2 * k + 1];
        if (alt < 1.0f) { sun_dense_idx[k] = -1; continue; }
        unsigned bi = (unsigned)(az / h_res);
        unsigned bj = (unsigned)(alt / v_res);
        sun_dense_idx[k] = (bi < hsize && bj < vsize) ? full_to_dense[bi * vsize + bj] : -1;
    }
    free(used);
    meta[0] = (int)hsize;
    meta[1] = (int)vsize;
    meta[2] = (int)(vsize * 2);
    meta[3] = active;
    meta[4] = (int)ceilf((float)active / 8.0f);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Direction set: include/cuda/viewshed_stage.cuh:64-80                */
/* ------------------------------------------------------------------ */

static const float kDegToRad = 0.0174532925f; /* include/pipeline_math_constants.h:15 */

/* dirs: [hsize*vsize_full][3]; dense: [..] (-1 for lower / unvisited);
   upper: [..].  Direction d = i * vsize_full + j. */
void orc_directions(int hsize, int vsize, float h_res, float v_res,
                    const int* full_to_dense, float* dirs, int* dense, int* upper)
{
    unsigned vfull = (unsigned)vsize * 2u;
    for (unsigned i = 0; i < (unsigned)hsize; ++i) {
        for (unsigned j = 0; j < vfull; ++j) {
            float cx, cy, cz;
            int is_up, dn = -1;
            if (j < (unsigned)vsize) {
                float e = (j + 0.5f) * v_res;
                cx = cosf(e * kDegToRad) * sinf(((i + 0.5f) * h_res) * kDegToRad);
                cy = -cosf(e * kDegToRad) * cosf(((i + 0.5f) * h_res) * kDegToRad);
                cz = sinf(e * kDegToRad);
                is_up = 1;
                dn = full_to_dense[i * (unsigned)vsize + j];
            } else {
                float e = (j - (unsigned)vsize + 0.5f) * v_res;
                cx = cosf(e * kDegToRad) * sinf(((i + 0.5f) * h_res) * kDegToRad);
                cy = -cosf(e * kDegToRad) * cosf(((i + 0.5f) * h_res) * kDegToRad);
                cz = -sinf(e * kDegToRad);
                is_up = 0;
            }
            float len = sqrtf(cx * cx + cy * cy + cz * cz);
            if (len > 0.0f) { cx /= len; cy /= len; cz /= len; }
            size_t d = (size_t)i * vfull + j;
            dirs[3 * d] = cx;
            dirs[3 * d + 1] = cy;
            dirs[3 * d + 2] = cz;
            dense[d] = dn;
            upper[d] = is_up;
        }
    }
}

/* ------------------------------------------------------------------ */
/* DDA viewshed: src/cuda/kernels/viewshed_kernels.cu:7-59             */
/* ------------------------------------------------------------------ */

typedef struct {
    const float* grid; int W, H;
    int num_total, num_top;
    const int* pix_parent; const float* wall_z;
    float maxz;
    const float* dirs; const int* dense; const int* upper; int D;
    int fma_mode;
} orc_scene;

/* Traces one ray from cell (gx, gy) at height base_z (the origin is the
   cell corner plus 2 * Cdir, viewshed_kernels.cu:27-29); returns the
   1-based hit cell id or 0. */
static int trace_ray_from(const orc_scene* s, int gx, int gy, float base_z, float cx, float cy, float cz,
                          int is_upper)
{
    /* Cdir * 2 is exact, so fused or not these three match. */
    float ox = (float)gx + cx * 2.0f;
    float oy = (float)gy + cy * 2.0f;
    float oz = base_z + cz * 2.0f;
    int ix = (int)floorf(ox);
    int iy = (int)floorf(oy);
    float ax = fmaxf(fabsf(cx), 1e-8f), ay = fmaxf(fabsf(cy), 1e-8f);
    float tMaxX = ((cx >= 0.0f) ? ((float)ix + 1.0f - ox) : (ox - (float)ix)) / ax;
    float tMaxY = ((cy >= 0.0f) ? ((float)iy + 1.0f - oy) : (oy - (float)iy)) / ay;
    float dX = 1.0f / ax, dY = 1.0f / ay;
    int sx = (cx >= 0.0f) ? 1 : -1, sy = (cy >= 0.0f) ? 1 : -1;
    float t = 0.0f;
    for (;;) {
        if (tMaxX < tMaxY) { t = tMaxX; ix += sx; tMaxX += dX; }
        else { t = tMaxY; iy += sy; tMaxY += dY; }
        if ((unsigned)ix >= (unsigned)s->W || (unsigned)iy >= (unsigned)s->H) return 0;
        float zr = s->fma_mode ? fmaf(cz, t, oz) : (oz + cz * t);
        if (is_upper && zr > s->maxz) return 0;
        if (!is_upper && zr < 0.0f) return 0;
        if (s->grid[ix + iy * s->W] - zr > 0.01f) return ix + iy * s->W + 1;
    }
}

/* Traces one ray of voxel t_id (viewshed_kernels.cu:15-25: a wall voxel
   starts at its parent column at wall_z). */
static int trace_ray(const orc_scene* s, int t_id, float cx, float cy, float cz, int is_upper)
{
    int top_id = s->pix_parent[t_id];
    int gx = top_id % s->W;
    int gy = top_id / s->W;
    float base_z = (t_id < s->num_top) ? s->grid[gx + gy * s->W] : s->wall_z[t_id - s->num_top];
    return trace_ray_from(s, gx, gy, base_z, cx, cy, cz, is_upper);
}

/* One ray over a bare heightmap (known-answer tests of the DDA). */
int orc_trace_one(const float* grid, int W, int H, float maxz, int gx, int gy, float base_z, float cx, float cy,
                  float cz, int is_upper, int fma_mode)
{
    orc_scene s;
    memset(&s, 0, sizeof s);
    s.grid = grid;
    s.W = W;
    s.H = H;
    s.maxz = maxz;
    s.fma_mode = fma_mode;
    return trace_ray_from(&s, gx, gy, base_z, cx, cy, cz, is_upper);
}

/* Per-voxel open-addressing set with generation stamps (dedupe helper). */
typedef struct { int* key; int* gen; int cur; } orc_set;

static int set_insert(orc_set* st, int key)
{
    unsigned h = ((unsigned)key * 2654435761u) >> 20; /* 12 bits */
    for (;;) {
        h &= 4095u;
        if (st->gen[h] != st->cur) { st->gen[h] = st->cur; st->key[h] = key; return 1; }
        if (st->key[h] == key) return 0;
        ++h;
    }
}

typedef struct {
    const orc_scene* s;
    int v0, v1;
    int* nb;        /* [v1-v0][D] first-occurrence lists */
    int* cnt;       /* [v1-v0] */
    uint32_t* shadow; int words32; /* [v1-v0][words32] */
    long long steps;
} trace_job;

static void* trace_worker(void* arg)
{
    trace_job* j = (trace_job*)arg;
    const orc_scene* s = j->s;
    orc_set st;
    st.key = (int*)malloc(4096 * sizeof(int));
    st.gen = (int*)calloc(4096, sizeof(int));
    st.cur = 0;
    for (int v = j->v0; v < j->v1; ++v) {
        size_t lv = (size_t)(v - j->v0);
        int* out = j->nb ? j->nb + lv * (size_t)s->D : NULL;
        uint32_t* sh = j->shadow ? j->shadow + lv * (size_t)j->words32 : NULL;
        if (sh) memset(sh, 0, sizeof(uint32_t) * (size_t)j->words32);
        ++st.cur;
        int n = 0;
        for (int d = 0; d < s->D; ++d) {
            int hit = trace_ray(s, v, s->dirs[3 * d], s->dirs[3 * d + 1], s->dirs[3 * d + 2], s->upper[d]);
            if (!hit) continue;
            if (sh && s->dense[d] >= 0) sh[s->dense[d] >> 5] |= 1u << (s->dense[d] & 31);
            if (set_insert(&st, hit)) { if (out) out[n] = hit; ++n; }
        }
        if (j->cnt) j->cnt[lv] = n;
    }
    free(st.key);
    free(st.gen);
    return NULL;
}

/* Traces voxels [v0, v1).  nb: [(v1-v0)][D] ints (may be NULL); cnt:
   [(v1-v0)]; shadow: [(v1-v0)][words32] u32 (bit b of word w = dense bin
   32w+b was hit, i.e. shadowed). */
int orc_trace(const float* grid, int W, int H, int num_total, int num_top,
              const int* pix_parent, const float* wall_z, float maxz,
              const float* dirs, const int* dense, const int* upper, int D,
              int v0, int v1, int* nb, int* cnt, uint32_t* shadow, int words32,
              int fma_mode, int nthreads)
{
    orc_scene s = { grid, W, H, num_total, num_top, pix_parent, wall_z, maxz,
                    dirs, dense, upper, D, fma_mode };
    if (nthreads < 1) nthreads = 1;
    int n = v1 - v0;
    if (n <= 0) return 0;
    if (nthreads > n) nthreads = n;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    trace_job* jobs = (trace_job*)malloc(sizeof(trace_job) * nthreads);
    for (int t = 0; t < nthreads; ++t) {
        int a = v0 + (int)((long long)n * t / nthreads);
        int b = v0 + (int)((long long)n * (t + 1) / nthreads);
        size_t off = (size_t)(a - v0);
        jobs[t].s = &s;
        jobs[t].v0 = a;
        jobs[t].v1 = b;
        jobs[t].nb = nb ? nb + off * (size_t)D : NULL;
        jobs[t].cnt = cnt ? cnt + off : NULL;
        jobs[t].shadow = shadow ? shadow + off * (size_t)words32 : NULL;
        jobs[t].words32 = words32;
        pthread_create(&th[t], NULL, trace_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th);
    free(jobs);
    return 0;
}

/* ------------------------------------------------------------------ */
/* ba-RLE encoder: src/barle_compression.cpp:12-187                     */
/* ------------------------------------------------------------------ */

enum { W4 = 0, W8 = 1, W16 = 2, W24 = 3, W32 = 4, END_OF_VOXEL = 7 };

typedef struct { int width, start, len; } orc_run;

static int width_class(unsigned x)
{
    if (x <= 15u) return W4;
    if (x <= 255u) return W8;
    if (x <= 65535u) return W16;
    if (x <= 16777215u) return W24;
    return W32;
}

static int cmp_desc(const void* a, const void* b)
{
    unsigned x = *(const unsigned*)a, y = *(const unsigned*)b;
    return (x < y) - (x > y);
}

/* Encodes one zero-terminated id list of at most n entries into out
   (capacity cap bytes).  Returns the byte count, or -1 if cap is too small. */
int orc_barle_encode(const int* raw, int n, uint8_t* out, int cap)
{
    unsigned* ids = (unsigned*)malloc(sizeof(unsigned) * (size_t)(n > 0 ? n : 1));
    int m = 0;
    for (int k = 0; k < n; ++k) { if (raw[k] == 0) break; ids[m++] = (unsigned)raw[k]; }
    if (m == 0) { free(ids); return 0; }
    qsort(ids, (size_t)m, sizeof(unsigned), cmp_desc);
    int u = 1;
    for (int k = 1; k < m; ++k) if (ids[k] != ids[u - 1]) ids[u++] = ids[k];
    m = u;
    if (ids[m - 1] == 0) --m;
    if (m == 0) { free(ids); return 0; }
    unsigned* delta = (unsigned*)malloc(sizeof(unsigned) * (size_t)m);
    delta[0] = ids[0];
    for (int k = 1; k < m; ++k) delta[k] = ids[k - 1] - ids[k];

    /* detect_runs (:90-105) */
    orc_run* runs = (orc_run*)malloc(sizeof(orc_run) * (size_t)m);
    orc_run* nxt = (orc_run*)malloc(sizeof(orc_run) * (size_t)m);
    int nr = 0;
    {
        int i = 0;
        while (i < m) {
            int w = width_class(delta[i]);
            int j = i + 1;
            while (j < m && width_class(delta[j]) == w) ++j;
            runs[nr].width = w; runs[nr].start = i; runs[nr].len = j - i; ++nr;
            i = j;
        }
    }
    /* optimize_runs (:112-152) */
    if (nr >= 2) {
        int changed = 1, done = 0;
        while (changed) {
            changed = 0;
            int nn = 0, i = 0;
            while (i < nr - 1) {
                if (runs[i + 1].len == 1 && runs[i + 1].width + 1 == runs[i].width) {
                    changed = 1;
                    nxt[nn] = runs[i]; nxt[nn].len++; ++nn;
                    i += 2;
                } else {
                    nxt[nn++] = runs[i];
                    ++i;
                }
            }
            if (i < nr) nxt[nn++] = runs[i];
            if (nn == 1) { runs[0] = nxt[0]; nr = 1; done = 1; break; }
            if (changed) { memcpy(runs, nxt, sizeof(orc_run) * (size_t)nn); nr = nn; }
        }
        if (!done) {
            int nn = 0, i = 0;
            while (i < nr) {
                orc_run mg = runs[i];
                int j = i + 1;
                while (j < nr && runs[j].width == mg.width) { mg.len += runs[j].len; ++j; }
                nxt[nn++] = mg;
                i = j;
            }
            memcpy(runs, nxt, sizeof(orc_run) * (size_t)nn);
            nr = nn;
        }
    }
    /* split_long_runs (:29-44) */
    int ns = 0;
    for (int r = 0; r < nr; ++r) ns += (runs[r].len + 254) / 255;
    orc_run* sp = (orc_run*)malloc(sizeof(orc_run) * (size_t)(ns > 0 ? ns : 1));
    ns = 0;
    for (int r = 0; r < nr; ++r) {
        int rem = runs[r].len, st = runs[r].start;
        while (rem > 255) { sp[ns].width = runs[r].width; sp[ns].start = st; sp[ns].len = 255; ++ns; st += 255; rem -= 255; }
        if (rem > 0) { sp[ns].width = runs[r].width; sp[ns].start = st; sp[ns].len = rem; ++ns; }
    }
    /* pack (:49-88, :180-185) */
    int pos = 0, ok = 1;
#define PUT(b) do { if (pos >= cap) { ok = 0; } else { out[pos] = (uint8_t)(b); } ++pos; } while (0)
    for (int base = 0; base < ns; base += 8) {
        uint32_t bits = 0;
        for (int j = 0; j < 8; ++j) {
            int code = (base + j < ns) ? sp[base + j].width : END_OF_VOXEL;
            bits |= (uint32_t)(code & 7) << ((7 - j) * 3);
        }
        PUT(bits >> 16); PUT(bits >> 8); PUT(bits);
        int cntb = ns - base < 8 ? ns - base : 8;
        for (int j = 0; j < cntb; ++j) PUT(sp[base + j].len);
        for (int j = 0; j < cntb; ++j) {
            int w = sp[base + j].width;
            unsigned p0 = (unsigned)sp[base + j].start, len = (unsigned)sp[base + j].len;
            for (unsigned k = 0; k < len;) {
                if (w == W4) {
                    unsigned v1 = delta[p0 + k];
                    unsigned v2 = (k + 1 < len) ? delta[p0 + k + 1] : 0u;
                    PUT((v1 << 4) | (v2 & 0x0Fu));
                    k += (k + 1 < len) ? 2u : 1u;
                } else {
                    unsigned x = delta[p0 + k];
                    for (int b = 0; b < w; ++b) PUT(x >> (8 * (w - 1 - b)));
                    ++k;
                }
            }
        }
    }
#undef PUT
    free(ids); free(delta); free(runs); free(nxt); free(sp);
    return ok ? pos : -1;
}

/* Encodes many lists: lists are CSR (offsets int64 [n+1], ids int32).
   Writes sizes[n]; if out != NULL also the concatenated bytes (capacity cap). */
long long orc_barle_encode_csr(const long long* off, const int* ids, int n,
                               long long* sizes, uint8_t* out, long long cap)
{
    uint8_t* tmp = (uint8_t*)malloc(1 << 16);
    long long pos = 0;
    for (int v = 0; v < n; ++v) {
        int len = (int)(off[v + 1] - off[v]);
        int b = orc_barle_encode(ids + off[v], len, tmp, 1 << 16);
        if (b < 0) { free(tmp); return -1; }
        sizes[v] = b;
        if (out) {
            if (pos + b > cap) { free(tmp); return -1; }
            memcpy(out + pos, tmp, (size_t)b);
        }
        pos += b;
    }
    free(tmp);
    return pos;
}

/* ------------------------------------------------------------------ */
/* ba-RLE decoder: reflection_kernels.cu:132-180                       */
/* ------------------------------------------------------------------ */

/* Decodes one voxel's byte range; writes every decoded value (the reference
   skips value 0 when accumulating).  Returns the count, -1 if the stream
   runs past `size`, -2 if more than `cap` values, -3 on a bad width code. */
int orc_barle_decode(const uint8_t* data, int size, unsigned* out, int cap)
{
    int idx = 0, n = 0;
    unsigned prev = 0;
    int first = 1;
    while (idx < size) {
        if (idx + 3 > size) return -1;
        uint32_t bits = ((uint32_t)data[idx] << 16) | ((uint32_t)data[idx + 1] << 8) | data[idx + 2];
        idx += 3;
        int widths[8], nc = 0;
        for (int j = 0; j < 8; ++j) {
            int code = (int)((bits >> (21 - 3 * j)) & 7u);
            if (code == END_OF_VOXEL) break;
            if (code > W32) return -3;
            widths[nc++] = code;
        }
        int lens[8];
        for (int j = 0; j < nc; ++j) { if (idx >= size) return -1; lens[j] = data[idx++]; }
        for (int j = 0; j < nc; ++j) {
            int w = widths[j], rl = lens[j];
            if (w == W4) {
                for (int i = 0; i < rl;) {
                    if (idx >= size) return -1;
                    unsigned packed = data[idx++];
                    unsigned hi = (packed >> 4) & 15u;
                    unsigned val = first ? hi : prev - hi;
                    first = 0; prev = val;
                    if (n >= cap) return -2;
                    out[n++] = val;
                    ++i;
                    if (i < rl) {
                        val = prev - (packed & 15u);
                        prev = val;
                        if (n >= cap) return -2;
                        out[n++] = val;
                        ++i;
                    }
                }
            } else {
                for (int i = 0; i < rl; ++i) {
                    if (idx + w > size) return -1;
                    unsigned dlt = 0;
                    for (int b = 0; b < w; ++b) dlt = (dlt << 8) | data[idx++];
                    unsigned val = first ? dlt : prev - dlt;
                    first = 0; prev = val;
                    if (n >= cap) return -2;
                    out[n++] = val;
                }
            }
        }
    }
    return n;
}

/* ------------------------------------------------------------------ */
/* FP64 irradiance: solar_kernel.cu:8-85, reflection_kernels.cu:18-65   */
/* ------------------------------------------------------------------ */

/* Reference constants at their float values. */
#define FC(x) ((double)(float)(x))
static const double kF[6][8] = { /* src/cuda/device_globals.cu:50-57 */
    { FC(-0.0083117), FC(0.1299457), FC(0.3296958), FC(0.5682053), FC(0.8730280), FC(1.1326077), FC(1.0601591), FC(0.6777470) },
    { FC(0.5877285), FC(0.6825954), FC(0.4868735), FC(0.1874525), FC(-0.3920403), FC(-1.2367284), FC(-1.5999137), FC(-0.3272588) },
    { FC(-0.0620636), FC(-0.1513752), FC(-0.2210958), FC(-0.2951290), FC(-0.3616149), FC(-0.4118494), FC(-0.3589221), FC(-0.2504286) },
    { FC(-0.0596012), FC(-0.0189325), FC(0.0554140), FC(0.1088631), FC(0.2255647), FC(0.2877813), FC(0.2642124), FC(0.1561313) },
    { FC(0.0721249), FC(0.0659650), FC(-0.0639588), FC(-0.1519229), FC(-0.4620442), FC(-0.8230357), FC(-1.1272340), FC(-1.3765031) },
    { FC(-0.0220216), FC(-0.0288748), FC(-0.0260542), FC(-0.0139754), FC(0.0012448), FC(0.0558651), FC(0.1310694), FC(0.2506212) },
};

/* Per daylight hour quantities (FP64). */
typedef struct {
    int hour;       /* 0..8759 */
    int dense;      /* sun bin, -1 if none */
    double cz, sz;  /* cos / sin of zenith */
    double caz, saz;/* cos / sin of azimuth */
    double dni, dni_eff, dhi;
    double F1, F2, b;
} orc_hour;

static double fmax_nan(double a, double b) { return fmax(a, b); }

/* Fills hours[] for every hour whose nudged altitude is >= 1 deg (the
   reference's daylight gate, gpu_irradiance_uncompressed.cu:117).  Returns
   the count. */
int orc_hour_table(const float* nudged, const int* sun_dense_idx, const float* dni,
                   const float* dhi, orc_hour* hours)
{
    const double kDeg = FC(0.0174532925);
    const double pi_f = FC(3.14159265358979323846);
    int n = 0;
    for (int k = 0; k < ORC_HOURS; ++k) {
        float alt = nudged[2 * k + 1];
        if (alt < 1.0f) continue;
        double az = nudged[2 * k];
        orc_hour* h = &hours[n++];
        h->hour = k;
        h->dense = sun_dense_idx[k];
        double cz = cos((90.0 - (double)alt) * kDeg);
        double z = acos(cz);
        h->cz = cz;
        h->sz = sin(z);
        h->caz = cos(az * kDeg);
        h->saz = sin(az * kDeg);
        double dn = dni[k], df = dhi[k];
        h->dni = dn;
        h->dni_eff = fmax_nan(dn, FC(1e-3));
        h->dhi = df;
        /* Perez (solar_kernel.cu:8-50); day index n = k / 24 */
        double z_deg = z * (180.0 / pi_f);
        double AM = 1.0 / (cz + FC(0.50572) * pow(FC(96.07995) - z_deg, FC(-1.6364)));
        double b = fmax_nan(FC(0.08715574), cz);
        double z3 = z * z * z;
        double eps = ((df + dn / cos(z)) / df + FC(1.041) * z3) / (1.0 + FC(1.041) * z3);
        double day = (double)(k / 24);
        double B = 2.0 * pi_f * (day / 365.0);
        double E0 = 1367.0 * (FC(1.00011) + FC(0.034221) * cos(B) + FC(0.00128) * sin(B)
                              + FC(0.000719) * cos(2 * B) + FC(0.000077) * sin(2 * B));
        double delta = (AM * df) / E0;
        eps = fmax_nan(1.0, eps);
        int e = 7;
        if (eps < FC(1.065)) e = 0;
        else if (eps < FC(1.230)) e = 1;
        else if (eps < FC(1.500)) e = 2;
        else if (eps < FC(1.950)) e = 3;
        else if (eps < FC(2.800)) e = 4;
        else if (eps < FC(4.500)) e = 5;
        else if (eps < FC(6.200)) e = 6;
        h->F1 = fmax_nan(0.0, kF[0][e] + kF[1][e] * delta + kF[2][e] * z);
        h->F2 = kF[3][e] + kF[4][e] * delta + kF[5][e] * z;
        h->b = b;
    }
    return n;
}

typedef struct {
    double cs, ss, ca, sa;        /* cos/sin slope, cos/sin aspect */
    double nx, ny, nz;            /* surface normal, reflection_kernels.cu:59-64 */
    double z; int gx, gy;
} orc_vox;

static void vox_geom(const orc_scene* s, const float* slopes, const float* aspects, int v, orc_vox* o)
{
    int top = s->pix_parent[v];
    o->gx = top % s->W;
    o->gy = top / s->W;
    o->z = (v < s->num_top) ? s->grid[o->gx + o->gy * s->W] : s->wall_z[v - s->num_top];
    double sl = slopes[v], as = aspects[v];
    o->cs = cos(sl); o->ss = sin(sl);
    o->ca = cos(as); o->sa = sin(as);
    o->nx = o->ss * o->sa;
    o->ny = -o->ss * o->ca;
    o->nz = o->cs;
}

/* Direct + diffuse of voxel geometry g at hour h (solar_kernel.cu:54-77). */
static double solar_I(const orc_vox* g, const orc_hour* h, int shadow_bit)
{
    /* cos(az - aspect) expanded */
    double caoi = h->cz * g->cs + h->sz * g->ss * (h->caz * g->ca + h->saz * g->sa);
    double I = 0.0;
    if (caoi > 0.0 && h->dense >= 0 && !shadow_bit)
        I += fmax_nan(0.0, h->dni_eff * caoi);
    double a = fmax_nan(0.0, caoi);
    double dif = h->dhi * ((1.0 - h->F1) * ((1.0 + g->cs) / 2.0) + h->F1 * (a / h->b) + h->F2 * g->ss);
    I += fmax_nan(0.0, dif);
    return I;
}

static double refl_w(const orc_scene* s, const orc_vox* me, int ngid)
{
    if (ngid < 0 || ngid >= s->W * s->H) return 0.0;
    int ngx = ngid % s->W, ngy = ngid / s->W;
    double dx = (double)(ngx - me->gx), dy = (double)(ngy - me->gy);
    double dz = (double)s->grid[ngid] - me->z;
    double d2 = dx * dx + dy * dy + dz * dz;
    if (d2 < FC(1e-4)) return 0.0;
    double d = sqrt(d2);
    double crecv = (me->nx * dx + me->ny * dy + me->nz * dz) / d;
    if (crecv <= 0.0) return 0.0;
    double csend = fmax_nan(fabs(dz) / d, FC(0.1));
    return FC(0.2) * crecv * csend / (FC(3.14159265) * d2);
}

static int bit_of(const uint32_t* shadow, int words32, int v, int dense)
{
    if (dense < 0) return 0;
    return (int)((shadow[(size_t)v * words32 + (dense >> 5)] >> (dense & 31)) & 1u);
}

typedef struct {
    const orc_scene* s;
    const float *slopes, *aspects;
    const orc_hour* hours; int nh;
    const uint32_t* shadow; int words32;
    const long long* off; const int* ids;
    const double* annual_top;  /* per top cell sum over hours of I (annual form) */
    int v0, v1;
    int per_hour;
    double* out;
    double* out_direct_diffuse;
    /* per-hour form scratch */
    const double* I_top_block; int hb0, hb1;
} irr_job;

static void* annual_top_worker(void* arg)
{
    irr_job* j = (irr_job*)arg;
    double* at = (double*)j->out;
    for (int v = j->v0; v < j->v1; ++v) {
        orc_vox g;
        vox_geom(j->s, j->slopes, j->aspects, v, &g);
        double acc = 0.0;
        for (int h = 0; h < j->nh; ++h)
            acc += solar_I(&g, &j->hours[h], bit_of(j->shadow, j->words32, v, j->hours[h].dense));
        at[v] = acc;
    }
    return NULL;
}

static void* annual_worker(void* arg)
{
    irr_job* j = (irr_job*)arg;
    for (int v = j->v0; v < j->v1; ++v) {
        orc_vox me;
        vox_geom(j->s, j->slopes, j->aspects, v, &me);
        double own;
        if (v < j->s->num_top) own = j->annual_top[v];
        else {
            own = 0.0;
            for (int h = 0; h < j->nh; ++h)
                own += solar_I(&me, &j->hours[h], bit_of(j->shadow, j->words32, v, j->hours[h].dense));
        }
        double r = 0.0;
        for (long long k = j->off[v]; k < j->off[v + 1]; ++k) {
            int ng = j->ids[k] - 1;
            double w = refl_w(j->s, &me, ng);
            if (w != 0.0) r += w * j->annual_top[ng];
        }
        j->out[v] = own + r;
        if (j->out_direct_diffuse) j->out_direct_diffuse[v] = own;
    }
    return NULL;
}

/* Annual FP64 irradiance per voxel, Wh/m^2.  Uses linearity of the
   reflection sum: sum_h sum_g w I(g,h) = sum_g w sum_h I(g,h), exact up to
   FP64 reassociation.  off/ids: first-occurrence CSR (1-based ids).
   out_dd (optional): the direct+diffuse part alone. */
int orc_annual_fp64(const float* grid, int W, int H, int num_total, int num_top,
                    const int* pix_parent, const float* wall_z,
                    const float* slopes, const float* aspects,
                    const float* sun_az_alt, const float* dni, const float* dhi,
                    const uint32_t* shadow, int words32,
                    const long long* off, const int* ids,
                    double* out, double* out_dd, int nthreads)
{
    int fd[72 * 18 + 64], meta[5];
    int* sdi = (int*)malloc(sizeof(int) * ORC_HOURS);
    float* nudged = (float*)malloc(sizeof(float) * 2 * ORC_HOURS);
    orc_hour* hours = (orc_hour*)malloc(sizeof(orc_hour) * ORC_HOURS);
    orc_sky_bins(sun_az_alt, 5.0f, 5.0f, fd, sdi, nudged, meta);
    int nh = orc_hour_table(nudged, sdi, dni, dhi, hours);
    orc_scene s = { grid, W, H, num_total, num_top, pix_parent, wall_z, 0.0f, NULL, NULL, NULL, 0, 1 };
    double* at = (double*)malloc(sizeof(double) * (size_t)num_top);
    if (nthreads < 1) nthreads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    irr_job* jobs = (irr_job*)calloc((size_t)nthreads, sizeof(irr_job));
    for (int pass = 0; pass < 2; ++pass) {
        int n = pass == 0 ? num_top : num_total;
        for (int t = 0; t < nthreads; ++t) {
            irr_job* j = &jobs[t];
            j->s = &s; j->slopes = slopes; j->aspects = aspects;
            j->hours = hours; j->nh = nh; j->shadow = shadow; j->words32 = words32;
            j->off = off; j->ids = ids; j->annual_top = at;
            j->v0 = (int)((long long)n * t / nthreads);
            j->v1 = (int)((long long)n * (t + 1) / nthreads);
            j->out = pass == 0 ? at : out;
            j->out_direct_diffuse = out_dd;
            pthread_create(&th[t], NULL, pass == 0 ? annual_top_worker : annual_worker, j);
        }
        for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    }
    free(th); free(jobs); free(at); free(sdi); free(nudged); free(hours);
    return nh;
}

/* ------------------------------------------------------------------ */
/* Per-hour FP64 method (the CPU baseline): for each voxel and daylight  */
/* hour, direct + diffuse plus the neighbor sum sum_g w(v,g) I(g,h).     */
/* I(g,h) for the top cells is tabulated per block of hours.             */
/* ------------------------------------------------------------------ */

static void* hourly_top_worker(void* arg)
{
    irr_job* j = (irr_job*)arg;
    int hb = j->hb1 - j->hb0;
    double* I = (double*)j->I_top_block;
    for (int v = j->v0; v < j->v1; ++v) {
        orc_vox g;
        vox_geom(j->s, j->slopes, j->aspects, v, &g);
        for (int h = j->hb0; h < j->hb1; ++h)
            I[(size_t)v * hb + (h - j->hb0)] = solar_I(&g, &j->hours[h], bit_of(j->shadow, j->words32, v, j->hours[h].dense));
    }
    return NULL;
}

static void* hourly_worker(void* arg)
{
    irr_job* j = (irr_job*)arg;
    int hb = j->hb1 - j->hb0;
    double* acc = (double*)malloc(sizeof(double) * (size_t)hb);
    for (int v = j->v0; v < j->v1; ++v) {
        orc_vox me;
        vox_geom(j->s, j->slopes, j->aspects, v, &me);
        for (int h = 0; h < hb; ++h)
            acc[h] = solar_I(&me, &j->hours[j->hb0 + h], bit_of(j->shadow, j->words32, v, j->hours[j->hb0 + h].dense));
        for (long long k = j->off[v]; k < j->off[v + 1]; ++k) {
            int ng = j->ids[k] - 1;
            double w = refl_w(j->s, &me, ng);
            if (w == 0.0) continue;
            const double* row = j->I_top_block + (size_t)ng * hb;
            for (int h = 0; h < hb; ++h) acc[h] += w * row[h];
        }
        double sum = 0.0;
        for (int h = 0; h < hb; ++h) sum += acc[h];
        j->out[v] += sum;
    }
    free(acc);
    return NULL;
}

/* Per-hour FP64 annual irradiance for voxels [v0, v1) (out has v1-v0
   entries).  Needs the shadow words of every top cell (neighbors) and of
   the voxels in range.  Hours are processed in blocks of `hblock`. */
int orc_hourly_fp64(const float* grid, int W, int H, int num_total, int num_top,
                    const int* pix_parent, const float* wall_z,
                    const float* slopes, const float* aspects,
                    const float* sun_az_alt, const float* dni, const float* dhi,
                    const uint32_t* shadow, int words32,
                    const long long* off, const int* ids,
                    int v0, int v1, int hblock, double* out, int nthreads)
{
    int fd[72 * 18 + 64], meta[5];
    int* sdi = (int*)malloc(sizeof(int) * ORC_HOURS);
    float* nudged = (float*)malloc(sizeof(float) * 2 * ORC_HOURS);
    orc_hour* hours = (orc_hour*)malloc(sizeof(orc_hour) * ORC_HOURS);
    orc_sky_bins(sun_az_alt, 5.0f, 5.0f, fd, sdi, nudged, meta);
    int nh = orc_hour_table(nudged, sdi, dni, dhi, hours);
    orc_scene s = { grid, W, H, num_total, num_top, pix_parent, wall_z, 0.0f, NULL, NULL, NULL, 0, 1 };
    if (hblock < 1) hblock = 64;
    double* Itop = (double*)malloc(sizeof(double) * (size_t)num_top * (size_t)hblock);
    double* res = (double*)calloc((size_t)num_total, sizeof(double));
    if (nthreads < 1) nthreads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    irr_job* jobs = (irr_job*)calloc((size_t)nthreads, sizeof(irr_job));
    for (int h0 = 0; h0 < nh; h0 += hblock) {
        int h1 = h0 + hblock < nh ? h0 + hblock : nh;
        for (int pass = 0; pass < 2; ++pass) {
            int a0 = pass == 0 ? 0 : v0, a1 = pass == 0 ? num_top : v1;
            int n = a1 - a0;
            for (int t = 0; t < nthreads; ++t) {
                irr_job* j = &jobs[t];
                j->s = &s; j->slopes = slopes; j->aspects = aspects;
                j->hours = hours; j->nh = nh; j->shadow = shadow; j->words32 = words32;
                j->off = off; j->ids = ids;
                j->v0 = a0 + (int)((long long)n * t / nthreads);
                j->v1 = a0 + (int)((long long)n * (t + 1) / nthreads);
                j->out = res;
                j->I_top_block = Itop; j->hb0 = h0; j->hb1 = h1;
                pthread_create(&th[t], NULL, pass == 0 ? hourly_top_worker : hourly_worker, j);
            }
            for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
        }
    }
    for (int v = v0; v < v1; ++v) out[v - v0] = res[v];
    free(th); free(jobs); free(Itop); free(res); free(sdi); free(nudged); free(hours);
    return nh;
}

/* Exposes the hour table for tests: writes per daylight hour
   [hour, dense, cz, sz, caz, saz, dni_eff, dhi, F1, F2, b] as doubles. */
int orc_hour_table_dump(const float* sun_az_alt, const float* dni, const float* dhi, double* out)
{
    int fd[72 * 18 + 64], meta[5];
    int* sdi = (int*)malloc(sizeof(int) * ORC_HOURS);
    float* nudged = (float*)malloc(sizeof(float) * 2 * ORC_HOURS);
    orc_hour* hours = (orc_hour*)malloc(sizeof(orc_hour) * ORC_HOURS);
    orc_sky_bins(sun_az_alt, 5.0f, 5.0f, fd, sdi, nudged, meta);
    int nh = orc_hour_table(nudged, sdi, dni, dhi, hours);
    for (int i = 0; i < nh; ++i) {
        double* o = out + 11 * (size_t)i;
        o[0] = hours[i].hour; o[1] = hours[i].dense; o[2] = hours[i].cz; o[3] = hours[i].sz;
        o[4] = hours[i].caz; o[5] = hours[i].saz; o[6] = hours[i].dni_eff; o[7] = hours[i].dhi;
        o[8] = hours[i].F1; o[9] = hours[i].F2; o[10] = hours[i].b;
    }
    free(sdi); free(nudged); free(hours);
    return nh;
}

/* ------------------------------------------------------------------ */
/* CPU baseline sample: times the FP64 method on a bounded sample of a   */
/* scene.  Stage 1 = full 2592-direction trace + dedupe of `ns` sampled  */
/* voxels; Stage 2/3 = one block of `hblock` daylight hours: the top-cell */
/* solar table for all T cells, then the per-hour reflection sums of the */
/* sampled voxels.  Returns wall seconds in times[0..2] = {trace, table, */
/* voxel sums}; the caller scales them to the whole workload.            */
/* ------------------------------------------------------------------ */

#include <time.h>

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

typedef struct {
    const orc_scene* s;
    const int* sample; int a, b;
    int* nb; int* cnt; uint32_t* sh; int words32;
} sample_job;

static void* sample_trace_worker(void* arg)
{
    sample_job* j = (sample_job*)arg;
    const orc_scene* s = j->s;
    orc_set st;
    st.key = (int*)malloc(4096 * sizeof(int));
    st.gen = (int*)calloc(4096, sizeof(int));
    st.cur = 0;
    for (int i = j->a; i < j->b; ++i) {
        int v = j->sample[i];
        int* out = j->nb ? j->nb + (size_t)i * s->D : NULL;
        uint32_t* sh = j->sh + (size_t)i * j->words32;
        memset(sh, 0, sizeof(uint32_t) * (size_t)j->words32);
        ++st.cur;
        int n = 0;
        for (int d = 0; d < s->D; ++d) {
            int hit = trace_ray(s, v, s->dirs[3 * d], s->dirs[3 * d + 1], s->dirs[3 * d + 2], s->upper[d]);
            if (!hit) continue;
            if (s->dense[d] >= 0) sh[s->dense[d] >> 5] |= 1u << (s->dense[d] & 31);
            if (set_insert(&st, hit)) { if (out) out[n] = hit; ++n; }
        }
        if (j->cnt) j->cnt[i] = n;
    }
    free(st.key); free(st.gen);
    return NULL;
}

typedef struct {
    const orc_scene* s; const float *slopes, *aspects;
    const orc_hour* hours; int h0, h1;
    double* Itop; int a, b;
    const int* sample; const int* nb; const int* cnt; const uint32_t* sh; int words32;
    double* out;
} sample_irr_job;

static void* sample_table_worker(void* arg)
{
    sample_irr_job* j = (sample_irr_job*)arg;
    int hb = j->h1 - j->h0;
    for (int g = j->a; g < j->b; ++g) {
        orc_vox gv;
        vox_geom(j->s, j->slopes, j->aspects, g, &gv);
        for (int h = j->h0; h < j->h1; ++h)
            j->Itop[(size_t)g * hb + (h - j->h0)] = solar_I(&gv, &j->hours[h], 0);
    }
    return NULL;
}

static void* sample_sum_worker(void* arg)
{
    sample_irr_job* j = (sample_irr_job*)arg;
    int hb = j->h1 - j->h0;
    double* acc = (double*)malloc(sizeof(double) * (size_t)hb);
    for (int i = j->a; i < j->b; ++i) {
        int v = j->sample[i];
        orc_vox me;
        vox_geom(j->s, j->slopes, j->aspects, v, &me);
        for (int h = 0; h < hb; ++h)
            acc[h] = solar_I(&me, &j->hours[j->h0 + h], bit_of(j->sh, j->words32, i, j->hours[j->h0 + h].dense));
        const int* l = j->nb + (size_t)i * j->s->D;
        for (int k = 0; k < j->cnt[i]; ++k) {
            double w = refl_w(j->s, &me, l[k] - 1);
            if (w == 0.0) continue;
            const double* row = j->Itop + (size_t)(l[k] - 1) * hb;
            for (int h = 0; h < hb; ++h) acc[h] += w * row[h];
        }
        double sum = 0.0;
        for (int h = 0; h < hb; ++h) sum += acc[h];
        j->out[i] = sum;
    }
    free(acc);
    return NULL;
}

int orc_cpu_sample(const float* grid, int W, int H, int num_total, int num_top,
                   const int* pix_parent, const float* wall_z, float maxz,
                   const float* slopes, const float* aspects,
                   const float* sun_az_alt, const float* dni, const float* dhi,
                   const int* sample, int ns, int hblock, int nthreads, double* times)
{
    int fd[72 * 18 + 64], meta[5];
    int* sdi = (int*)malloc(sizeof(int) * ORC_HOURS);
    float* nudged = (float*)malloc(sizeof(float) * 2 * ORC_HOURS);
    orc_hour* hours = (orc_hour*)malloc(sizeof(orc_hour) * ORC_HOURS);
    orc_sky_bins(sun_az_alt, 5.0f, 5.0f, fd, sdi, nudged, meta);
    int nh = orc_hour_table(nudged, sdi, dni, dhi, hours);
    int D = meta[0] * meta[2];
    float* dirs = (float*)malloc(sizeof(float) * 3 * D);
    int* dense = (int*)malloc(sizeof(int) * D);
    int* upper = (int*)malloc(sizeof(int) * D);
    orc_directions(meta[0], meta[1], 5.0f, 5.0f, fd, dirs, dense, upper);
    int words32 = (meta[3] + 31) / 32;
    if (words32 < 1) words32 = 1;
    orc_scene s = { grid, W, H, num_total, num_top, pix_parent, wall_z, maxz, dirs, dense, upper, D, 1 };
    if (nthreads < 1) nthreads = 1;
    if (hblock > nh) hblock = nh;
    int* nb = (int*)malloc(sizeof(int) * (size_t)ns * D);
    int* cnt = (int*)malloc(sizeof(int) * (size_t)ns);
    uint32_t* sh = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)ns * words32);
    double* Itop = (double*)malloc(sizeof(double) * (size_t)num_top * (size_t)hblock);
    double* out = (double*)malloc(sizeof(double) * (size_t)ns);
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    sample_job* tj = (sample_job*)calloc((size_t)nthreads, sizeof(sample_job));
    sample_irr_job* ij = (sample_irr_job*)calloc((size_t)nthreads, sizeof(sample_irr_job));

    double t0 = now_s();
    for (int t = 0; t < nthreads; ++t) {
        tj[t].s = &s; tj[t].sample = sample;
        tj[t].a = (int)((long long)ns * t / nthreads); tj[t].b = (int)((long long)ns * (t + 1) / nthreads);
        tj[t].nb = nb; tj[t].cnt = cnt; tj[t].sh = sh; tj[t].words32 = words32;
        pthread_create(&th[t], NULL, sample_trace_worker, &tj[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    double t1 = now_s();
    for (int pass = 0; pass < 2; ++pass) {
        int n = pass == 0 ? num_top : ns;
        for (int t = 0; t < nthreads; ++t) {
            sample_irr_job* j = &ij[t];
            j->s = &s; j->slopes = slopes; j->aspects = aspects; j->hours = hours;
            j->h0 = 0; j->h1 = hblock; j->Itop = Itop;
            j->a = (int)((long long)n * t / nthreads); j->b = (int)((long long)n * (t + 1) / nthreads);
            j->sample = sample; j->nb = nb; j->cnt = cnt; j->sh = sh; j->words32 = words32; j->out = out;
            pthread_create(&th[t], NULL, pass == 0 ? sample_table_worker : sample_sum_worker, j);
        }
        for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
        if (pass == 0) times[1] = now_s() - t1;
    }
    times[0] = t1 - t0;
    times[2] = now_s() - t1 - times[1];
    free(th); free(tj); free(ij); free(nb); free(cnt); free(sh); free(Itop); free(out);
    free(dirs); free(dense); free(upper); free(sdi); free(nudged); free(hours);
    return nh;
}

/* Step counts of every (voxel, direction) ray, for studying lane grouping of
   the GPU tracer.  steps: [(v1-v0)][D] (int16, saturating). */
static int trace_ray_steps(const orc_scene* s, int t_id, float cx, float cy, float cz, int is_upper)
{
    int top_id = s->pix_parent[t_id];
    int gx = top_id % s->W, gy = top_id / s->W;
    float base_z = (t_id < s->num_top) ? s->grid[gx + gy * s->W] : s->wall_z[t_id - s->num_top];
    float ox = (float)gx + cx * 2.0f, oy = (float)gy + cy * 2.0f, oz = base_z + cz * 2.0f;
    int ix = (int)floorf(ox), iy = (int)floorf(oy);
    float ax = fmaxf(fabsf(cx), 1e-8f), ay = fmaxf(fabsf(cy), 1e-8f);
    float tMaxX = ((cx >= 0.0f) ? ((float)ix + 1.0f - ox) : (ox - (float)ix)) / ax;
    float tMaxY = ((cy >= 0.0f) ? ((float)iy + 1.0f - oy) : (oy - (float)iy)) / ay;
    float dX = 1.0f / ax, dY = 1.0f / ay;
    int sx = (cx >= 0.0f) ? 1 : -1, sy = (cy >= 0.0f) ? 1 : -1;
    int n = 0;
    for (;;) {
        float t;
        ++n;
        if (tMaxX < tMaxY) { t = tMaxX; ix += sx; tMaxX += dX; } else { t = tMaxY; iy += sy; tMaxY += dY; }
        if ((unsigned)ix >= (unsigned)s->W || (unsigned)iy >= (unsigned)s->H) return n;
        float zr = fmaf(cz, t, oz);
        if (is_upper && zr > s->maxz) return n;
        if (!is_upper && zr < 0.0f) return n;
        if (s->grid[ix + iy * s->W] - zr > 0.01f) return n;
    }
}

int orc_trace_steps(const float* grid, int W, int H, int num_total, int num_top,
                    const int* pix_parent, const float* wall_z, float maxz,
                    const float* dirs, const int* dense, const int* upper, int D,
                    const int* voxels, int nv, short* steps)
{
    orc_scene s = { grid, W, H, num_total, num_top, pix_parent, wall_z, maxz, dirs, dense, upper, D, 1 };
    for (int i = 0; i < nv; ++i)
        for (int d = 0; d < D; ++d) {
            int n = trace_ray_steps(&s, voxels[i], dirs[3 * d], dirs[3 * d + 1], dirs[3 * d + 2], upper[d]);
            steps[(size_t)i * D + d] = (short)(n > 32767 ? 32767 : n);
        }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Sampled checks for scenes too large for a full CPU pass: Stage 1 of  */
/* an arbitrary voxel list, and the FP64 annual irradiance of a voxel   */
/* sample computed from oracle-built lists and shadow words.            */
/* ------------------------------------------------------------------ */

/* Traces the listed voxels (any order) exactly as orc_trace traces each
   one: nb [n][D] first-occurrence lists (may be NULL), cnt [n] (may be
   NULL), shadow [n][words32]. */
int orc_trace_list(const float* grid, int W, int H, int num_total, int num_top,
                   const int* pix_parent, const float* wall_z, float maxz,
                   const float* dirs, const int* dense, const int* upper, int D,
                   const int* voxels, int n, int* nb, int* cnt, uint32_t* shadow, int words32,
                   int fma_mode, int nthreads)
{
    orc_scene s = { grid, W, H, num_total, num_top, pix_parent, wall_z, maxz,
                    dirs, dense, upper, D, fma_mode };
    if (n <= 0) return 0;
    for (int i = 0; i < n; ++i)
        if (voxels[i] < 0 || voxels[i] >= num_total) return -1;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > n) nthreads = n;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    sample_job* tj = (sample_job*)calloc((size_t)nthreads, sizeof(sample_job));
    for (int t = 0; t < nthreads; ++t) {
        tj[t].s = &s; tj[t].sample = voxels;
        tj[t].a = (int)((long long)n * t / nthreads); tj[t].b = (int)((long long)n * (t + 1) / nthreads);
        tj[t].nb = nb; tj[t].cnt = cnt; tj[t].sh = shadow; tj[t].words32 = words32;
        pthread_create(&th[t], NULL, sample_trace_worker, &tj[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th); free(tj);
    return 0;
}

typedef struct {
    const orc_scene* s; const float *slopes, *aspects;
    const orc_hour* hours; int nh; int words32;
    const int* cells; int nc; const uint32_t* csh; double* at;   /* per listed top cell */
    const int* sample; const uint32_t* sh; const long long* off; const int* ids;
    int a, b; double* out; int missing;
} subset_job;

static void* subset_cell_worker(void* arg)
{
    subset_job* j = (subset_job*)arg;
    for (int c = j->a; c < j->b; ++c) {
        orc_vox g;
        vox_geom(j->s, j->slopes, j->aspects, j->cells[c], &g);
        double acc = 0.0;
        for (int h = 0; h < j->nh; ++h)
            acc += solar_I(&g, &j->hours[h], bit_of(j->csh, j->words32, c, j->hours[h].dense));
        j->at[c] = acc;
    }
    return NULL;
}

static int find_cell(const int* cells, int nc, int x)
{
    int lo = 0, hi = nc - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if (cells[mid] == x) return mid;
        if (cells[mid] < x) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

static void* subset_voxel_worker(void* arg)
{
    subset_job* j = (subset_job*)arg;
    for (int i = j->a; i < j->b; ++i) {
        orc_vox me;
        vox_geom(j->s, j->slopes, j->aspects, j->sample[i], &me);
        double own = 0.0;
        for (int h = 0; h < j->nh; ++h)
            own += solar_I(&me, &j->hours[h], bit_of(j->sh, j->words32, i, j->hours[h].dense));
        double r = 0.0;
        for (long long k = j->off[i]; k < j->off[i + 1]; ++k) {
            int ng = j->ids[k] - 1;
            double w = refl_w(j->s, &me, ng);
            if (w == 0.0) continue;
            int c = find_cell(j->cells, j->nc, ng);
            if (c < 0) { j->missing = 1; continue; }
            r += w * j->at[c];
        }
        j->out[i] = own + r;
    }
    return NULL;
}

/* FP64 annual irradiance (Wh/m^2, the annual-sum form of orc_annual_fp64)
   of the voxels sample[ns], from their first-occurrence lists (off [ns+1]
   from 0, ids 1-based cells) and shadow words sh [ns][words32], given the
   shadow words csh [nc][words32] of every top cell the lists name (cells
   [nc], ascending).  out [ns].  Returns the daylight hour count, or -1 if a
   list names a cell missing from `cells`. */
int orc_annual_fp64_sample(const float* grid, int W, int H, int num_total, int num_top,
                           const int* pix_parent, const float* wall_z,
                           const float* slopes, const float* aspects,
                           const float* sun_az_alt, const float* dni, const float* dhi,
                           const int* sample, int ns, const uint32_t* sh, const long long* off, const int* ids,
                           const int* cells, int nc, const uint32_t* csh, int words32,
                           double* out, int nthreads)
{
    int fd[72 * 18 + 64], meta[5];
    int* sdi = (int*)malloc(sizeof(int) * ORC_HOURS);
    float* nudged = (float*)malloc(sizeof(float) * 2 * ORC_HOURS);
    orc_hour* hours = (orc_hour*)malloc(sizeof(orc_hour) * ORC_HOURS);
    orc_sky_bins(sun_az_alt, 5.0f, 5.0f, fd, sdi, nudged, meta);
    int nh = orc_hour_table(nudged, sdi, dni, dhi, hours);
    orc_scene s = { grid, W, H, num_total, num_top, pix_parent, wall_z, 0.0f, NULL, NULL, NULL, 0, 1 };
    double* at = (double*)malloc(sizeof(double) * (size_t)(nc > 0 ? nc : 1));
    if (nthreads < 1) nthreads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
    subset_job* jobs = (subset_job*)calloc((size_t)nthreads, sizeof(subset_job));
    int missing = 0;
    for (int pass = 0; pass < 2; ++pass) {
        int n = pass == 0 ? nc : ns;
        for (int t = 0; t < nthreads; ++t) {
            subset_job* j = &jobs[t];
            j->s = &s; j->slopes = slopes; j->aspects = aspects; j->hours = hours; j->nh = nh;
            j->words32 = words32; j->cells = cells; j->nc = nc; j->csh = csh; j->at = at;
            j->sample = sample; j->sh = sh; j->off = off; j->ids = ids; j->out = out; j->missing = 0;
            j->a = (int)((long long)n * t / nthreads);
            j->b = (int)((long long)n * (t + 1) / nthreads);
            pthread_create(&th[t], NULL, pass == 0 ? subset_cell_worker : subset_voxel_worker, j);
        }
        for (int t = 0; t < nthreads; ++t) {
            pthread_join(th[t], NULL);
            missing |= jobs[t].missing;
        }
    }
    free(th); free(jobs); free(at); free(sdi); free(nudged); free(hours);
    return missing ? -1 : nh;
}
