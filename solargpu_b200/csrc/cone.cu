// Early-exit bounds for upward rays of the tracer.
//
// The reference ends an upward ray when its height passes the scene maximum
// (viewshed_kernels.cu:42).  A ray that is already above every cell it can
// still reach cannot hit anything either, so it may end there with the same
// result.  For each group of directions this file builds one table over the
// bordered grid,
//
//     bound[cell] = min(maxz, max of the heights of every cell a ray of the
//                   group can visit from `cell` on),
//
// and the tracer ends an upward ray with no hit when its height exceeds the
// bound of a cell it has reached (it loads the bound of the cell a group of
// steps starts on and compares it with the height at the group's end, every
// cell after that being reachable from the first).  The result is the
// reference's, bit for bit:
//   * upward rays only rise (t never decreases, cz > 0, and the fused
//     multiply-add is monotone in t), so every later height test compares a
//     cell height <= bound with a ray height > bound and fails;
//   * bound <= maxz, so a ray the reference ends on the range test ends here
//     too, and the tracer checks the range test first after the loop.
//
// Which cells a ray can still visit.  Work in the quadrant's unsigned
// coordinates (X grows along the ray's x step, Y along its y step).  The DDA
// adds dX and dY (floats) to its crossing times; without rounding its cells
// are exactly the cells a straight line of direction (1/dX, 1/dY) passes
// through.  After i additions a crossing time is off by at most i * 2^-24 of
// itself, i.e. the crossing moves by at most eps = L(L + 1) 2^-24 cells for
// L crossings, so every visited cell lies within eps of that line at the same
// time.  The cells from the current cell c on therefore lie in
// c + (-1 - 2 eps, 1 + 2 eps]^2 + K, where K is any closed cone containing
// (1/dX, 1/dY).  K is taken between two consecutive primitive vectors a, b
// of the Farey set of order 8 (all primitive (p, q) with p, q <= 8, sorted by
// angle), so det(a, b) = 1 and the lattice points of K are exactly the
// non-negative combinations of a and b.  Then
//   M(c)     = max(h(c), M(c + a), M(c + b))      (max over c + K)
// is two suffix maxima along lattice lines (first along a, then along b), and
// any lattice point of p + K with p in the box above is in e + K for the
// lattice point e = p - frac_ab(p), frac_ab(p) in {s a + t b : s, t in [0,1)};
// so the bound is the maximum of M over the window
//   e_X in [-(r + a_X + b_X), r],  e_Y in [-(r + a_Y + b_Y), r],
//   r = 1 + ceil(2 eps),
// taken as two one-dimensional passes.  Window apexes past the grid's far
// sides (in unsigned coordinates) reach no cell and are skipped; an apex
// before its near sides would need M outside the grid, so the bound there is
// +inf (the range test alone, as the reference).  Non-finite heights: NaN
// never hits and fmaxf skips it; +inf enters the maximum as itself.
#include "sgb_internal.cuh"

#include <climits>
#include <cmath>

namespace sgb {
namespace {

__device__ __forceinline__ size_t pad_index(int x, int y, int W)
{
    return (size_t)(x + 1) + (size_t)(y + 1) * (size_t)(W + 2);
}

__device__ __forceinline__ void to_grid(const ConeSpec& c, int X, int Y, int W, int H, int& x, int& y)
{
    x = c.sx > 0 ? X : W - 1 - X;
    y = c.sy > 0 ? Y : H - 1 - Y;
}

// Suffix maxima along the lattice lines of one cone vector (u, v) (unsigned
// coordinates): dst(c) = max(src(c), dst(c + (u, v))).  One thread a line,
// started at the line's last cell inside the grid (c + (u, v) outside).
// PASS 0: src = the grid's heights ([H][W]);  PASS 1: src = a bordered table.
template <int PASS>
__global__ void k_cone_lines(const float* __restrict__ src, int W, int H, const ConeSpec* __restrict__ specs,
                             float* __restrict__ dst, size_t stride)
{
    const ConeSpec c = specs[blockIdx.y];
    const int u = PASS == 0 ? c.ax : c.bx, v = PASS == 0 ? c.ay : c.by;
    const int uu = min(u, W), vv = min(v, H);
    const long long n1 = (long long)uu * H, n2 = (long long)(W - uu) * vv;
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n1 + n2) return;
    int X, Y;
    if (k < n1) { X = W - uu + (int)(k % uu); Y = (int)(k / uu); }
    else        { const long long k2 = k - n1; X = (int)(k2 % (W - uu)); Y = H - vv + (int)(k2 / (W - uu)); }
    const float* in = PASS == 0 ? src : src + stride * blockIdx.y;
    float* out = dst + stride * blockIdx.y;
    // a known trip count lets the loads of an unrolled stretch issue together
    const int n = min(u > 0 ? X / u : INT_MAX, v > 0 ? Y / v : INT_MAX) + 1;
    float m = -__int_as_float(0x7f800000);
#pragma unroll 4
    for (int i = 0; i < n; ++i, X -= u, Y -= v) {
        int x, y;
        to_grid(c, X, Y, W, H, x, y);
        const size_t p = pad_index(x, y, W);
        m = fmaxf(m, in[PASS == 0 ? (size_t)y * W + x : p]);
        out[p] = m;
    }
}

// Window maxima of M: PASS 0 over X offsets, PASS 1 over Y offsets (then
// min with maxz); both read src and write dst (bordered tables).  A block
// stages the stretch of its rows (PASS 0: 256 cells of one row; PASS 1: 64
// rows of 32 columns) plus the window's reach in shared memory, cells past
// the grid as -inf (a window clipped at the grid's edge), and each cell
// takes the maximum of its window from there.
constexpr int kWinRow = 256;          // PASS 0: cells of a row per block
constexpr int kWinCols = 32, kWinRows = 64, kWinRowsPerThread = 8;   // PASS 1 (256 threads)

template <int PASS>
__global__ void __launch_bounds__(256)
k_cone_window(int W, int H, float maxz, int r, const ConeSpec* __restrict__ specs,
              const float* __restrict__ src, float* __restrict__ dst, size_t stride)
{
    extern __shared__ float span[];
    const ConeSpec c = specs[blockIdx.y];
    const float* in = src + stride * blockIdx.y;
    float* out = dst + stride * blockIdx.y;
    // window in unsigned offsets [-(r + a + b), r], mirrored into grid offsets
    const int back = r + (PASS == 0 ? c.ax + c.bx : c.ay + c.by);
    const int s = PASS == 0 ? c.sx : c.sy;
    const int lo = s > 0 ? -back : -r, hi = s > 0 ? r : back;
    const int width = hi - lo + 1;
    const float ninf = -__int_as_float(0x7f800000), pinf = __int_as_float(0x7f800000);
    if (PASS == 0) {
        const int segs = (W + kWinRow - 1) / kWinRow;
        const int y = (int)(blockIdx.x / segs), x0 = (int)(blockIdx.x % segs) * kWinRow;
        const int n = kWinRow + width - 1;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const int q = x0 + lo + j;
            span[j] = (q >= 0 && q < W) ? in[pad_index(q, y, W)] : ninf;
        }
        __syncthreads();
        const int x = x0 + (int)threadIdx.x;
        if (x >= W) return;
        // the window's near end (unsigned offset -(r + a + b)) must lie inside
        const bool open = s > 0 ? x + lo < 0 : x + hi > W - 1;
        float m = open ? pinf : ninf;
        if (!open)
            for (int j = 0; j < width; ++j) m = fmaxf(m, span[threadIdx.x + j]);
        out[pad_index(x, y, W)] = m;
    } else {
        const int cols = (W + kWinCols - 1) / kWinCols;
        const int x0 = (int)(blockIdx.x % cols) * kWinCols, y0 = (int)(blockIdx.x / cols) * kWinRows;
        const int tx = threadIdx.x % kWinCols, ty = threadIdx.x / kWinCols;
        const int x = x0 + tx;
        const int rows = kWinRows + width - 1;
        for (int j = ty; j < rows; j += blockDim.x / kWinCols) {
            const int q = y0 + lo + j;
            span[j * kWinCols + tx] = (x < W && q >= 0 && q < H) ? in[pad_index(x, q, W)] : ninf;
        }
        __syncthreads();
        if (x >= W) return;
        for (int k = 0; k < kWinRowsPerThread; ++k) {
            const int yl = ty * kWinRowsPerThread + k, y = y0 + yl;
            if (y >= H) break;
            const bool open = s > 0 ? y + lo < 0 : y + hi > H - 1;
            float m = open ? pinf : ninf;
            if (!open)
                for (int j = 0; j < width; ++j) m = fmaxf(m, span[(yl + j) * kWinCols + tx]);
            out[pad_index(x, y, W)] = fminf(maxz, m);
        }
    }
}

// The border cells of every table: +inf (a ray there stops on the height
// test of the bordered heightmap, never on its bound).
__global__ void k_cone_border(int W, int H, float* __restrict__ tabs, size_t stride)
{
    const int Wp = W + 2;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2LL * (Wp + H)) return;
    size_t p;
    if (i < Wp)                p = (size_t)i;                                     // top row
    else if (i < 2 * Wp)       p = (size_t)(i - Wp) + (size_t)(H + 1) * Wp;       // bottom row
    else if (i < 2 * Wp + H)   p = (size_t)(i - 2 * Wp + 1) * Wp;                 // left column
    else                       p = (size_t)(i - 2 * Wp - H + 1) * Wp + (Wp - 1);  // right column
    tabs[stride * blockIdx.y + p] = __int_as_float(0x7f800000);
}

}  // namespace

int cone_window_radius(int W, int H)
{
    const double L = (double)(W > H ? W : H) + 4.0;
    const double eps2 = 2.0 * L * (L + 1.0) / 16777216.0;
    return 1 + (int)std::ceil(eps2);
}

cudaError_t launch_cone_tables(const float* grid, int W, int H, float maxz, const ConeSpec* specs, int n_specs,
                               float* tabs, float* tmp, size_t stride, cudaStream_t st)
{
    if (W <= 0 || H <= 0 || n_specs <= 0) return cudaSuccess;
    const unsigned border = (unsigned)((2LL * (W + 2 + H) + 255) / 256);
    // start cells of a line family: at most kConeOrder (W + H)
    const unsigned lines = (unsigned)(((long long)kConeOrder * (W + H) + 255) / 256);
    const int r = cone_window_radius(W, H);
    k_cone_lines<0><<<dim3(lines, n_specs), 256, 0, st>>>(grid, W, H, specs, tmp, stride);
    k_cone_lines<1><<<dim3(lines, n_specs), 256, 0, st>>>(tmp, W, H, specs, tabs, stride);
    // the widest window: r on one side, r + a + b (components <= kConeOrder each) on the other
    const int wmax = 2 * r + 2 * kConeOrder + 1;
    const unsigned win0 = (unsigned)(((long long)W + kWinRow - 1) / kWinRow * H);
    const unsigned win1 = (unsigned)(((long long)W + kWinCols - 1) / kWinCols * ((H + kWinRows - 1) / kWinRows));
    k_cone_window<0><<<dim3(win0, n_specs), 256, sizeof(float) * (kWinRow + wmax), st>>>(W, H, maxz, r, specs,
                                                                                       tabs, tmp, stride);
    k_cone_window<1><<<dim3(win1, n_specs), 256, sizeof(float) * kWinCols * (kWinRows + wmax), st>>>(
        W, H, maxz, r, specs, tmp, tabs, stride);
    k_cone_border<<<dim3(border, n_specs), 256, 0, st>>>(W, H, tabs, stride);
    return cudaGetLastError();
}

}  // namespace sgb
