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
// and the tracer ends an upward ray with no hit when its height at the cell
// it is about to test exceeds `bound` (it checks every few steps).  The result is the reference's, bit for bit:
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
    float m = -__int_as_float(0x7f800000);
    for (; X >= 0 && Y >= 0; X -= u, Y -= v) {
        int x, y;
        to_grid(c, X, Y, W, H, x, y);
        const size_t p = pad_index(x, y, W);
        m = fmaxf(m, in[PASS == 0 ? (size_t)y * W + x : p]);
        out[p] = m;
    }
}

// Window maxima of M: PASS 0 over X offsets, PASS 1 over Y offsets (then
// min with maxz); both read src and write dst (bordered tables).
template <int PASS>
__global__ void k_cone_window(int W, int H, float maxz, int r, const ConeSpec* __restrict__ specs,
                              const float* __restrict__ src, float* __restrict__ dst, size_t stride)
{
    const ConeSpec c = specs[blockIdx.y];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)W * H) return;
    const int x = (int)(i % W), y = (int)(i / W);
    const float* in = src + stride * blockIdx.y;
    // window in unsigned offsets [-(r + a + b), r], mirrored into grid offsets
    const int back = r + (PASS == 0 ? c.ax + c.bx : c.ay + c.by);
    const int s = PASS == 0 ? c.sx : c.sy;
    const int lo = s > 0 ? -back : -r, hi = s > 0 ? r : back;
    const int pos = PASS == 0 ? x : y, len = PASS == 0 ? W : H;
    // the window's near end (unsigned offset -(r + a + b)) must lie inside
    const bool open = s > 0 ? pos + lo < 0 : pos + hi > len - 1;
    const int b0 = max(pos + lo, 0), b1 = min(pos + hi, len - 1);
    float m = open ? __int_as_float(0x7f800000) : -__int_as_float(0x7f800000);
    for (int q = open ? b1 + 1 : b0; q <= b1; ++q)
        m = fmaxf(m, in[PASS == 0 ? pad_index(q, y, W) : pad_index(x, q, W)]);
    dst[stride * blockIdx.y + pad_index(x, y, W)] = PASS == 0 ? m : fminf(maxz, m);
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
    const unsigned cells = (unsigned)(((long long)W * H + 255) / 256);
    const unsigned border = (unsigned)((2LL * (W + 2 + H) + 255) / 256);
    // start cells of a line family: at most kConeOrder (W + H)
    const unsigned lines = (unsigned)(((long long)kConeOrder * (W + H) + 255) / 256);
    const int r = cone_window_radius(W, H);
    k_cone_lines<0><<<dim3(lines, n_specs), 256, 0, st>>>(grid, W, H, specs, tmp, stride);
    k_cone_lines<1><<<dim3(lines, n_specs), 256, 0, st>>>(tmp, W, H, specs, tabs, stride);
    k_cone_window<0><<<dim3(cells, n_specs), 256, 0, st>>>(W, H, maxz, r, specs, tabs, tmp, stride);
    k_cone_window<1><<<dim3(cells, n_specs), 256, 0, st>>>(W, H, maxz, r, specs, tmp, tabs, stride);
    k_cone_border<<<dim3(border, n_specs), 256, 0, st>>>(W, H, tabs, stride);
    return cudaGetLastError();
}

}  // namespace sgb
