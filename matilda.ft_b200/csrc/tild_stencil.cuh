// tild_stencil.cuh -- particle/grid stencil helpers shared by the TILD kernels.
#pragma once
#include "tild_device.h"

namespace tild {


// =====================================================================================
// Stencil weights: ps_grid_utils.cu:17-67 with the rounding of the reference build
// (nvcc contracts a*b+c into one FMA by default), written with explicit intrinsics so
// indices and weights are reproducible bit for bit.
// =====================================================================================
template <int P>
__device__ __forceinline__ void spline_w(float gdx, float H, int quirk4, float *W)
{
    const float sx = __fdiv_rn(gdx, H);
    if (P == 0) {
        W[0] = 1.f;
    } else if (P == 1) {
        W[0] = __fsub_rn(0.5f, sx);
        W[1] = __fadd_rn(0.5f, sx);
    } else if (P == 2) {
        const float sx2 = __fmul_rn(sx, sx);
        W[0] = __fmaf_rn(0.5f, sx2, __fmaf_rn(-0.5f, sx, 0.125f));
        W[1] = __fsub_rn(0.75f, sx2);
        W[2] = __fmaf_rn(0.5f, sx2, __fmaf_rn(0.5f, sx, 0.125f));
    } else if (P == 3) {
        const float sx2 = __fmul_rn(sx, sx), sx3 = __fmul_rn(sx2, sx);
        W[0] = __fdiv_rn(__fmaf_rn(-8.f, sx3, __fmaf_rn(12.f, sx2, __fmaf_rn(-6.f, sx, 1.f))), 48.f);
        W[1] = __fdiv_rn(__fmaf_rn(24.f, sx3, __fmaf_rn(-12.f, sx2, __fmaf_rn(-30.f, sx, 23.f))), 48.f);
        W[2] = __fdiv_rn(__fmaf_rn(-24.f, sx3, __fmaf_rn(-12.f, sx2, __fmaf_rn(30.f, sx, 23.f))), 48.f);
        W[3] = __fdiv_rn(__fmaf_rn(8.f, sx3, __fmaf_rn(12.f, sx2, __fmaf_rn(6.f, sx, 1.f))), 48.f);
    } else {
        const float sx2 = __fmul_rn(sx, sx);
        const float sx3 = quirk4 ? __fmul_rn(sx2, sx2) : __fmul_rn(sx2, sx);
        const float sx4 = __fmul_rn(sx2, sx2);
        W[0] = __fdiv_rn(__fmaf_rn(16.f, sx4, __fmaf_rn(-32.f, sx3, __fmaf_rn(24.f, sx2, __fmaf_rn(-8.f, sx, 1.f)))), 384.f);
        W[1] = __fdiv_rn(__fmaf_rn(-16.f, sx4, __fmaf_rn(16.f, sx3, __fmaf_rn(24.f, sx2, __fmaf_rn(-44.f, sx, 19.f)))), 96.f);
        W[2] = __fdiv_rn(__fmaf_rn(48.f, sx4, __fmaf_rn(-120.f, sx2, 115.f)), 192.f);
        W[3] = __fdiv_rn(__fmaf_rn(-16.f, sx4, __fmaf_rn(-16.f, sx3, __fmaf_rn(24.f, sx2, __fmaf_rn(44.f, sx, 19.f)))), 96.f);
        W[4] = __fdiv_rn(__fmaf_rn(16.f, sx4, __fmaf_rn(32.f, sx3, __fmaf_rn(24.f, sx2, __fmaf_rn(8.f, sx, 1.f)))), 384.f);
    }
}

// Nearest grid point (even P) or cell (odd P) of one coordinate and its P+1 weights
// (ps_grid_utils.cu:105-115).  Returns the first stencil index g - P/2 (unwrapped).
template <int P>
__device__ __forceinline__ int stencil_axis(float x, float d, int quirk4, float *W)
{
    int g;
    float gdx;
    if (P % 2 == 0) {
        g = (int)__fdiv_rn(__fmaf_rn(0.5f, d, x), d);
        gdx = __fmaf_rn(-(float)g, d, x);
    } else {
        g = (int)__fdiv_rn(x, d);
        gdx = __fmaf_rn(-__fadd_rn((float)g, 0.5f), d, x);
    }
    spline_w<P>(gdx, d, quirk4, W);
    return g - P / 2;
}

// Fast stencil for the deposit and the gather: the reference's cell choice and spline
// polynomials, evaluated with a reciprocal multiply and Horner FMAs instead of IEEE
// divisions.  The cell is picked from t = x / d; the offset inside it is then taken from
// x - c d with d split into its FP32 value and the FP32 remainder of L / Nx (g.dxf, g.dlo),
// each product folded in by one FMA, so the offset carries an error of a few units in the
// last place of d instead of t's rounding (which grows with x: about 1e-5 of a cell at
// x / d = 160).  Weights therefore differ from exact B-spline weights at the FP64 position
// by rounding only, and from the reference's by its own rounding (the splines are continuous
// across cell edges, so a different cell pick at an edge moves nothing).
// Returns the first stencil index; W[0..P] are the 1-D weights (unscaled, sum 1).
template <int P>
__device__ __forceinline__ int stencil_fast(float x, const Geom &g, int j, int quirk4, float *W)
{
    const float inv_d = g.inv[j];
    const float t = x * inv_d;
    int g0;
    float c;
    if (P % 2 == 0) {
        g0 = (int)(t + 0.5f);
        c = (float)g0;
    } else {
        g0 = (int)t;
        c = (float)g0 + 0.5f;
    }
    const float s = __fmaf_rn(-c, g.dlo[j], __fmaf_rn(-c, g.dxf[j], x)) * inv_d;
    if (P == 0) {
        W[0] = 1.f;
    } else if (P == 1) {
        W[0] = 0.5f - s;
        W[1] = 0.5f + s;
    } else if (P == 2) {
        const float s2 = s * s;
        W[0] = fmaf(0.5f, s2, fmaf(-0.5f, s, 0.125f));
        W[1] = 0.75f - s2;
        W[2] = fmaf(0.5f, s2, fmaf(0.5f, s, 0.125f));
    } else if (P == 3) {
        W[0] = fmaf(fmaf(fmaf(-1.f / 6.f, s, 0.25f), s, -0.125f), s, 1.f / 48.f);
        W[1] = fmaf(fmaf(fmaf(0.5f, s, -0.25f), s, -0.625f), s, 23.f / 48.f);
        W[2] = fmaf(fmaf(fmaf(-0.5f, s, -0.25f), s, 0.625f), s, 23.f / 48.f);
        W[3] = fmaf(fmaf(fmaf(1.f / 6.f, s, 0.25f), s, 0.125f), s, 1.f / 48.f);
    } else {
        const float s2 = s * s, s4 = s2 * s2, s3 = quirk4 ? s4 : s2 * s;
        W[0] = (1.f - 8.f * s + 24.f * s2 - 32.f * s3 + 16.f * s4) * (1.f / 384.f);
        W[1] = (19.f - 44.f * s + 24.f * s2 + 16.f * s3 - 16.f * s4) * (1.f / 96.f);
        W[2] = (115.f - 120.f * s2 + 48.f * s4) * (1.f / 192.f);
        W[3] = (19.f + 44.f * s + 24.f * s2 - 16.f * s3 - 16.f * s4) * (1.f / 96.f);
        W[4] = (1.f + 8.f * s + 24.f * s2 + 32.f * s3 + 16.f * s4) * (1.f / 384.f);
    }
    return g0 - P / 2;
}

// Batched launches: CTA b of a launch over several replicas belongs to replica r with
// pre[r] <= b < pre[r + 1] (pre: the exclusive prefix of the replicas' CTA counts).
__device__ __forceinline__ int batch_replica(const int *__restrict__ pre, int R, int b)
{
    int lo = 0, hi = R;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pre[mid] <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}

// -------------------------------------------------------------------------------------
// Tiles of spatially sorted particles.  A CTA takes the particles of `codes` (a power of
// two >= 8) consecutive brick Morton codes -- contiguous slots after the sort, an aligned
// block of bricks of 4^3 cells -- and works on the box of grid points their stencils
// cover, staged in shared memory.  The host sizes codes and the CTA from the density so
// that a CTA holds about one particle per thread.  The box is described relative to the stencil origin of the CTA's first
// particle (periodic unwrap); per-axis index tables turn a box coordinate into a grid
// offset without divisions.
// -------------------------------------------------------------------------------------
constexpr int kMaxBoxEdge = 64;

struct TileShared {
    int ref[3], lo[3], hi[3];
    unsigned fm;
    int xi[kMaxBoxEdge];   // wrapped x index of box column lx
    int yb[kMaxBoxEdge];   // nx * wrapped y of box row ly
    int zb[kMaxBoxEdge];   // nx * ny * wrapped z of box plane lz
};

__device__ __forceinline__ int unwrap_delta(int d, int n)
{
    int t = (d >= 0 && d < n) ? d : d % n;
    if (t < 0) t += n;
    if (t >= (n + 1) / 2) t -= n;
    return t;
}

// first stencil index of the fast stencil (same cell choice as stencil_fast)
template <int P>
__device__ __forceinline__ int stencil_origin(float x, const Geom &g, int j)
{
    const float t = x * g.inv[j];
    const int g0 = (P % 2 == 0) ? (int)(t + 0.5f) : (int)t;
    return g0 - P / 2;
}

// The z axis of a 2-D box is one plane (nz == 1, every particle at z = 0): its stencil is
// the single point 0 with weight 1 (the z loops still run over P + 1 points, the others
// with weight 0), so products Wx*Wy*Wz are exactly the 2-D weights Wx*Wy.
template <int P>
__device__ __forceinline__ int stencil_fast_z(float z, const Geom &g, int quirk4, float *W)
{
    if (g.nz != 1) return stencil_fast<P>(z, g, 2, quirk4, W);
    W[0] = 1.f;
#pragma unroll
    for (int k = 1; k <= P; k++) W[k] = 0.f;
    return 0;
}

template <int P>
__device__ __forceinline__ int stencil_axis_z(float z, float d, int quirk4, float *W, int nz)
{
    if (nz != 1) return stencil_axis<P>(z, d, quirk4, W);
    W[0] = 1.f;
#pragma unroll
    for (int k = 1; k <= P; k++) W[k] = 0.f;
    return 0;
}

template <int P>
__device__ __forceinline__ int stencil_origin_z(float z, const Geom &g)
{
    return g.nz == 1 ? 0 : stencil_origin<P>(z, g, 2);
}

// the CTA's tile: entry bx (the CTA's index among the launch's tiles) of the list of tiles
// that meet the grid, when there is one
__device__ __forceinline__ uint32_t tile_id(const TileCfg &tc, unsigned bx) { return tc.list ? tc.list[bx] : bx; }
__device__ __forceinline__ uint32_t tile_id(const TileCfg &tc) { return tile_id(tc, blockIdx.x); }

// number of CTAs of a launch over the tiles (host)
inline int tile_ctas(const TileCfg &tc) { return tc.list ? tc.nlist : (tc.nkeys + tc.codes - 1) / tc.codes; }

// [b0, b1) of CTA bx: a tile of sorted particles, or a fixed window of slots
__device__ __forceinline__ void tile_range(const TileCfg &tc, int N, int window, int &b0, int &b1, unsigned bx)
{
    if (tc.start) {
        const int k0 = (int)tile_id(tc, bx) * tc.codes;
        b0 = (int)tc.start[k0];
        b1 = (k0 + tc.codes < tc.nkeys) ? (int)tc.start[k0 + tc.codes] : N;
    } else {
        b0 = (int)bx * window;
        b1 = min(N, b0 + window);
    }
}
__device__ __forceinline__ void tile_range(const TileCfg &tc, int N, int window, int &b0, int &b1)
{
    tile_range(tc, N, window, b0, b1, blockIdx.x);
}

// every third bit -> 10-bit value (inverse of the sort's brick-key interleave)
__device__ __forceinline__ int compact3(uint32_t v)
{
    v &= 0x09249249u;
    v = (v | (v >> 2)) & 0x030C30C3u;
    v = (v | (v >> 4)) & 0x0300F00Fu;
    v = (v | (v >> 8)) & 0x030000FFu;
    v = (v | (v >> 16)) & 0x000003FFu;
    return (int)v;
}

// Fixed box of a sorted tile: the grid cells of its block of bricks (where its particles
// were at the last sort) widened by tc.margin cells per side, as stencil origins
// lo[j] .. lo[j] + span[j]; E[j] = span[j] + P + 1 grid points per axis.
template <int P>
__device__ __forceinline__ void tile_box(const TileCfg &tc, const int *nn, int *lo, int *span, int *E, unsigned bx)
{
    int bits = 0;
    while ((1 << bits) < tc.codes) bits++;
    const uint32_t k0 = tile_id(tc, bx) * (uint32_t)tc.codes;
    const int nbr[3] = {1 << ((bits + 2) / 3), 1 << ((bits + 1) / 3), 1 << (bits / 3)};
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int c0 = 4 * compact3(k0 >> j);
        const int c1 = min(c0 + 4 * nbr[j], nn[j]) - 1;
        lo[j] = c0 - P / 2 - tc.margin;
        span[j] = c1 - c0 + (P % 2 == 0 ? 1 : 0) + 2 * tc.margin;
        E[j] = span[j] + P + 1;
    }
}
template <int P>
__device__ __forceinline__ void tile_box(const TileCfg &tc, const int *nn, int *lo, int *span, int *E)
{
    tile_box<P>(tc, nn, lo, span, E, blockIdx.x);
}

// Fill the per-axis index tables of a box with edges E (all threads; E[d] <= kMaxBoxEdge).
__device__ __forceinline__ void tile_tables(TileShared &ts, int nx, int ny, int nz, const int *E)
{
    const int n3[3] = {nx, ny, nz};
    for (int t = threadIdx.x; t < E[0] + E[1] + E[2]; t += blockDim.x) {
        const int d = t < E[0] ? 0 : (t < E[0] + E[1] ? 1 : 2);
        const int l = t - (d == 0 ? 0 : (d == 1 ? E[0] : E[0] + E[1]));
        int v = (ts.ref[d] + ts.lo[d] + l) % n3[d];
        if (v < 0) v += n3[d];
        if (d == 0) ts.xi[l] = v;
        else if (d == 1) ts.yb[l] = v * nx;
        else ts.zb[l] = v * nx * ny;
    }
}

// Visit every box element (x fastest) with lanes along x: f(v, grid_offset), where v is
// the element's offset in a box stored with row pitch p1 and plane pitch p2.  A row of
// E[0] <= 32 elements takes E[0] consecutive threads; rows advance by counters, with no
// division inside the loop.
template <typename F>
__device__ __forceinline__ void tile_for_each(const TileShared &ts, const int *E, int p1, int p2, F f)
{
    const int E0 = E[0], E1 = E[1], rows = E1 * E[2];
    const int xw = E0 <= 32 ? E0 : 32;
    const int rpp = blockDim.x / xw;
    if ((int)threadIdx.x >= rpp * xw) return;
    int row = threadIdx.x / xw;
    const int lx0 = threadIdx.x - row * xw;
    int lz = row / E1, ly = row - lz * E1;
    const int dz = rpp / E1, dy = rpp - dz * E1;
    for (; row < rows; row += rpp) {
        const int rb = ts.zb[lz] + ts.yb[ly];
        const int vb = lz * p2 + ly * p1;
        for (int lx = lx0; lx < E0; lx += xw) f(vb + lx, rb + ts.xi[lx]);
        lz += dz;
        ly += dy;
        if (ly >= E1) {
            ly -= E1;
            lz++;
        }
    }
}

// tile_for_each that also passes the element's box coordinates: f(v, m, lx, ly, lz).
template <typename F>
__device__ __forceinline__ void tile_for_each_xyz(const TileShared &ts, const int *E, int p1, int p2, F f)
{
    const int E0 = E[0], E1 = E[1], rows = E1 * E[2];
    const int xw = E0 <= 32 ? E0 : 32;
    const int rpp = blockDim.x / xw;
    if ((int)threadIdx.x >= rpp * xw) return;
    int row = threadIdx.x / xw;
    const int lx0 = threadIdx.x - row * xw;
    int lz = row / E1, ly = row - lz * E1;
    const int dz = rpp / E1, dy = rpp - dz * E1;
    for (; row < rows; row += rpp) {
        const int rb = ts.zb[lz] + ts.yb[ly];
        const int vb = lz * p2 + ly * p1;
        for (int lx = lx0; lx < E0; lx += xw) f(vb + lx, rb + ts.xi[lx], lx, ly, lz);
        lz += dz;
        ly += dy;
        if (ly >= E1) {
            ly -= E1;
            lz++;
        }
    }
}

// (g + i - shift + N) % N in the reference; a true modulo here so that positions the
// reference would send out of bounds still land on the grid.
__device__ __forceinline__ int wrapi(int v, int n)
{
    if ((unsigned)v < (unsigned)n) return v;   // the common case: already on the grid
    v %= n;
    return v < 0 ? v + n : v;
}


// Element i of a small register array without dynamic indexing (keeps it in registers
// when the loop over i is not unrolled).
template <int P, typename T>
__device__ __forceinline__ T sel(const T *a, int i)
{
    T r = a[0];
#pragma unroll
    for (int k = 1; k <= P; k++)
        if (i == k) r = a[k];
    return r;
}

}  // namespace tild
