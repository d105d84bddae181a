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

// (g + i - shift + N) % N in the reference; a true modulo here so that positions the
// reference would send out of bounds still land on the grid.
__device__ __forceinline__ int wrapi(int v, int n)
{
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
