// tild_grid.cu -- density deposit and reference-exact stencil tables (sm_100a).
#include "tild_stencil.cuh"

#include <cmath>
#include <cstdio>
#include <vector>

namespace tild {

// =====================================================================================
// Density deposit.  Fast mode: float atomics (float2 vector atomics for packed pairs).
// Deterministic mode: 64-bit fixed-point integer atomics (exact, order independent).
// The deposit stores S = sum Wx*Wy*Wz; the 1/gvol of the reference's weights is folded
// into the k-space constants.
// =====================================================================================

template <int P>
__global__ void __launch_bounds__(256) k_deposit(Geom g, int N, int quirk4, int nd, unsigned dq,
                                                 const float *__restrict__ X0, const float *__restrict__ X1,
                                                 const long long *__restrict__ d_step,
                                                 const uint32_t *__restrict__ pflags,
                                                 const float *__restrict__ q,
                                                 float2 *__restrict__ dep,
                                                 unsigned long long *__restrict__ depfix)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const uint32_t dm = pflags[p] & 0xffu;
    if (!dm) return;
    const float *__restrict__ X = (*d_step & 1) ? X1 : X0;
    float Wx[P + 1], Wy[P + 1], Wz[P + 1];
    int ix[P + 1], iy[P + 1], iz[P + 1];
    const int gx = stencil_axis<P>(X[3 * p + 0], g.dxf[0], quirk4, Wx);
    const int gy = stencil_axis<P>(X[3 * p + 1], g.dxf[1], quirk4, Wy);
    const int gz = stencil_axis<P>(X[3 * p + 2], g.dxf[2], quirk4, Wz);
#pragma unroll
    for (int i = 0; i <= P; i++) {
        ix[i] = wrapi(gx + i, g.nx);
        iy[i] = wrapi(gy + i, g.ny);
        iz[i] = wrapi(gz + i, g.nz);
    }
    const float qp = q ? q[p] : 0.f;
    float c[kMaxFields];
#pragma unroll
    for (int i = 0; i < kMaxFields; i++)
        c[i] = (i < nd && ((dm >> i) & 1u)) ? (((dq >> i) & 1u) ? qp : 1.f) : 0.f;
    const int npair = (nd + 1) >> 1;
    const long long plane = (long long)g.nx * g.ny;
#pragma unroll 1
    for (int e = 0; e <= P; e++) {
        const float wz = sel<P>(Wz, e);
        const long long mz = plane * sel<P>(iz, e);
#pragma unroll
        for (int b = 0; b <= P; b++) {
            const float wyz = Wy[b] * wz;
            const long long my = mz + (long long)g.nx * iy[b];
#pragma unroll
            for (int a = 0; a <= P; a++) {
                const float w = Wx[a] * wyz;
                const long long m = my + ix[a];
                for (int t = 0; t < npair; t++) {
                    const float v0 = c[2 * t] * w, v1 = c[2 * t + 1] * w;
                    if (depfix) {
                        if (v0 != 0.f)
                            atomicAdd(depfix + (2 * t) * g.M + m,
                                      (unsigned long long)__double2ll_rn((double)v0 * kFixScale));
                        if (v1 != 0.f)
                            atomicAdd(depfix + (2 * t + 1) * g.M + m,
                                      (unsigned long long)__double2ll_rn((double)v1 * kFixScale));
                    } else if (v0 != 0.f && v1 != 0.f) {
                        atomicAdd(dep + t * g.M + m, make_float2(v0, v1));
                    } else if (v0 != 0.f) {
                        atomicAdd(&dep[t * g.M + m].x, v0);
                    } else if (v1 != 0.f) {
                        atomicAdd(&dep[t * g.M + m].y, v1);
                    }
                }
            }
        }
    }
}

// Reference-exact stencil table (d_calcGridWeights, ps_grid_utils.cu:74-204), 3-D.
template <int P>
__global__ void k_grid_weights(Geom g, int quirk4, const float *X, int N, int *inds, float *W)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    float Wx[P + 1], Wy[P + 1], Wz[P + 1];
    const int gx = stencil_axis<P>(X[3 * p], g.dxf[0], quirk4, Wx);
    const int gy = stencil_axis<P>(X[3 * p + 1], g.dxf[1], quirk4, Wy);
    const int gz = stencil_axis<P>(X[3 * p + 2], g.dxf[2], quirk4, Wz);
    const float gvol = __fmul_rn(__fmul_rn(__fmul_rn(1.0f, g.dxf[0]), g.dxf[1]), g.dxf[2]);
    constexpr int G = (P + 1) * (P + 1) * (P + 1);
    int ct = 0;
    for (int a = 0; a <= P; a++) {
        const int n0 = wrapi(gx + a, g.nx);
        for (int b = 0; b <= P; b++) {
            const int n1 = wrapi(gy + b, g.ny);
            for (int e = 0; e <= P; e++) {
                const int n2 = wrapi(gz + e, g.nz);
                inds[(long long)p * G + ct] = n0 + (n1 + n2 * g.ny) * g.nx;
                W[(long long)p * G + ct] = __fdiv_rn(__fmul_rn(__fmul_rn(Wx[a], Wy[b]), Wz[e]), gvol);
                ct++;
            }
        }
    }
}

// One group's density (or charge density) with the reference's weights (/gvol).
template <int P>
__global__ void k_density_single(Geom g, int quirk4, const float *X, const int *sites, int ns,
                                 const float *q, int charge, float *rho)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    const int p = sites[s];
    float Wx[P + 1], Wy[P + 1], Wz[P + 1];
    const int gx = stencil_axis<P>(X[3 * p], g.dxf[0], quirk4, Wx);
    const int gy = stencil_axis<P>(X[3 * p + 1], g.dxf[1], quirk4, Wy);
    const int gz = stencil_axis<P>(X[3 * p + 2], g.dxf[2], quirk4, Wz);
    const float gvol = __fmul_rn(__fmul_rn(g.dxf[0], g.dxf[1]), g.dxf[2]);
    const float c = charge ? q[p] : 1.f;
    for (int a = 0; a <= P; a++)
        for (int b = 0; b <= P; b++)
            for (int e = 0; e <= P; e++) {
                const long long m = wrapi(gx + a, g.nx) + (long long)g.nx * (wrapi(gy + b, g.ny) + (long long)g.ny * wrapi(gz + e, g.nz));
                atomicAdd(rho + m, __fdiv_rn(__fmul_rn(__fmul_rn(Wx[a], Wy[b]), Wz[e]), gvol) * c);
            }
}


// ---- launchers ----
cudaError_t launch_zero(void *p, size_t bytes, cudaStream_t st) { return cudaMemsetAsync(p, 0, bytes, st); }

template <int P>
static void dep_launch(const Geom &g, const ParticleParams &pp, const float *X0, const float *X1,
                       const long long *d_step, const uint32_t *pflags, const float *q, float2 *dep,
                       unsigned long long *depfix, cudaStream_t st)
{
    const int bs = 256, nb = (pp.N + bs - 1) / bs;
    k_deposit<P><<<nb, bs, 0, st>>>(g, pp.N, pp.quirk4, pp.nd, pp.dchan_charge, X0, X1, d_step, pflags, q, dep,
                                    depfix);
}

cudaError_t launch_deposit(const Geom &g, const ParticleParams &pp, const float *X0, const float *X1,
                           const long long *d_step, const uint32_t *pflags, const float *q, float2 *dep,
                           unsigned long long *dep_fixed, int deterministic, cudaStream_t st)
{
    if (pp.N == 0) return cudaSuccess;
    unsigned long long *df = deterministic ? dep_fixed : nullptr;
    switch (pp.order) {
        case 0: dep_launch<0>(g, pp, X0, X1, d_step, pflags, q, dep, df, st); break;
        case 1: dep_launch<1>(g, pp, X0, X1, d_step, pflags, q, dep, df, st); break;
        case 2: dep_launch<2>(g, pp, X0, X1, d_step, pflags, q, dep, df, st); break;
        case 3: dep_launch<3>(g, pp, X0, X1, d_step, pflags, q, dep, df, st); break;
        default: dep_launch<4>(g, pp, X0, X1, d_step, pflags, q, dep, df, st); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_grid_weights(const Geom &g, int order, int quirk4, const float *X, int N, int *inds, float *W,
                                cudaStream_t st)
{
    if (N == 0) return cudaSuccess;
    const int nbk = (N + 255) / 256;
    switch (order) {
        case 0: k_grid_weights<0><<<nbk, 256, 0, st>>>(g, quirk4, X, N, inds, W); break;
        case 1: k_grid_weights<1><<<nbk, 256, 0, st>>>(g, quirk4, X, N, inds, W); break;
        case 2: k_grid_weights<2><<<nbk, 256, 0, st>>>(g, quirk4, X, N, inds, W); break;
        case 3: k_grid_weights<3><<<nbk, 256, 0, st>>>(g, quirk4, X, N, inds, W); break;
        default: k_grid_weights<4><<<nbk, 256, 0, st>>>(g, quirk4, X, N, inds, W); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_density_single(const Geom &g, const ParticleParams &pp, const float *X, const int *sites, int ns,
                                  const float *q, int charge, float *rho, cudaStream_t st)
{
    if (ns == 0) return cudaSuccess;
    const int nbk = (ns + 255) / 256;
    switch (pp.order) {
        case 0: k_density_single<0><<<nbk, 256, 0, st>>>(g, pp.quirk4, X, sites, ns, q, charge, rho); break;
        case 1: k_density_single<1><<<nbk, 256, 0, st>>>(g, pp.quirk4, X, sites, ns, q, charge, rho); break;
        case 2: k_density_single<2><<<nbk, 256, 0, st>>>(g, pp.quirk4, X, sites, ns, q, charge, rho); break;
        case 3: k_density_single<3><<<nbk, 256, 0, st>>>(g, pp.quirk4, X, sites, ns, q, charge, rho); break;
        default: k_density_single<4><<<nbk, 256, 0, st>>>(g, pp.quirk4, X, sites, ns, q, charge, rho); break;
    }
    return cudaGetLastError();
}

}  // namespace tild
