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

// -------------------------------------------------------------------------------------
// Shared-memory staged deposit for spatially sorted particles.  Each CTA takes
// kDepPB consecutive slots, finds the box of grid points their stencils cover (relative
// to the first particle, periodic unwrap), accumulates into that box in shared memory
// and flushes every touched point once with a global (float2 or u64) atomic.  A CTA
// whose box does not fit falls back to per-point global atomics.
// -------------------------------------------------------------------------------------
constexpr int kDepPB = 512;
// float pointer to field f of the packed pair array (field 2t in .x, 2t+1 in .y of pair t)
#define FIELD_PTR(dep, f, M) (reinterpret_cast<float *>((dep) + ((f) >> 1) * (M)) + ((f) & 1))
constexpr int kDepSmemFast = 64 * 1024;
constexpr int kDepSmemFixed = 128 * 1024;

__device__ __forceinline__ int unwrap_delta(int d, int n)
{
    int t = d % n;
    if (t < 0) t += n;
    if (t >= (n + 1) / 2) t -= n;
    return t;
}

template <int P>
__device__ __forceinline__ int stencil_origin(float x, float d)
{
    int g;
    if (P % 2 == 0) g = (int)__fdiv_rn(__fmaf_rn(0.5f, d, x), d);
    else g = (int)__fdiv_rn(x, d);
    return g - P / 2;
}

template <int P, bool FIXED>
__global__ void __launch_bounds__(256) k_deposit_tiled(Geom g, int N, int quirk4, int nd, unsigned dq,
                                                       const float *__restrict__ X0, const float *__restrict__ X1,
                                                       const long long *__restrict__ d_step,
                                                       const uint32_t *__restrict__ pflags,
                                                       const float *__restrict__ q, float2 *__restrict__ dep,
                                                       unsigned long long *__restrict__ depfix, int cap_bytes)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ int s_ref[3], s_min[3], s_max[3];
    const float *__restrict__ X = (*d_step & 1) ? X1 : X0;
    const int b0 = blockIdx.x * kDepPB;
    const int nloc = min(kDepPB, N - b0);
    const int nn[3] = {g.nx, g.ny, g.nz};
    if (threadIdx.x < 3) {
        s_ref[threadIdx.x] = stencil_origin<P>(X[3 * b0 + threadIdx.x], g.dxf[threadIdx.x]);
        s_min[threadIdx.x] = 0x7fffffff;
        s_max[threadIdx.x] = -0x7fffffff;
    }
    __syncthreads();
    int lo[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, hi[3] = {-0x7fffffff, -0x7fffffff, -0x7fffffff};
    for (int k = threadIdx.x; k < nloc; k += blockDim.x) {
        const int p = b0 + k;
        if (!(pflags[p] & 0xffu)) continue;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int dd = unwrap_delta(stencil_origin<P>(X[3 * p + j], g.dxf[j]) - s_ref[j], nn[j]);
            lo[j] = min(lo[j], dd);
            hi[j] = max(hi[j], dd);
        }
    }
#pragma unroll
    for (int j = 0; j < 3; j++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[j] = min(lo[j], __shfl_xor_sync(0xffffffffu, lo[j], o));
            hi[j] = max(hi[j], __shfl_xor_sync(0xffffffffu, hi[j], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&s_min[j], lo[j]);
            atomicMax(&s_max[j], hi[j]);
        }
    }
    __syncthreads();
    if (s_max[0] < s_min[0]) return;   // no depositing particle in this CTA
    const int E0 = s_max[0] - s_min[0] + P + 1, E1 = s_max[1] - s_min[1] + P + 1, E2 = s_max[2] - s_min[2] + P + 1;
    const long long V = (long long)E0 * E1 * E2;
    const size_t esz = FIXED ? sizeof(unsigned long long) : sizeof(float);
    const bool staged = V * nd * (long long)esz <= cap_bytes;
    float *tf = reinterpret_cast<float *>(smraw);
    unsigned long long *tu = reinterpret_cast<unsigned long long *>(smraw);
    if (staged) {
        for (long long v = threadIdx.x; v < V * nd; v += blockDim.x) {
            if (FIXED) tu[v] = 0ull;
            else tf[v] = 0.f;
        }
    }
    __syncthreads();
    const long long plane = (long long)g.nx * g.ny;
    for (int k = threadIdx.x; k < nloc; k += blockDim.x) {
        const int p = b0 + k;
        const uint32_t dm = pflags[p] & 0xffu;
        if (!dm) continue;
        float Wx[P + 1], Wy[P + 1], Wz[P + 1];
        const int gx = stencil_axis<P>(X[3 * p + 0], g.dxf[0], quirk4, Wx);
        const int gy = stencil_axis<P>(X[3 * p + 1], g.dxf[1], quirk4, Wy);
        const int gz = stencil_axis<P>(X[3 * p + 2], g.dxf[2], quirk4, Wz);
        const float qp = q ? q[p] : 0.f;
        float c[kMaxFields];
#pragma unroll
        for (int i = 0; i < kMaxFields; i++)
            c[i] = (i < nd && ((dm >> i) & 1u)) ? (((dq >> i) & 1u) ? qp : 1.f) : 0.f;
        if (staged) {
            const int lx = unwrap_delta(gx - s_ref[0], g.nx) - s_min[0];
            const int ly = unwrap_delta(gy - s_ref[1], g.ny) - s_min[1];
            const int lz = unwrap_delta(gz - s_ref[2], g.nz) - s_min[2];
#pragma unroll 1
            for (int e = 0; e <= P; e++) {
                const float wz = sel<P>(Wz, e);
#pragma unroll
                for (int b = 0; b <= P; b++) {
                    const float wyz = Wy[b] * wz;
                    const long long row = (long long)(lz + e) * E1 * E0 + (long long)(ly + b) * E0 + lx;
#pragma unroll
                    for (int a = 0; a <= P; a++) {
                        const float w = Wx[a] * wyz;
                        for (int f = 0; f < nd; f++) {
                            const float v = c[f] * w;
                            if (v == 0.f) continue;
                            if (FIXED)
                                atomicAdd(tu + f * V + row + a,
                                          (unsigned long long)__double2ll_rn((double)v * kFixScale));
                            else
                                atomicAdd(tf + f * V + row + a, v);
                        }
                    }
                }
            }
        } else {
            int ix[P + 1], iy[P + 1], iz[P + 1];
#pragma unroll
            for (int i = 0; i <= P; i++) {
                ix[i] = wrapi(gx + i, g.nx);
                iy[i] = wrapi(gy + i, g.ny);
                iz[i] = wrapi(gz + i, g.nz);
            }
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
                        for (int f = 0; f < nd; f++) {
                            const float v = c[f] * w;
                            if (v == 0.f) continue;
                            if (FIXED)
                                atomicAdd(depfix + f * g.M + my + ix[a],
                                          (unsigned long long)__double2ll_rn((double)v * kFixScale));
                            else
                                atomicAdd(FIELD_PTR(dep, f, g.M) + 2 * (my + ix[a]), v);
                        }
                    }
                }
            }
        }
    }
    if (!staged) return;
    __syncthreads();
    const int npair = (nd + 1) >> 1;
    for (long long v = threadIdx.x; v < V; v += blockDim.x) {
        const int lz = (int)(v / ((long long)E1 * E0));
        const int rem = (int)(v - (long long)lz * E1 * E0);
        const int ly = rem / E0, lx = rem - ly * E0;
        const long long m = wrapi(s_ref[0] + s_min[0] + lx, g.nx) +
                            (long long)g.nx * (wrapi(s_ref[1] + s_min[1] + ly, g.ny) +
                                               (long long)g.ny * wrapi(s_ref[2] + s_min[2] + lz, g.nz));
        if (FIXED) {
            for (int f = 0; f < nd; f++) {
                const unsigned long long u = tu[f * V + v];
                if (u) atomicAdd(depfix + f * g.M + m, u);
            }
        } else {
            for (int t = 0; t < npair; t++) {
                const float a0 = tf[(2 * t) * V + v];
                const float a1 = (2 * t + 1 < nd) ? tf[(2 * t + 1) * V + v] : 0.f;
                if (a0 != 0.f && a1 != 0.f) atomicAdd(dep + t * g.M + m, make_float2(a0, a1));
                else if (a0 != 0.f) atomicAdd(&dep[t * g.M + m].x, a0);
                else if (a1 != 0.f) atomicAdd(&dep[t * g.M + m].y, a1);
            }
        }
    }
}

template <int P>
static void dep_launch(const Geom &g, const ParticleParams &pp, const float *X0, const float *X1,
                       const long long *d_step, const uint32_t *pflags, const float *q, float2 *dep,
                       unsigned long long *depfix, cudaStream_t st)
{
    const int nb = (pp.N + kDepPB - 1) / kDepPB;
    if (depfix)
        k_deposit_tiled<P, true><<<nb, 256, kDepSmemFixed, st>>>(g, pp.N, pp.quirk4, pp.nd, pp.dchan_charge, X0, X1,
                                                                 d_step, pflags, q, dep, depfix, kDepSmemFixed);
    else
        k_deposit_tiled<P, false><<<nb, 256, kDepSmemFast, st>>>(g, pp.N, pp.quirk4, pp.nd, pp.dchan_charge, X0, X1,
                                                                 d_step, pflags, q, dep, depfix, kDepSmemFast);
}

void init_deposit_attributes()
{
#define TILD_DA(P)                                                                                       \
    cudaFuncSetAttribute(k_deposit_tiled<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDepSmemFixed); \
    cudaFuncSetAttribute(k_deposit_tiled<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDepSmemFast)
    TILD_DA(0);
    TILD_DA(1);
    TILD_DA(2);
    TILD_DA(3);
    TILD_DA(4);
#undef TILD_DA
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
