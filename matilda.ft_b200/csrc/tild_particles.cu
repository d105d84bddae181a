// tild_particles.cu -- particle pass (gather + bonds + GJF/EM), RNG and thermo
// reductions (sm_100a).
#include "tild_stencil.cuh"

#include <curand_kernel.h>

#include <cmath>

namespace tild {

// =====================================================================================
// Particle pass: bonds (ps_deviceBonds.cu:7-79), grid->particle gather per force group
// in group order (device_utils.cu:358-461), then GJF (ps_integratorGJF.cu:102-163) or
// EM (ps_integratorEM.cu:39-82).  x_t is read from Xc; the GJF old position x_{t-1} is
// read from Xn and replaced by x_{t+1} (same thread), so no copy of x is ever made.
// =====================================================================================
__device__ __forceinline__ void philox_round(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
}

// Philox4x32-10 (Salmon et al., SC'11): counter (step, particle id, 0, 0), key = seed.
__device__ __forceinline__ void philox_normals3(unsigned long long seed, uint32_t step, uint32_t id,
                                                float out[3])
{
    uint32_t c[4] = {step, id, 0u, 0u};
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; r++) {
        philox_round(c, k0, k1);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    const float s = 2.3283064365386963e-10f;  // 2^-32
    const float u0 = fmaf((float)c[0], s, 0.5f * s), u1 = fmaf((float)c[1], s, 0.5f * s);
    const float u2 = fmaf((float)c[2], s, 0.5f * s), u3 = fmaf((float)c[3], s, 0.5f * s);
    const float r0 = sqrtf(-2.f * logf(u0)), r1 = sqrtf(-2.f * logf(u2));
    float sn, cs;
    sincospif(2.f * u1, &sn, &cs);
    out[0] = r0 * cs;
    out[1] = r0 * sn;
    out[2] = r1 * cospif(2.f * u3);
}

template <int P>
__global__ void __launch_bounds__(256) k_particles(Geom g, const ParticleParams *__restrict__ ppd, int N,
                                                   float *__restrict__ X0, float *__restrict__ X1,
                                                   float *__restrict__ noise,
                                                   const uint32_t *__restrict__ pflags,
                                                   const float *__restrict__ q, const uint8_t *__restrict__ nb,
                                                   const int *__restrict__ partner,
                                                   const uint8_t *__restrict__ btype,
                                                   const float4 *__restrict__ rec,
                                                   const int *__restrict__ orig_id,
                                                   curandState *__restrict__ rng,
                                                   const long long *__restrict__ d_step,
                                                   float *__restrict__ fout, int integrate)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const ParticleParams &pp = *ppd;
    const long long step = *d_step;
    const float *__restrict__ Xc = (step & 1) ? X1 : X0;   // x_t
    float *__restrict__ Xn = (step & 1) ? X0 : X1;         // x_{t-1} in, x_{t+1} out
    const uint32_t fl = pflags[p];
    const float x0 = Xc[3 * p], x1 = Xc[3 * p + 1], x2 = Xc[3 * p + 2];
    float f0 = 0.f, f1 = 0.f, f2 = 0.f;

    // 1. bonds
    const int nbp = nb ? nb[p] : 0;
    for (int b = 0; b < nbp; b++) {
        const int o = partner[p * pp.maxb + b];
        const int t = btype[p * pp.maxb + b];
        float dr[3] = {x0 - Xc[3 * o], x1 - Xc[3 * o + 1], x2 - Xc[3 * o + 2]};
        float mdr2 = 0.f;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if (dr[j] > g.Lh[j]) dr[j] -= g.L[j];
            else if (dr[j] < -g.Lh[j]) dr[j] += g.L[j];
            mdr2 = __fmaf_rn(dr[j], dr[j], mdr2);
        }
        float mf = 0.f;
        if (mdr2 > 1.0e-4f) {
            const float mdr = sqrtf(mdr2);
            if (pp.bstyle[t] == 0) {
                mf = 2.0f * pp.bk[t] * (mdr - pp.breq[t]) / mdr;
            } else {
                const float u = mdr / pp.breq[t];
                mf = 2.0f * pp.bk[t] * mdr / (1.f - u * u) / mdr;
            }
        }
        f0 = __fmaf_rn(-mf, dr[0], f0);
        f1 = __fmaf_rn(-mf, dr[1], f1);
        f2 = __fmaf_rn(-mf, dr[2], f2);
    }

    // 2. grid forces, force groups in the reference's group order
    const uint32_t fm = (fl >> 8) & 0xffu;
    if (fm) {
        float Wx[P + 1], Wy[P + 1], Wz[P + 1];
        int ix[P + 1], iy[P + 1], iz[P + 1];
        const int gx = stencil_axis<P>(x0, g.dxf[0], pp.quirk4, Wx);
        const int gy = stencil_axis<P>(x1, g.dxf[1], pp.quirk4, Wy);
        const int gz = stencil_axis<P>(x2, g.dxf[2], pp.quirk4, Wz);
#pragma unroll
        for (int i = 0; i <= P; i++) {
            ix[i] = wrapi(gx + i, g.nx);
            iy[i] = wrapi(gy + i, g.ny);
            iz[i] = wrapi(gz + i, g.nz);
        }
        const long long plane = (long long)g.nx * g.ny;
        for (int fg = 0; fg < pp.nfg; fg++) {
            if (!((fm >> fg) & 1u)) continue;
            const float4 *rf = rec + (long long)fg * g.M;
            float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll 1
            for (int e = 0; e <= P; e++) {
                const float wz = sel<P>(Wz, e);
                const float4 *rz = rf + plane * sel<P>(iz, e);
#pragma unroll
                for (int b = 0; b <= P; b++) {
                    const float4 *ry = rz + (long long)g.nx * iy[b];
                    const float wyz = Wy[b] * wz;
#pragma unroll
                    for (int a = 0; a <= P; a++) {
                        const float w = Wx[a] * wyz;
                        const float4 r = __ldg(ry + ix[a]);
                        a0 = __fmaf_rn(r.x, w, a0);
                        a1 = __fmaf_rn(r.y, w, a1);
                        a2 = __fmaf_rn(r.z, w, a2);
                    }
                }
            }
            if ((pp.fg_qweighted >> fg) & 1u) {
                const float qp = q[p];
                f0 = __fmaf_rn(a0, qp, f0);
                f1 = __fmaf_rn(a1, qp, f1);
                f2 = __fmaf_rn(a2, qp, f2);
            } else {
                f0 += a0;
                f1 += a1;
                f2 += a2;
            }
        }
    }
    if (fout) {
        fout[3 * p] = f0;
        fout[3 * p + 1] = f1;
        fout[3 * p + 2] = f2;
    }
    if (!integrate) return;

    // 3. integrator
    const int slot = (fl >> 16) & 0xfu;
    if (slot == kNoIntegrator) {
        Xn[3 * p] = x0;
        Xn[3 * p + 1] = x1;
        Xn[3 * p + 2] = x2;
        return;
    }
    float nz3[3];
    if (pp.rng_compat) {
        curandState st = rng[p];
        nz3[0] = curand_normal(&st);
        nz3[1] = curand_normal(&st);
        nz3[2] = curand_normal(&st);
        rng[p] = st;
    } else {
        philox_normals3(pp.seed, (uint32_t)step, (uint32_t)orig_id[p], nz3);
    }
    const float xs[3] = {x0, x1, x2}, fs[3] = {f0, f1, f2};
    if (pp.integ_kind[slot] == 0) {
        const int t = (fl >> 20) & 0xfu;
        const TypeCoef cf = pp.coef[slot][t];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int ai = 3 * p + j;
            const float nn = cf.noiseMag * nz3[j];
            const float xt = xs[j];
            float xo = Xn[ai];
            if (xo - xt > g.L[j] / 2.0f) xo -= g.L[j];
            else if (xo - xt < -g.L[j] / 2.0f) xo += g.L[j];
            float xv = 2.0f * cf.b * xt - cf.a * xo + cf.bdt2m * fs[j] + cf.bdt2m2 * (nn + noise[ai]);
            noise[ai] = nn;
            if (xv > g.L[j]) xv -= g.L[j];
            else if (xv < 0.0f) xv += g.L[j];
            Xn[ai] = xv;
        }
    } else {
        const float dt = pp.em_delt[slot], nm = pp.em_noise[slot];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            float xv = xs[j] + dt * fs[j] + nm * nz3[j];
            if (xv > g.L[j]) xv -= g.L[j];
            else if (xv < 0.0f) xv += g.L[j];
            Xn[3 * p + j] = xv;
        }
    }
}

__global__ void k_tick(long long *d_step) { *d_step += 1; }

// curand_init(seed, particle, 0) per particle (device_utils.cu:465-472).
__global__ void k_rng_init(curandState *st, const int *orig_id, int n, unsigned long long seed)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    curand_init(seed, (unsigned long long)orig_id[p], 0ull, &st[p]);
}

// Per-particle bond energy and virial (ps_deviceBonds.cu:85-171, including its
// minimum-image threshold 0.5*Lh), summed per block in FP64: cols = e, vir[6].
__global__ void __launch_bounds__(256) k_bond_energy(Geom g, const ParticleParams *__restrict__ ppd, int N,
                                                     const float *__restrict__ X0, const float *__restrict__ X1,
                                                     const long long *__restrict__ d_step,
                                                     const uint8_t *__restrict__ nb,
                                                     const int *__restrict__ partner,
                                                     const uint8_t *__restrict__ btype,
                                                     double *__restrict__ partials)
{
    __shared__ double red[8][7];
    const ParticleParams &pp = *ppd;
    const float *__restrict__ X = (*d_step & 1) ? X1 : X0;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    if (p < N && nb) {
        float e = 0.f, vir[6] = {0, 0, 0, 0, 0, 0};
        for (int b = 0; b < nb[p]; b++) {
            const int o = partner[p * pp.maxb + b], t = btype[p * pp.maxb + b];
            float dr[3], mdr2 = 0.f, mf = 0.f;
            for (int j = 0; j < 3; j++) {
                dr[j] = X[3 * p + j] - X[3 * o + j];
                if (dr[j] > 0.5f * g.Lh[j]) dr[j] -= g.L[j];
                else if (dr[j] < -0.5f * g.Lh[j]) dr[j] += g.L[j];
                mdr2 = __fmaf_rn(dr[j], dr[j], mdr2);
            }
            if (mdr2 > 1.0e-4f) {
                const float mdr = sqrtf(mdr2);
                if (pp.bstyle[t] == 0) {
                    const float arg = mdr - pp.breq[t];
                    mf = 2.0f * pp.bk[t] * arg / mdr;
                    e += pp.bk[t] * arg * arg;
                } else if (mdr / pp.breq[t] < 1.f) {
                    const float u = mdr / pp.breq[t];
                    const float arg = 1.f / (1.f - u * u);
                    mf = 2.0f * pp.bk[t] * arg;
                    e += mf * mdr;
                }
            }
            vir[0] += -mf * dr[0] * dr[0];
            vir[1] += -mf * dr[1] * dr[1];
            vir[2] += -mf * dr[2] * dr[2];
            vir[3] += -mf * dr[0] * dr[1];
            vir[4] += -mf * dr[0] * dr[2];
            vir[5] += -mf * dr[1] * dr[2];
        }
        acc[0] = e;
        for (int c = 0; c < 6; c++) acc[c + 1] = vir[c];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = 0; c < 7; c++) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w][threadIdx.x];
        partials[(long long)blockIdx.x * 7 + threadIdx.x] = s;
    }
}

// Deterministic sum of per-block partials: out[c] = sum_b partials[b*ncols + c].
__global__ void k_reduce_partials(const double *partials, int nblocks, int ncols, double *out)
{
    __shared__ double red[256];
    for (int c = 0; c < ncols; c++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(long long)b * ncols + c];
        red[threadIdx.x] = s;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[c] = red[0];
        __syncthreads();
    }
}


// ---- launchers ----
template <int P>
static void part_launch(const Geom &g, const ParticleParams *ppd, int N, float *X0, float *X1, float *noise,
                        const uint32_t *pflags, const float *q, const uint8_t *nb, const int *partner,
                        const uint8_t *btype, const float4 *rec, const int *orig_id, void *rng,
                        const long long *d_step, float *fout, int integrate, cudaStream_t st)
{
    const int bs = 256, nbk = (N + bs - 1) / bs;
    k_particles<P><<<nbk, bs, 0, st>>>(g, ppd, N, X0, X1, noise, pflags, q, nb, partner, btype, rec, orig_id,
                                       reinterpret_cast<curandState *>(rng), d_step, fout, integrate);
}

cudaError_t launch_particles(const Geom &g, const ParticleParams &pp, const ParticleParams *ppd, float *X0,
                             float *X1, float *noise, const uint32_t *pflags, const float *q, const uint8_t *nb,
                             const int *partner, const uint8_t *btype, const float4 *rec, const int *orig_id,
                             void *rng_states, const long long *d_step, float *fout, int integrate,
                             cudaStream_t st)
{
    if (pp.N == 0) return cudaSuccess;
#define TILD_PL(P) part_launch<P>(g, ppd, pp.N, X0, X1, noise, pflags, q, nb, partner, btype, rec, orig_id, \
                                  rng_states, d_step, fout, integrate, st)
    switch (pp.order) {
        case 0: TILD_PL(0); break;
        case 1: TILD_PL(1); break;
        case 2: TILD_PL(2); break;
        case 3: TILD_PL(3); break;
        default: TILD_PL(4); break;
    }
#undef TILD_PL
    return cudaGetLastError();
}

cudaError_t launch_tick(long long *d_step, cudaStream_t st)
{
    k_tick<<<1, 1, 0, st>>>(d_step);
    return cudaGetLastError();
}

size_t rng_state_bytes() { return sizeof(curandState); }

cudaError_t launch_rng_init(void *states, const int *orig_id, int n, unsigned long long seed, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    k_rng_init<<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<curandState *>(states), orig_id, n, seed);
    return cudaGetLastError();
}

cudaError_t launch_bond_energy(const Geom &g, const ParticleParams &pp, const ParticleParams *ppd, const float *X0,
                               const float *X1, const long long *d_step, const uint8_t *nb, const int *partner,
                               const uint8_t *btype, double *partials, int *nblocks_out, cudaStream_t st)
{
    const int nbk = pp.N > 0 ? (pp.N + 255) / 256 : 1;
    k_bond_energy<<<nbk, 256, 0, st>>>(g, ppd, pp.N, X0, X1, d_step, nb, partner, btype, partials);
    if (nblocks_out) *nblocks_out = nbk;
    return cudaGetLastError();
}

cudaError_t launch_reduce_partials(const double *partials, int nblocks, int ncols, double *out, cudaStream_t st)
{
    k_reduce_partials<<<1, 256, 0, st>>>(partials, nblocks, ncols, out);
    return cudaGetLastError();
}

}  // namespace tild
