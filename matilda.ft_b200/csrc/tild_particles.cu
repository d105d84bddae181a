// tild_particles.cu -- particle pass (gather + bonds + GJF/EM), RNG and thermo
// reductions (sm_100a).
#include "tild_stencil.cuh"

#include <curand_kernel.h>

#include <algorithm>
#include <cmath>
#include <cstring>

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

// Bond force on particle p (ps_deviceBonds.cu:7-79): minimum image with Lh, skipped for
// r^2 <= 1e-4, harmonic mf = 2k(r - req)/r or FENE; f -= mf * dr over every stored partner.
// The reference keeps a padded [N x MAXBONDS] partner list; here the partners form a CSR
// list (row offsets brow[N+1]), renumbered and re-packed by every spatial sort, so a
// branched molecule's high-degree particles cost no padding for all the others.
// A bond across the periodic boundary is measured as (x_p - L) - x_o or x_p - (x_o - L):
// the coordinate above L/2 is shifted first, which is exact in FP32, so the short image
// vector is rounded once at its own magnitude instead of at the box length's (the
// reference's x_p - x_o then -L loses up to half an ulp of L, ~2e-6 at L = 60).
__device__ __forceinline__ void bond_force(const Geom &g, const ParticleParams &pp, int p, const float *x,
                                           const float *__restrict__ Xc, const int *__restrict__ brow,
                                           const int *__restrict__ partner, const uint8_t *__restrict__ btype,
                                           float *f)
{
    const int k0 = brow ? brow[p] : 0, k1 = brow ? brow[p + 1] : 0;
    for (int k = k0; k < k1; k++) {   // this particle's row of the CSR bond list
        const int o = partner[k];
        const int t = btype[k];
        float dr[3];
        float mdr2 = 0.f;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const float xo = Xc[3 * o + j];
            dr[j] = x[j] - xo;
            if (dr[j] > g.Lh[j]) dr[j] = (x[j] - g.L[j]) - xo;
            else if (dr[j] < -g.Lh[j]) dr[j] = x[j] - (xo - g.L[j]);
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
#pragma unroll
        for (int j = 0; j < 3; j++) f[j] = __fmaf_rn(-mf, dr[j], f[j]);
    }
}

// One angle (ps_deviceAngles.cu:26-120): the two bond vectors from the middle particle j
// (minimum image with Lh), cos(theta), and the forces fi on i and fk on k (the middle
// particle takes -(fi + fk)); wlc U = k (1 + cos), harmonic U = k (theta - theta_eq)^2.
// Returns false when the reference skips the angle (a bond shorter than 1e-2, or
// |cos| > 1 for the harmonic style); e and the vectors are filled otherwise.
__device__ __forceinline__ bool angle_terms(const Geom &g, const ParticleParams &pp, const float *__restrict__ X,
                                            int ai, int aj, int ak, int atp, float *rij, float *rkj, float *fi,
                                            float *fk, float &e)
{
    float mrij2 = 0.f, mrkj2 = 0.f;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        rij[j] = X[3 * ai + j] - X[3 * aj + j];
        if (rij[j] > g.Lh[j]) rij[j] -= g.L[j];
        else if (rij[j] < -g.Lh[j]) rij[j] += g.L[j];
        mrij2 = __fmaf_rn(rij[j], rij[j], mrij2);
    }
    if (mrij2 < 1.0e-4f) return false;
    const float mrij = sqrtf(mrij2);
#pragma unroll
    for (int j = 0; j < 3; j++) {
        rkj[j] = X[3 * ak + j] - X[3 * aj + j];
        if (rkj[j] > g.Lh[j]) rkj[j] -= g.L[j];
        else if (rkj[j] < -g.Lh[j]) rkj[j] += g.L[j];
        mrkj2 = __fmaf_rn(rkj[j], rkj[j], mrkj2);
    }
    if (mrkj2 < 1.0e-4f) return false;
    const float mrkj = sqrtf(mrkj2);
    float dot = 0.f;
#pragma unroll
    for (int j = 0; j < 3; j++) dot = __fmaf_rn(rij[j], rkj[j], dot);
    const float cos_th = dot / mrij / mrkj;
    const float kang = pp.ak[atp];
    if (pp.astyle[atp] == 0) {   // wlc
        e = kang * (1.0f + cos_th);
#pragma unroll
        for (int j = 0; j < 3; j++) {
            fi[j] = -kang * (rkj[j] / mrij / mrkj - cos_th * rij[j] / mrij2);
            fk[j] = -kang * (rij[j] / mrkj / mrij - cos_th * rkj[j] / mrkj2);
        }
        return true;
    }
    if (cos_th < -1.f || cos_th > 1.f) return false;
    const float theta = acosf(cos_th);
    const float denom = sqrtf(1.f - cos_th * cos_th);
    const float isin = denom > 1.0e-4f ? (float)(1.0 / (double)denom) : 0.f;
    const float dtheta = theta - pp.atheq[atp];
    const float du = 2.f * kang * dtheta;
    e = kang * dtheta * dtheta;
#pragma unroll
    for (int j = 0; j < 3; j++) {
        fi[j] = du * isin * (rkj[j] / mrij / mrkj - cos_th * rij[j] / mrij2);
        fk[j] = du * isin * (rij[j] / mrij / mrkj - cos_th * rkj[j] / mrkj2);
    }
    return true;
}

// Angle force on particle p summed over its angles, added after the bonds (the order of
// d_bonds then d_angles, PS_Box.cu:245-254).
__device__ __forceinline__ void angle_force(const Geom &g, const ParticleParams &pp, int p, const float *__restrict__ X,
                                            const AngleArrays &aa, float *f)
{
    const int nap = aa.na[p];
    float lf[3] = {0.f, 0.f, 0.f};
    for (int i = 0; i < nap; i++) {
        const int b = (p * pp.maxa + i) * 3;
        const int ai = aa.ang[b], aj = aa.ang[b + 1], ak = aa.ang[b + 2];
        float rij[3], rkj[3], fi[3], fk[3], e;
        if (!angle_terms(g, pp, X, ai, aj, ak, aa.atype[p * pp.maxa + i], rij, rkj, fi, fk, e)) continue;
#pragma unroll
        for (int j = 0; j < 3; j++) {
            if (p == ai) lf[j] += fi[j];
            else if (p == aj) lf[j] -= fi[j] + fk[j];
            else if (p == ak) lf[j] += fk[j];
        }
    }
#pragma unroll
    for (int j = 0; j < 3; j++) f[j] += lf[j];
}

// GJF (ps_integratorGJF.cu:102-163) or EM (ps_integratorEM.cu:39-82) update of particle p;
// x_{t-1} is read from Xn and replaced by x_{t+1}.
__device__ __forceinline__ void integrate(const Geom &g, const ParticleParams &pp, int p, uint32_t fl,
                                          const float *xs, const float *fs, float *__restrict__ Xn,
                                          float *__restrict__ noise, const float *xold, const float *nold, int oid,
                                          curandState *__restrict__ rng, long long step)
{
    const int slot = (fl >> 16) & 0xfu;
    if (slot == kNoIntegrator) {
        Xn[3 * p] = xs[0];
        Xn[3 * p + 1] = xs[1];
        Xn[3 * p + 2] = xs[2];
        return;
    }
    float nz3[3];
    if (pp.rng_compat) {   // one normal per dimension, as the reference draws them
        curandState st = rng[p];
        nz3[0] = curand_normal(&st);
        nz3[1] = curand_normal(&st);
        nz3[2] = pp.dim == 3 ? curand_normal(&st) : 0.f;
        rng[p] = st;
    } else {
        philox_normals3(pp.seed, (uint32_t)step, (uint32_t)oid, nz3);
        if (pp.dim == 2) nz3[2] = 0.f;   // z (always 0 in a 2-D box) takes no noise
    }
    if (pp.integ_kind[slot] == 0) {
        const int t = (fl >> 20) & 0xfu;
        const TypeCoef cf = pp.coef[slot][t];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int ai = 3 * p + j;
            const float nn = cf.noiseMag * nz3[j];
            const float xt = xs[j];
            float xo = xold[j];
            if (xo - xt > g.L[j] / 2.0f) xo -= g.L[j];
            else if (xo - xt < -g.L[j] / 2.0f) xo += g.L[j];
            float xv = 2.0f * cf.b * xt - cf.a * xo + cf.bdt2m * fs[j] + cf.bdt2m2 * (nn + nold[j]);
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

// Harmonic walls (d_wallHarmonicForce, ps_potentialWall.cu:92-108): k (pos - x_n) along
// the wall's axis on the forbidden side sign (pos - x_n) > 0; e: the energy k disp^2 / 2.
__device__ __forceinline__ void wall_terms(const ParticleParams &pp, uint32_t fl, const float *x, float *f, float *e)
{
    for (int w = 0; w < pp.nwall; w++) {
        if (!((fl >> (24 + w)) & 1u)) continue;
        const int a = pp.wall_axis[w];
        const float disp = pp.wall_pos[w] - x[a];
        if ((float)pp.wall_sign[w] * disp > 0.0f) {
            if (f) f[a] += pp.wall_k[w] * disp;
            if (e) e[w] = 0.5f * pp.wall_k[w] * disp * disp;
        }
    }
}

__device__ __forceinline__ void cp_async16p(void *smem_dst, const void *gsrc)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}

// ---- TMA staging of the force-record box (cp.async.bulk.tensor with an mbarrier) ----
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *mb)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mb)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// One thread: the box of force group f whose first point is grid point (x, y, z)
// (unwrapped; points outside the grid arrive as zeros) into dst, completing on mb.
__device__ __forceinline__ void tma_load_records(float4 *dst, const CUtensorMap *map, int x, int y, int z, int f,
                                                 unsigned long long *mb, unsigned bytes)
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // earlier reads of dst come first
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n"
                 ::"r"(smem_u32(mb)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n"
                 ::"r"(smem_u32(dst)), "l"(map), "r"(0), "r"(x), "r"(y), "r"(z), "r"(f), "r"(smem_u32(mb))
                 : "memory");
}

// Bounded wait for phase `phase` of mb: false if it did not complete within the limit.
__device__ __forceinline__ bool mbar_wait(unsigned long long *mb, unsigned phase)
{
    for (int i = 0; i < (1 << 22); i++) {
        unsigned ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(ok) : "r"(smem_u32(mb)), "r"(phase) : "memory");
        if (ok) return true;
    }
    return false;
}

// The cubic stencil (P = 3) is summed in the order of the 8-lane tile gather on every path,
// so that every path gives the same bits: lane k of a particle's eight (column a = k & 3,
// rows b = 2 (k >> 2) + i) chains its eight points over the planes e, then i, with one FMA
// each, w = Wx[a] (Wy[b] Wz[e]); the eight lane sums then add as the tree
// ((s0 + s1) + (s2 + s3)) + ((s4 + s5) + (s6 + s7)).  fetch(a, b, e, r) gives the NC
// components r[] of one stencil point; out[] receives the NC sums.
template <int NC, typename Fetch>
__device__ __forceinline__ void sum8_cubic(const float *Wx, const float *Wy, const float *Wz, Fetch fetch, float *out)
{
    float lo[NC], hi[NC], cur[NC];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        float sk[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) sk[c] = 0.f;
        const int a = k & 3, bh = k >> 2;
#pragma unroll
        for (int e = 0; e < 4; e++)
#pragma unroll
            for (int i = 0; i < 2; i++) {
                const int b = 2 * bh + i;
                const float w = Wx[a] * (Wy[b] * Wz[e]);
                float r[NC];
                fetch(a, b, e, r);
#pragma unroll
                for (int c = 0; c < NC; c++) sk[c] = __fmaf_rn(r[c], w, sk[c]);
            }
#pragma unroll
        for (int c = 0; c < NC; c++) {
            if ((k & 1) == 0) cur[c] = sk[c];
            else cur[c] = cur[c] + sk[c];             // s0 + s1, s2 + s3, ...
        }
        if (k == 1 || k == 5) {
#pragma unroll
            for (int c = 0; c < NC; c++) lo[c] = cur[c];
        } else if (k == 3 || k == 7) {
#pragma unroll
            for (int c = 0; c < NC; c++) cur[c] = lo[c] + cur[c];   // (s0 + s1) + (s2 + s3), ...
            if (k == 3) {
#pragma unroll
                for (int c = 0; c < NC; c++) hi[c] = cur[c];
            }
        }
    }
#pragma unroll
    for (int c = 0; c < NC; c++) out[c] = hi[c] + cur[c];
}

constexpr int kPartBox = 4096;     // float4 records staged per force group (64 KB)
constexpr int kPartWindow = 256;   // slots per CTA when the particles are not sorted

// Gather of one force group's records at a particle's stencil straight from global memory
// (device_utils.cu:358-461), summed in the same order as the shared-memory gather so the
// two paths give the same bits.  UNROLL: all (P+1)^3 loads in flight at once (the direct
// gathers of a whole CTA), else one plane at a time (the few helpers' gathers).
template <int P, bool UNROLL>
__device__ __forceinline__ void gather_global(const Geom &g, const float4 *__restrict__ rf, const int *gs,
                                              const float *Wx, const float *Wy, const float *Wz, float *acc)
{
    // a true modulo past one box length: a position outside [0, L) still reads the grid
    auto wrap = [](int v, int n) { return wrapi(v, n); };
    if constexpr (P == 3) {
        sum8_cubic<3>(Wx, Wy, Wz, [&](int a, int b, int e, float *r) {
            const float4 v = __ldg(rf + (long long)g.nx * ((long long)g.ny * wrap(gs[2] + e, g.nz) + wrap(gs[1] + b, g.ny)) +
                                   wrap(gs[0] + a, g.nx));
            r[0] = v.x;
            r[1] = v.y;
            r[2] = v.z;
        }, acc);
    } else {
        float2 a01 = make_float2(0.f, 0.f);
        float a2 = 0.f;
#pragma unroll(UNROLL ? P + 1 : 1)
        for (int e = 0; e <= P; e++) {
            const float wz = sel<P>(Wz, e);
            const float4 *rz = rf + (long long)g.nx * g.ny * wrap(gs[2] + e, g.nz);
#pragma unroll
            for (int b = 0; b <= P; b++) {
                const float4 *ry = rz + (long long)g.nx * wrap(gs[1] + b, g.ny);
                const float wyz = Wy[b] * wz;
#pragma unroll
                for (int a = 0; a <= P; a++) {
                    const float w = Wx[a] * wyz;
                    const float4 r = __ldg(ry + wrap(gs[0] + a, g.nx));
                    a01 = __ffma2_rn(make_float2(r.x, r.y), make_float2(w, w), a01);
                    a2 = __fmaf_rn(r.z, w, a2);
                }
            }
        }
        acc[0] = a01.x;
        acc[1] = a01.y;
        acc[2] = a2;
    }
}

// Force of one group added to a particle's grid force, in group order: q-weighted for the
// 'charges' group (device_utils.cu:412-461 multiplies by the charge).
__device__ __forceinline__ void add_group(float *fg, const float *a, bool qw, float qp)
{
#pragma unroll
    for (int j = 0; j < 3; j++) fg[j] = qw ? __fmaf_rn(a[j], qp, fg[j]) : fg[j] + a[j];
}

constexpr int kPartOut = 32;   // particles per pass gathered from global memory by helpers
// threads of a particle-pass CTA at most: the launch bound that caps registers at 72
// (a tile with more particles takes more than one pass)
constexpr int kPartThreadsMax = 448;

// Planar gather (device_utils.cu:358-461): every particle's grid force, the sum over its
// force groups in group order, into fgrid[3p].  One particle per thread and pass, over one
// Morton tile of particles (or a window of slots); the records are planar, rec[F][M].
//
// Sorted tiles stage a fixed box per force group in shared memory: the grid points of the
// tile's block of bricks (where its particles were at the last sort), widened by the
// stencil and by `tc.margin` cells for the drift since.  A particle whose stencil has
// drifted out of the box is gathered from global memory, before the staging wait, by a
// helper thread (thread o for the pass's o-th such particle); its owner adds the result in
// group order like any other, so the sums do not depend on which path served them.
// TMA: sorted tiles stage their boxes with one TMA load (the host selects this instantiation
// when it holds a descriptor for the tiles' box); else with per-thread cp.async copies.
// This kernel serves 2-D boxes, more than two force groups, unsorted particles and the
// direct gathers; the paired tile gather below serves the rest.
template <int P, bool TMA>
__global__ void __launch_bounds__(kPartThreadsMax, 2) k_gather_planar(Geom g, const ParticleParams *__restrict__ ppd, int N,
                                                      const float *__restrict__ X0, const float *__restrict__ X1,
                                                      const uint32_t *__restrict__ pflags,
                                                      const float *__restrict__ q, const float4 *__restrict__ rec,
                                                      const long long *__restrict__ d_step, float *__restrict__ fgrid,
                                                      TileCfg tc, int box_cap,
                                                      const __grid_constant__ CUtensorMap rmap, int *__restrict__ err)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    // the box starts on a 128-byte boundary of the shared window (a TMA destination)
    float4 *box = reinterpret_cast<float4 *>(smraw + ((128u - (smem_u32(smraw) & 127u)) & 127u));
    __shared__ TileShared ts;
    __shared__ float Ao[kPartOut][kMaxFGroups][3];
    __shared__ int outP[kPartOut];
    __shared__ int nout;
    __shared__ int deal_src[kPartThreadsMax];   // per warp: the lane whose particle a lane gathers
    __shared__ __align__(8) unsigned long long tma_bar;   // completion of a TMA box load
    const ParticleParams &pp = *ppd;
    const long long step = *d_step;
    const float *__restrict__ Xc = (step & 1) ? X1 : X0;   // x_t
    const int nn[3] = {g.nx, g.ny, g.nz};
    int r0, r1;
    tile_range(tc, N, kPartWindow, r0, r1);
    // the tile's fixed box: stencil origins lo[j] .. lo[j] + span[j]
    int lo[3] = {0, 0, 0}, span[3] = {-1, -1, -1}, E[3] = {0, 0, 0};
    bool staged = false;
    if (tc.start && !tc.direct) {
        tile_box<P>(tc, nn, lo, span, E);
        staged = E[0] <= kMaxBoxEdge && E[1] <= kMaxBoxEdge && E[2] <= kMaxBoxEdge &&
                 (long long)((((E[0] | 1) * E[1]) | 1)) * E[2] <= box_cap;
    }
    // The box arrives by one TMA load of the fixed box te[] (odd edges, so the dense
    // pitches stay odd), or by per-thread cp.async copies with odd pitches.  A box that
    // leaves the grid gets its periodic images by cp.async after the TMA load.
    const bool use_tma = TMA && staged;
    const int E0 = TMA ? tc.te[0] : (E[0] | 1);
    const int E01 = TMA ? tc.te[0] * tc.te[1] : ((E0 * E[1]) | 1);
    const bool wraps = use_tma && (lo[0] < 0 || lo[1] < 0 || lo[2] < 0 || lo[0] + tc.te[0] > g.nx ||
                                   lo[1] + tc.te[1] > g.ny || lo[2] + tc.te[2] > g.nz);
    unsigned tphase = 0u;
    if (staged) {
        if (threadIdx.x < 3) {
            ts.ref[threadIdx.x] = lo[threadIdx.x];
            ts.lo[threadIdx.x] = 0;
        }
        if (use_tma && threadIdx.x == 0) mbar_init(&tma_bar);
        __syncthreads();
        tile_tables(ts, g.nx, g.ny, g.nz, use_tma ? tc.te : E);
    }
    const int te[3] = {tc.te[0], tc.te[1], tc.te[2]};
    const unsigned tbytes = (unsigned)(E01 * te[2]) * 16u;
// start the copy of force group f's box (every thread calls it)
#define TILD_STAGE(f)                                                                                      \
    do {                                                                                                   \
        if (TMA) {                                                                                         \
            if (threadIdx.x == 0) tma_load_records(box, &rmap, lo[0], lo[1], lo[2], (f), &tma_bar, tbytes); \
        } else {                                                                                           \
            const float4 *rf_ = rec + (long long)(f) * g.M;                                                \
            tile_for_each(ts, E, E0, E01, [&](int v, int m) { cp_async16p(box + v, rf_ + m); });           \
            asm volatile("cp.async.commit_group;\n" ::: "memory");                                         \
        }                                                                                                  \
    } while (0)
// wait for it; a TMA box that leaves the grid then gets its periodic images by cp.async
#define TILD_STAGE_WAIT(f)                                                                                 \
    do {                                                                                                   \
        if (TMA) {                                                                                         \
            if (!mbar_wait(&tma_bar, tphase)) { /* record the failure, wait once more for the copy */      \
                if (threadIdx.x == 0) atomicAdd(err, 1);                                                   \
                mbar_wait(&tma_bar, tphase);                                                               \
            }                                                                                              \
            tphase ^= 1u;                                                                                  \
            if (wraps) {                                                                                   \
                const float4 *rf_ = rec + (long long)(f) * g.M;                                            \
                const int l0 = lo[0], l1 = lo[1], l2 = lo[2];                                              \
                tile_for_each_xyz(ts, te, E0, E01, [=](int v, int m, int lx, int ly, int lz) {             \
                    if ((unsigned)(l0 + lx) >= (unsigned)g.nx || (unsigned)(l1 + ly) >= (unsigned)g.ny ||  \
                        (unsigned)(l2 + lz) >= (unsigned)g.nz)                                             \
                        cp_async16p(box + v, rf_ + m);                                                     \
                });                                                                                        \
            }                                                                                              \
        }                                                                                                  \
        asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");                    \
    } while (0)
    for (int c0 = r0; c0 < r1; c0 += blockDim.x) {
        const int p = c0 + threadIdx.x;
        const bool act = p < r1;
        float x[3] = {0.f, 0.f, 0.f};
        uint32_t fl = 0u;
        if (act) {
            x[0] = Xc[3 * p];
            x[1] = Xc[3 * p + 1];
            x[2] = Xc[3 * p + 2];
            fl = pflags[p];
            if (q) asm volatile("prefetch.global.L2 [%0];" ::"l"(q + p));
        }
        const unsigned fm = (fl >> 8) & 0xffu;
        int gs[3] = {0, 0, 0};
        if (fm) {
            gs[0] = stencil_origin<P>(x[0], g, 0);
            gs[1] = stencil_origin<P>(x[1], g, 1);
            gs[2] = stencil_origin_z<P>(x[2], g);
        }
        if (threadIdx.x == 0) {
            nout = 0;
            ts.fm = 0u;
        }
        __syncthreads();
        // 1. box offset, or a slot in the helpers' list
        int d[3], slot = -1;
        bool inbox = false;
#pragma unroll
        for (int j = 0; j < 3; j++) d[j] = staged ? wrapi(gs[j] - lo[j], nn[j]) : 0;
        if (fm) {
            inbox = staged && d[0] <= span[0] && d[1] <= span[1] && d[2] <= span[2];
            if (staged && !inbox) {
                slot = atomicAdd(&nout, 1);
                if (slot < kPartOut) outP[slot] = p;
            }
        }
        unsigned fmor = fm;
        for (int o = 16; o > 0; o >>= 1) fmor |= __shfl_xor_sync(0xffffffffu, fmor, o);
        if ((threadIdx.x & 31) == 0 && fmor) atomicOr(&ts.fm, fmor);
        __syncthreads();
        const unsigned fmall = ts.fm;
        const int nhelp = min(nout, kPartOut);
        int fg = 0;
        while (fg < pp.nfg && !((fmall >> fg) & 1u)) fg++;
        // 2. start staging the first force group's box
        if (staged && fg < pp.nfg) TILD_STAGE(fg);
        // 3. helpers gather the out-of-box particles of every group from global memory
        if (threadIdx.x < nhelp) {
            const int ph = outP[threadIdx.x];
            const uint32_t flh = pflags[ph];
            float Hx[P + 1], Hy[P + 1], Hz[P + 1];
            int hs[3];
            hs[0] = stencil_fast<P>(Xc[3 * ph], g, 0, pp.quirk4, Hx);
            hs[1] = stencil_fast<P>(Xc[3 * ph + 1], g, 1, pp.quirk4, Hy);
            hs[2] = stencil_fast_z<P>(Xc[3 * ph + 2], g, pp.quirk4, Hz);
            for (int h = 0; h < pp.nfg; h++)
                if ((flh >> (8 + h)) & 1u) gather_global<P, false>(g, rec + (long long)h * g.M, hs, Hx, Hy, Hz, Ao[threadIdx.x][h]);
        }
        const int base = d[2] * E01 + d[1] * E0 + d[0];
        const float qp = (act && q) ? q[p] : 0.f;
        float Wx[P + 1], Wy[P + 1], Wz[P + 1];
        if (fm) {
            stencil_fast<P>(x[0], g, 0, pp.quirk4, Wx);
            stencil_fast<P>(x[1], g, 1, pp.quirk4, Wy);
            stencil_fast_z<P>(x[2], g, pp.quirk4, Wz);
        }
        // 4. deal the box gathers of the warp over its lanes by bank group.  A float4
        // record gather of a quarter warp takes one shared-memory wavefront only when its
        // eight lanes start at eight distinct 16-byte bank groups (record offset mod 8);
        // particles of a warp start at random offsets.  So the warp orders its particles
        // by that offset (class 8: nothing to gather from the box) and lane 8q + a takes
        // the particle at position 4a + q of the order: the eight lanes of a quarter warp
        // get positions four apart, which spreads them over the bank groups.  The lane
        // gathers for that particle with its stencil (shuffled in) and sends the result
        // back to the particle's own lane, which keeps every other access coalesced.
        const unsigned full = 0xffffffffu;
        const int lane = threadIdx.x & 31;
        int tp = lane, src = lane;
        if (staged) {
            const int r = inbox ? (base & 7) : 8;
            int below = 0;
#pragma unroll
            for (int v = 0; v < 8; v++) {
                const unsigned bl = __ballot_sync(full, r == v);
                below += v < r ? __popc(bl) : 0;
            }
            const int j = below + __popc(__match_any_sync(full, r) & ((1u << lane) - 1u));
            tp = ((j & 3) << 3) | (j >> 2);
            deal_src[(threadIdx.x & ~31) + tp] = lane;
            __syncwarp();
            src = deal_src[threadIdx.x];
            __syncwarp();
        }
        int bsrc = base;
        uint32_t flsrc = 0u;   // the groups this lane gathers from the box
        if (staged) {
            bsrc = __shfl_sync(full, base, src);
            flsrc = __shfl_sync(full, inbox ? fl : 0u, src);
#pragma unroll
            for (int i = 0; i <= P; i++) {
                Wx[i] = __shfl_sync(full, Wx[i], src);
                Wy[i] = __shfl_sync(full, Wy[i], src);
                Wz[i] = __shfl_sync(full, Wz[i], src);
            }
        }
        // 5. gather each force group in group order
        float fgv[3] = {0.f, 0.f, 0.f};
        bool first = true;
        for (; fg < pp.nfg; fg++) {
            if (!((fmall >> fg) & 1u)) continue;
            const float4 *rf = rec + (long long)fg * g.M;
            if (staged) {
                if (!first) {
                    __syncthreads();   // every gather from the previous group's box is done
                    TILD_STAGE(fg);
                }
                TILD_STAGE_WAIT(fg);
                __syncthreads();   // every thread's copies have landed (and the helpers' results)
            } else if (first) {
                __syncthreads();   // the helpers' results are visible
            }
            first = false;
            float2 a01 = make_float2(0.f, 0.f);
            float a2 = 0.f;
            if (P == 3 && ((flsrc >> (8 + fg)) & 1u)) {
                float sv[3];
                sum8_cubic<3>(Wx, Wy, Wz, [&](int a, int b, int e, float *r) {
                    const float4 v = box[bsrc + e * E01 + b * E0 + a];
                    r[0] = v.x;
                    r[1] = v.y;
                    r[2] = v.z;
                }, sv);
                a01 = make_float2(sv[0], sv[1]);
                a2 = sv[2];
            } else if ((flsrc >> (8 + fg)) & 1u) {   // the box gather of the particle dealt to this lane
#pragma unroll
                for (int e = 0; e <= P; e++) {
#pragma unroll
                    for (int b = 0; b <= P; b++) {
                        const float wyz = Wy[b] * Wz[e];
                        const int row = bsrc + e * E01 + b * E0;
#pragma unroll
                        for (int aa = 0; aa <= P; aa++) {
                            const float w = Wx[aa] * wyz;
                            const float4 r = box[row + aa];
                            a01 = __ffma2_rn(make_float2(r.x, r.y), make_float2(w, w), a01);   // paired FP32 FMA
                            a2 = __fmaf_rn(r.z, w, a2);
                        }
                    }
                }
            }
            float a[3] = {__shfl_sync(full, a01.x, tp), __shfl_sync(full, a01.y, tp), __shfl_sync(full, a2, tp)};
            if (!((fl >> (8 + fg)) & 1u)) continue;
            if (inbox) {
                // a[] holds this particle's box gather
            } else if (slot >= 0 && slot < kPartOut) {
                a[0] = Ao[slot][fg][0];
                a[1] = Ao[slot][fg][1];
                a[2] = Ao[slot][fg][2];
            } else if (staged) {   // own stencil again (the registers hold the dealt particle's)
                float Ux[P + 1], Uy[P + 1], Uz[P + 1];
                stencil_fast<P>(x[0], g, 0, pp.quirk4, Ux);
                stencil_fast<P>(x[1], g, 1, pp.quirk4, Uy);
                stencil_fast_z<P>(x[2], g, pp.quirk4, Uz);
                gather_global<P, true>(g, rf, gs, Ux, Uy, Uz, a);
            } else {
                gather_global<P, true>(g, rf, gs, Wx, Wy, Wz, a);
            }
            add_group(fgv, a, (pp.fg_qweighted >> fg) & 1u, qp);
        }
        if (act) {
            fgrid[3 * p] = fgv[0];
            fgrid[3 * p + 1] = fgv[1];
            fgrid[3 * p + 2] = fgv[2];
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");   // no copy outlives the pass
        __syncthreads();   // the box, nout and the helpers' results are reused by the next pass
    }
}

#undef TILD_STAGE
#undef TILD_STAGE_WAIT

// ---- tile gather over the paired records (RecLayout) ----
// Gather of one particle's stencil from the paired planes in global memory (the helpers'
// path for particles that drifted out of their tile's box), in the order and with the
// arithmetic of the box gather: a0 = (g0.x, g0.y), a1 = (g1.x, g1.y), a2 = (g0.z, g1.z);
// for one force group a0 = (x, y) and a1.x = z.
template <int P, int NFG>
__device__ __forceinline__ void gather_paired_global(const Geom &g, const RecLayout &rl, const int *gs,
                                                     const float *Wx, const float *Wy, const float *Wz,
                                                     float2 &a0, float2 &a1, float2 &a2)
{
    a0 = a1 = a2 = make_float2(0.f, 0.f);
    if constexpr (P == 3) {
        auto pt = [&](int a, int b, int e) {
            return ((long long)rl.py * (wrapi(gs[2] + e, g.nz) + rl.gl) + wrapi(gs[1] + b, g.ny) + rl.gl) * rl.px + rl.gl +
                   wrapi(gs[0] + a, g.nx);
        };
        if (NFG == 2) {
            float v[6];
            sum8_cubic<6>(Wx, Wy, Wz, [&](int a, int b, int e, float *r) {
                const long long m = pt(a, b, e);
                const float4 q4 = __ldg(rl.A + m);
                const float2 q2 = __ldg(rl.B + m);
                r[0] = q4.x;
                r[1] = q4.y;
                r[2] = q4.z;
                r[3] = q4.w;
                r[4] = q2.x;
                r[5] = q2.y;
            }, v);
            a0 = make_float2(v[0], v[1]);
            a1 = make_float2(v[2], v[3]);
            a2 = make_float2(v[4], v[5]);
        } else {
            float v[3];
            sum8_cubic<3>(Wx, Wy, Wz, [&](int a, int b, int e, float *r) {
                const float4 q4 = __ldg(rl.A + pt(a, b, e));
                r[0] = q4.x;
                r[1] = q4.y;
                r[2] = q4.z;
            }, v);
            a0 = make_float2(v[0], v[1]);
            a1.x = v[2];
        }
    } else {
#pragma unroll 1
        for (int e = 0; e <= P; e++) {
            const float wz = sel<P>(Wz, e);
            const long long rz = (long long)rl.py * (wrapi(gs[2] + e, g.nz) + rl.gl);
#pragma unroll
            for (int b = 0; b <= P; b++) {
                const long long ry = ((long long)rl.px) * (rz + wrapi(gs[1] + b, g.ny) + rl.gl) + rl.gl;
                const float wyz = Wy[b] * wz;
#pragma unroll
                for (int a = 0; a <= P; a++) {
                    const float w = Wx[a] * wyz;
                    const long long m = ry + wrapi(gs[0] + a, g.nx);
                    const float4 r = __ldg(rl.A + m);
                    a0 = __ffma2_rn(make_float2(r.x, r.y), make_float2(w, w), a0);
                    if (NFG == 2) {
                        a1 = __ffma2_rn(make_float2(r.z, r.w), make_float2(w, w), a1);
                        const float2 s = __ldg(rl.B + m);
                        a2 = __ffma2_rn(s, make_float2(w, w), a2);
                    } else {
                        a1.x = __fmaf_rn(r.z, w, a1.x);
                    }
                }
            }
        }
    }
}

// Mark of a particle whose stencil left its tile's box, written over fgrid[3p] by the tile
// gather: a NaN bit pattern that no arithmetic produces (the GPU's NaNs are 0x7fffffff),
// so that the integrator pass, which gathers such particles from global memory, tells
// them apart from any force.
constexpr unsigned kGatherLater = 0x7fa11e57u;

// The tile gather: every particle's grid force into fgrid[3p], for boxes of one or two
// force groups over the paired records.  One CTA per Morton tile, one particle per thread
// and pass.  The tile's box (its bricks widened by the stencil and one cell of drift per
// side) arrives by TMA loads of plane A and plane B, issued first, so that they fly while
// the particles' positions and stencils are read and computed; the ghost layers of the
// planes hold the periodic images, so a box never wraps.  Each warp deals its box gathers
// over its lanes by bank position (below), gathers both force groups in one pass (three
// paired FMAs per stencil point: (g0.x, g0.y), (g1.x, g1.y), (g0.z, g1.z)), and returns
// the sums to the particles' own lanes.  A particle that drifted out of the box gets the
// mark kGatherLater instead: its gather from global memory, a chain of dependent loads,
// is left to the integrator pass, where many more warps hide it.  Sums per group are
// formed in the order of the planar gather, so both kernels give the same bits.
template <int P, int NFG>
__device__ __forceinline__ void gather_paired_body(const Geom &g, const ParticleParams *__restrict__ ppd, int N,
                                                   const float *__restrict__ X0, const float *__restrict__ X1,
                                                   const uint32_t *__restrict__ pflags, const float *__restrict__ q,
                                                   const RecLayout &rl, const long long *__restrict__ d_step,
                                                   float *__restrict__ fgrid, const TileCfg &tc,
                                                   const CUtensorMap *mapA, const CUtensorMap *mapB,
                                                   int *__restrict__ err, unsigned bx, bool maps_in_global)
{
    // All of the CTA's shared memory is dynamic (paired_smem): plane A's box, plane B's, the
    // dealing table (a lane index per thread) and the barrier, with no static variables, so
    // that the window starts 128-byte aligned for the TMA boxes and no alignment slack is
    // spent (an 8-brick tile's box then fits four CTAs per SM).  Should the window ever
    // start unaligned, the CTA loads no box and leaves its particles to the integrator
    // pass's global gather: slower, the same forces.
    extern __shared__ __align__(128) unsigned char smbox[];
    const int te0 = tc.te[0], te1 = tc.te[1], te2 = tc.te[2];
    const int te01 = te0 * te1, V = te01 * te2;
    const size_t offB = ((size_t)V * 16 + 127) & ~(size_t)127;
    const size_t offD = offB + (NFG == 2 ? (((size_t)V * 8 + 15) & ~(size_t)15) : 0);
    float4 *boxA = reinterpret_cast<float4 *>(smbox);
    float2 *boxB = reinterpret_cast<float2 *>(smbox + offB);
    unsigned char *deal_src = smbox + offD;
    unsigned long long &bar = *reinterpret_cast<unsigned long long *>(smbox + offD + kPartThreadsMax);
    const bool aligned = (smem_u32(smbox) & 127u) == 0u;
    const ParticleParams &pp = *ppd;
    const long long step = *d_step;
    const float *__restrict__ Xc = (step & 1) ? X1 : X0;
    const int nn[3] = {g.nx, g.ny, g.nz};
    int r0, r1;
    tile_range(tc, N, kPartWindow, r0, r1, bx);
    if (r1 <= r0) return;   // an empty tile
    int lo[3], span[3], E[3];
    tile_box<P>(tc, nn, lo, span, E, bx);
    // 1. the box: one TMA load per plane, coordinates in the padded grid (lo + gl >= 0)
    if (threadIdx.x == 0 && aligned) {
        mbar_init(&bar);
        if (maps_in_global) {   // descriptors in a device table: acquire them for the tensor-map proxy
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(mapA) : "memory");
            if (NFG == 2) asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(mapB) : "memory");
        }
        const unsigned bytes = (unsigned)V * (NFG == 2 ? 24u : 16u);
        asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n"
                     ::"r"(smem_u32(&bar)), "r"(bytes) : "memory");
        const int cx = lo[0] + rl.gl, cy = lo[1] + rl.gl, cz = lo[2] + rl.gl;
        asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                     " [%0], [%1, {%2, %3, %4, %5}], [%6];\n"
                     ::"r"(smem_u32(boxA)), "l"(mapA), "r"(0), "r"(cx), "r"(cy), "r"(cz), "r"(smem_u32(&bar))
                     : "memory");
        if (NFG == 2)
            asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                         " [%0], [%1, {%2, %3, %4}], [%5];\n"
                         ::"r"(smem_u32(boxB)), "l"(mapB), "r"(2 * cx), "r"(cy), "r"(cz), "r"(smem_u32(&bar))
                         : "memory");
    }
    __syncthreads();   // the barrier is initialised before anyone waits on it
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    bool waited = false;
    for (int c0 = r0; c0 < r1; c0 += blockDim.x) {
        int p = c0 + threadIdx.x;
        bool act = p < r1;
        if constexpr (P == 3) {
            // the pass's particles spread evenly over the warps, k consecutive ones each, so
            // that no warp holds more rounds of box gathers than it must
            const int cnt = min(r1 - c0, (int)blockDim.x), nw = (int)(blockDim.x >> 5);
            const int k = (cnt + nw - 1) / nw;
            p = c0 + (int)(threadIdx.x >> 5) * k + lane;
            act = lane < k && p < c0 + cnt;
        }
        float x[3] = {0.f, 0.f, 0.f};
        uint32_t fl = 0u;
        float qp = 0.f;
        if (act) {
            x[0] = Xc[3 * p];
            x[1] = Xc[3 * p + 1];
            x[2] = Xc[3 * p + 2];
            fl = pflags[p];
            if (q) qp = q[p];
        }
        const unsigned fm = (fl >> 8) & ((1u << NFG) - 1u);
        float Wx[P + 1], Wy[P + 1], Wz[P + 1];
        int d[3] = {0, 0, 0};
        bool inbox = false;
        if (fm) {
            const int gs[3] = {stencil_fast<P>(x[0], g, 0, pp.quirk4, Wx), stencil_fast<P>(x[1], g, 1, pp.quirk4, Wy),
                               stencil_fast<P>(x[2], g, 2, pp.quirk4, Wz)};
#pragma unroll
            for (int j = 0; j < 3; j++) d[j] = wrapi(gs[j] - lo[j], nn[j]);
            inbox = aligned && d[0] <= span[0] && d[1] <= span[1] && d[2] <= span[2];
        } else {
#pragma unroll
            for (int i = 0; i <= P; i++) Wx[i] = Wy[i] = Wz[i] = 0.f;
        }
        const int base = d[2] * te01 + d[1] * te0 + d[0];
        float v[6];
        if constexpr (P == 3) {
            // 2. eight lanes per particle: lane k = 8 q' + k' of quarter q' takes column a = k' & 3
            // and rows b = 2 (k' >> 2) + i of every plane of the stencil.  With a box row pitch
            // te0 = 2 (mod 4), the eight starting records of a quarter warp are a + 2 (k' >> 2)
            // te0 = 0..7 (mod 8) after the particle's own offset: eight distinct 16-byte bank
            // groups, whatever the particle, so plane A's float4 loads take one wavefront per
            // quarter.  A half warp holds two particles; their plane-B float2 loads cover eight
            // consecutive 8-byte bank pairs each, so the warp orders its in-box particles by
            // offset mod 16 and pairs position j with j + ceil(m / 2), about 8 apart.  The lane
            // sums add by a fixed tree (the order of sum8_cubic) and the result goes back to the
            // particle's own lane.
            const int r16 = inbox ? (base & 15) : 16;
            int below = 0;
#pragma unroll
            for (int c = 0; c < 16; c++) {
                const unsigned bl = __ballot_sync(full, r16 == c);
                below += c < r16 ? __popc(bl) : 0;
            }
            const int j = below + __popc(__match_any_sync(full, r16) & ((1u << lane) - 1u));
            const int m = __popc(__ballot_sync(full, inbox));
            const int hm = (m + 1) >> 1;
            int myround = -1, myq = 0;
            if (inbox) {
                const int jj = j < hm ? j : j - hm;
                myround = jj >> 1;
                myq = 2 * (jj & 1) + (j < hm ? 0 : 1);
                deal_src[(threadIdx.x & ~31) + myround * 4 + myq] = lane;
            }
            __syncwarp();
            // 3. the box has landed (bounded wait: a copy that never completes is recorded)
            if (!waited && aligned) {
                if (!mbar_wait(&bar, 0u)) {
                    if (lane == 0) atomicAdd(err, 1);
                    mbar_wait(&bar, 0u);
                }
                waited = true;
            }
            const int qd = lane >> 3, ca = lane & 3, bh = (lane >> 2) & 1;
            const int rounds = (hm + 1) >> 1;
            float2 res0 = make_float2(0.f, 0.f), res1 = res0, res2 = res0;
            for (int rd = 0; rd < rounds; rd++) {
                // the particle of this quarter in this round, if any
                const int jj = 2 * rd + (qd >> 1);
                const bool filled = (qd & 1) == 0 ? jj < hm : jj < m - hm;
                const int src = filled ? deal_src[(threadIdx.x & ~31) + rd * 4 + qd] : lane;
                // the dealt particle's position and box offset; its weights are recomputed
                // here (the same bits as its own lane's), which takes fewer shuffles -- and
                // shuffles share the shared-memory pipe with the gathers
                const int bs = __shfl_sync(full, base, src);
                const float px = __shfl_sync(full, x[0], src), py = __shfl_sync(full, x[1], src),
                            pz = __shfl_sync(full, x[2], src);
                float wx[4], wy[4], wz[4];
                stencil_fast<3>(px, g, 0, pp.quirk4, wx);
                stencil_fast<3>(py, g, 1, pp.quirk4, wy);
                stencil_fast<3>(pz, g, 2, pp.quirk4, wz);
                const float wa = sel<3>(wx, ca), wy0 = sel<3>(wy, 2 * bh), wy1 = sel<3>(wy, 2 * bh + 1);
                float2 s0 = make_float2(0.f, 0.f), s1 = s0, s2 = s0;
                if (filled) {
                    const int col = bs + ca + 2 * bh * te0;
#pragma unroll
                    for (int e = 0; e < 4; e++)
#pragma unroll
                        for (int i = 0; i < 2; i++) {
                            const float w = wa * ((i ? wy1 : wy0) * wz[e]);
                            const int row = col + e * te01 + i * te0;
                            const float4 rA = boxA[row];
                            s0 = __ffma2_rn(make_float2(rA.x, rA.y), make_float2(w, w), s0);
                            if (NFG == 2) {
                                s1 = __ffma2_rn(make_float2(rA.z, rA.w), make_float2(w, w), s1);
                                s2 = __ffma2_rn(boxB[row], make_float2(w, w), s2);
                            } else {
                                s1.x = __fmaf_rn(rA.z, w, s1.x);
                            }
                        }
                }
                // ((s0 + s1) + (s2 + s3)) + ((s4 + s5) + (s6 + s7)) over the quarter's lanes, as a
                // reduce-scatter: at each level a lane keeps part of its values, adds its
                // partner's partial sums of that part (a + b = b + a: every node of the tree
                // gives the same bits in either lane) and passes on the rest, so each level
                // shuffles only the values it halves; the sums end spread over the quarter
                const int from = 8 * myq;
                const bool b0 = lane & 1, b1 = (lane >> 1) & 1, b2 = (lane >> 2) & 1;
                float2 t0, t1, t2 = make_float2(0.f, 0.f);
                if (NFG == 2) {
                    // values s0.x s0.y s1.x | s1.y s2.x s2.y: lane bit 0 picks a half, bit 1 two
                    // of its three or the third, bit 2 one of those two
                    const float a[6] = {s0.x, s0.y, s1.x, s1.y, s2.x, s2.y};
                    float k3[3];
#pragma unroll
                    for (int j = 0; j < 3; j++)
                        k3[j] = __fadd_rn(b0 ? a[j + 3] : a[j], __shfl_xor_sync(full, b0 ? a[j] : a[j + 3], 1));
                    const float r1 = __shfl_xor_sync(full, b1 ? k3[0] : k3[2], 2);
                    const float r2 = __shfl_xor_sync(full, k3[1], 2);
                    const float c0 = __fadd_rn(b1 ? k3[2] : k3[0], r1), c1 = __fadd_rn(k3[1], r2);
                    const float fin = __fadd_rn(b1 ? c0 : (b2 ? c1 : c0),
                                                __shfl_xor_sync(full, b1 ? c0 : (b2 ? c0 : c1), 4));
                    // the particle's own lane takes the sums of its quarter: s0.x at quarter
                    // lane 0, s0.y 4, s1.x 2, s1.y 1, s2.x 5, s2.y 3
                    t0 = make_float2(__shfl_sync(full, fin, from), __shfl_sync(full, fin, from + 4));
                    t1 = make_float2(__shfl_sync(full, fin, from + 2), __shfl_sync(full, fin, from + 1));
                    t2 = make_float2(__shfl_sync(full, fin, from + 5), __shfl_sync(full, fin, from + 3));
                } else {
                    // values s0.x s0.y | s1.x: bit 0 picks the pair or the single value, bit 1
                    // one of the pair
                    const float k0 = __fadd_rn(b0 ? s1.x : s0.x, __shfl_xor_sync(full, b0 ? s0.x : s1.x, 1));
                    const float k1 = __fadd_rn(s0.y, __shfl_xor_sync(full, s0.y, 1));
                    const float m = __fadd_rn(b0 ? k0 : (b1 ? k1 : k0),
                                              __shfl_xor_sync(full, b0 ? k0 : (b1 ? k0 : k1), 2));
                    const float fin = __fadd_rn(m, __shfl_xor_sync(full, m, 4));
                    // s0.x at quarter lane 0, s0.y 2, s1.x 1
                    t0 = make_float2(__shfl_sync(full, fin, from), __shfl_sync(full, fin, from + 2));
                    t1 = make_float2(__shfl_sync(full, fin, from + 1), 0.f);
                }
                if (myround == rd) {
                    res0 = t0;
                    res1 = t1;
                    res2 = t2;
                }
            }
            __syncwarp();   // deal_src is rewritten by the next pass
            v[0] = res0.x;
            v[1] = res0.y;
            if (NFG == 2) {
                v[2] = res2.x;
                v[3] = res1.x;
                v[4] = res1.y;
                v[5] = res2.y;
            } else {
                v[2] = res1.x;
            }
        } else {
            // 2. deal the box gathers of the warp over its lanes by bank group.  A float4 load
            // of a quarter warp takes one shared-memory wavefront when its eight lanes start at
            // distinct 16-byte bank groups (record offset mod 8); every stencil point adds the
            // same offset to all lanes, so the starts decide.  The warp orders its particles by
            // offset mod 8 (class 8: nothing to gather from the box) and lane 8q + a takes the
            // particle at position 4a + q of the order, so that the eight lanes of a quarter
            // warp get positions four apart, spread over the bank groups.  The lane gathers with
            // the dealt particle's stencil (shuffled in) and returns the sums to the particle's
            // own lane.
            const int r = inbox ? (base & 7) : 8;
            int below = 0;
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const unsigned bl = __ballot_sync(full, r == c);
                below += c < r ? __popc(bl) : 0;
            }
            const int j = below + __popc(__match_any_sync(full, r) & ((1u << lane) - 1u));
            const int tp = ((j & 3) << 3) | (j >> 2);
            deal_src[(threadIdx.x & ~31) + tp] = lane;
            __syncwarp();
            const int src = deal_src[threadIdx.x];
            __syncwarp();
            const int bsrc = __shfl_sync(full, base, src);
            const bool gsrc = __shfl_sync(full, inbox ? 1 : 0, src) != 0;
#pragma unroll
            for (int i = 0; i <= P; i++) {
                Wx[i] = __shfl_sync(full, Wx[i], src);
                Wy[i] = __shfl_sync(full, Wy[i], src);
                Wz[i] = __shfl_sync(full, Wz[i], src);
            }
            // 3. the box has landed (bounded wait: a copy that never completes is recorded)
            if (!waited && aligned) {
                if (!mbar_wait(&bar, 0u)) {
                    if (lane == 0) atomicAdd(err, 1);
                    mbar_wait(&bar, 0u);
                }
                waited = true;
            }
            // 4. the dealt particle's gather: both groups in one pass
            float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f), a2 = make_float2(0.f, 0.f);
            if (gsrc) {
#pragma unroll
                for (int e = 0; e <= P; e++) {
#pragma unroll
                    for (int b = 0; b <= P; b++) {
                        const float wyz = Wy[b] * Wz[e];
                        const int row = bsrc + e * te01 + b * te0;
#pragma unroll
                        for (int aa = 0; aa <= P; aa++) {
                            const float w = Wx[aa] * wyz;
                            const float4 rA = boxA[row + aa];
                            a0 = __ffma2_rn(make_float2(rA.x, rA.y), make_float2(w, w), a0);
                            if (NFG == 2) {
                                a1 = __ffma2_rn(make_float2(rA.z, rA.w), make_float2(w, w), a1);
                                const float2 rB = boxB[row + aa];
                                a2 = __ffma2_rn(rB, make_float2(w, w), a2);
                            } else {
                                a1.x = __fmaf_rn(rA.z, w, a1.x);
                            }
                        }
                    }
                }
            }
            // values back to the owning lanes: group 0 (x, y, z), then group 1 (x, y, z)
                v[0] = __shfl_sync(full, a0.x, tp);
            v[1] = __shfl_sync(full, a0.y, tp);
            if (NFG == 2) {
                v[2] = __shfl_sync(full, a2.x, tp);
                v[3] = __shfl_sync(full, a1.x, tp);
                v[4] = __shfl_sync(full, a1.y, tp);
                v[5] = __shfl_sync(full, a2.y, tp);
            } else {
                v[2] = __shfl_sync(full, a1.x, tp);
            }
        }
        if (act) {
            float fgv[3] = {0.f, 0.f, 0.f};
            if (fm && !inbox) {
                fgv[0] = __uint_as_float(kGatherLater);
            } else {
                if (fm & 1u) add_group(fgv, v, pp.fg_qweighted & 1u, qp);
                if (NFG == 2 && (fm & 2u)) add_group(fgv, v + 3, (pp.fg_qweighted >> 1) & 1u, qp);
            }
            fgrid[3 * p] = fgv[0];
            fgrid[3 * p + 1] = fgv[1];
            fgrid[3 * p + 2] = fgv[2];
        }
    }
}

// 64 registers: an 8-brick tile's box (57 KB) then fits four CTAs of 256 threads per SM,
// and the boxes in flight, not the registers, set the gather's pace (C2: 0.222 ->
// 0.200 ms; 56 registers: 0.207)
template <int P, int NFG>
__global__ void __maxnreg__(64) k_gather_paired(Geom g, const ParticleParams *__restrict__ ppd, int N,
                                                      const float *__restrict__ X0, const float *__restrict__ X1,
                                                      const uint32_t *__restrict__ pflags,
                                                      const float *__restrict__ q, RecLayout rl,
                                                      const long long *__restrict__ d_step, float *__restrict__ fgrid,
                                                      TileCfg tc, const __grid_constant__ CUtensorMap mapA,
                                                      const __grid_constant__ CUtensorMap mapB, int *__restrict__ err)
{
    gather_paired_body<P, NFG>(g, ppd, N, X0, X1, pflags, q, rl, d_step, fgrid, tc, &mapA, &mapB, err, blockIdx.x,
                               false);
}

// the tile gather over several replicas; each replica's TMA descriptors live in the table
template <int P, int NFG>
__global__ void __launch_bounds__(kPartThreadsMax, 2) k_gather_batch(const BatchRep *__restrict__ reps,
                                                                     const int *__restrict__ pre, int R)
{
    const int r = batch_replica(pre, R, blockIdx.x);
    const BatchRep &b = reps[r];
    gather_paired_body<P, NFG>(b.g, b.ppd, b.N, b.X0, b.X1, b.flags, b.q, b.rl, b.d_step, b.fgrid, b.tiles, &b.mapA,
                               &b.mapB, b.err, blockIdx.x - pre[r], true);
}

// ---- bonds, angles, walls and the integrator (one thread per particle) ----
// f = (bonds, then angles, then walls: the order of d_bonds, d_angles and the wall
// potential's CalcForces, PS_Box.cu:240-278) + the grid force fgrid[3p]; fout[3p] = f on
// request; then GJF (ps_integratorGJF.cu:102-163) or EM (ps_integratorEM.cu:39-82) reads
// x_t from Xc and replaces x_{t-1} in Xn by x_{t+1}.
// A particle the tile gather marked (kGatherLater) is gathered here from the paired
// records in global memory, with the arithmetic and order of the tile gather.
template <int P, bool EXTRA>
__device__ __forceinline__ void integrate_body(const Geom &g, const ParticleParams *__restrict__ ppd, int N,
                                               float *__restrict__ X0, float *__restrict__ X1,
                                               float *__restrict__ noise, const uint32_t *__restrict__ pflags,
                                               const float *__restrict__ q, const int *__restrict__ brow,
                                               const int *__restrict__ partner, const uint8_t *__restrict__ btype,
                                               const AngleArrays &aa, const float *__restrict__ fgrid,
                                               const RecLayout &rl, const int *__restrict__ orig_id,
                                               curandState *__restrict__ rng, const long long *__restrict__ d_step,
                                               float *__restrict__ fout, int integrate_flag, unsigned bx)
{
    const int p = (int)bx * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const ParticleParams &pp = *ppd;
    const long long step = *d_step;
    const float *__restrict__ Xc = (step & 1) ? X1 : X0;
    float *__restrict__ Xn = (step & 1) ? X0 : X1;
    const float x[3] = {Xc[3 * p], Xc[3 * p + 1], Xc[3 * p + 2]};
    const uint32_t fl = pflags[p];
    float f[3] = {0.f, 0.f, 0.f};
    bond_force(g, pp, p, x, Xc, brow, partner, btype, f);
    if (EXTRA) {
        if (aa.na) angle_force(g, pp, p, Xc, aa, f);
        if (pp.nwall) wall_terms(pp, fl, x, f, nullptr);
    }
    float fgv[3] = {fgrid[3 * p], fgrid[3 * p + 1], fgrid[3 * p + 2]};
    if (rl.paired && __float_as_uint(fgv[0]) == kGatherLater) {
        float Wx[P + 1], Wy[P + 1], Wz[P + 1];
        const int gs[3] = {stencil_fast<P>(x[0], g, 0, pp.quirk4, Wx), stencil_fast<P>(x[1], g, 1, pp.quirk4, Wy),
                           stencil_fast<P>(x[2], g, 2, pp.quirk4, Wz)};
        float2 h0, h1, h2;
        const float qp = q ? q[p] : 0.f;
        const unsigned fm = (fl >> 8) & 3u;
        fgv[0] = fgv[1] = fgv[2] = 0.f;
        if (rl.nfg == 2) {
            gather_paired_global<P, 2>(g, rl, gs, Wx, Wy, Wz, h0, h1, h2);
            const float v[6] = {h0.x, h0.y, h2.x, h1.x, h1.y, h2.y};
            if (fm & 1u) add_group(fgv, v, pp.fg_qweighted & 1u, qp);
            if (fm & 2u) add_group(fgv, v + 3, (pp.fg_qweighted >> 1) & 1u, qp);
        } else {
            gather_paired_global<P, 1>(g, rl, gs, Wx, Wy, Wz, h0, h1, h2);
            const float v[3] = {h0.x, h0.y, h1.x};
            if (fm & 1u) add_group(fgv, v, pp.fg_qweighted & 1u, qp);
        }
    }
#pragma unroll
    for (int j = 0; j < 3; j++) f[j] += fgv[j];
    if (fout) {
        fout[3 * p] = f[0];
        fout[3 * p + 1] = f[1];
        fout[3 * p + 2] = f[2];
    }
    if (integrate_flag) {
        const float xold[3] = {Xn[3 * p], Xn[3 * p + 1], Xn[3 * p + 2]};
        const float nold[3] = {noise[3 * p], noise[3 * p + 1], noise[3 * p + 2]};
        integrate(g, pp, p, fl, x, f, Xn, noise, xold, nold, orig_id[p], rng, step);
    }
}

// Eight CTAs per SM (32 registers) for boxes without angles or walls: the pass waits on
// loads (bond partners, the grid force, the old positions and noise) far more than it
// computes, so full occupancy pays for the values it keeps in local memory (C2: 0.079 ->
// 0.063 ms); with the extra terms, four.
template <int P, bool EXTRA>
__global__ void __launch_bounds__(256, EXTRA ? 4 : 8) k_integrate(Geom g, const ParticleParams *__restrict__ ppd, int N,
                                                   float *__restrict__ X0, float *__restrict__ X1,
                                                   float *__restrict__ noise, const uint32_t *__restrict__ pflags,
                                                   const float *__restrict__ q,
                                                   const int *__restrict__ brow, const int *__restrict__ partner,
                                                   const uint8_t *__restrict__ btype, AngleArrays aa,
                                                   const float *__restrict__ fgrid, RecLayout rl,
                                                   const int *__restrict__ orig_id,
                                                   curandState *__restrict__ rng, const long long *__restrict__ d_step,
                                                   float *__restrict__ fout, int integrate_flag)
{
    integrate_body<P, EXTRA>(g, ppd, N, X0, X1, noise, pflags, q, brow, partner, btype, aa, fgrid, rl, orig_id, rng,
                             d_step, fout, integrate_flag, blockIdx.x);
}

// the integrator pass over several replicas
template <int P, bool EXTRA>
__global__ void __launch_bounds__(256, EXTRA ? 4 : 8) k_integrate_batch(const BatchRep *__restrict__ reps, const int *__restrict__ pre,
                                                         int R)
{
    const int r = batch_replica(pre, R, blockIdx.x);
    const BatchRep &b = reps[r];
    integrate_body<P, EXTRA>(b.g, b.ppd, b.N, b.X0, b.X1, b.noise, b.flags, b.q, b.brow, b.partner, b.btype, b.aa,
                             b.fgrid, b.rl, b.orig, reinterpret_cast<curandState *>(b.rng), b.d_step, nullptr, 1,
                             blockIdx.x - pre[r]);
}

// every replica's step counter, one thread each
__global__ void k_tick_batch(const BatchRep *__restrict__ reps, int R)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < R) *reps[r].d_step += 1;
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
// minimum-image threshold 0.5*Lh) and angle energy and virial (ps_deviceAngles.cu:151-294,
// every angle counted on each of its three particles), summed per block in FP64:
// cols = bond e, vir[6], angle e, vir[6].
__global__ void __launch_bounds__(256) k_bond_energy(Geom g, const ParticleParams *__restrict__ ppd, int N,
                                                     const float *__restrict__ X0, const float *__restrict__ X1,
                                                     const long long *__restrict__ d_step,
                                                     const int *__restrict__ brow,
                                                     const int *__restrict__ partner,
                                                     const uint8_t *__restrict__ btype, AngleArrays aa,
                                                     const uint32_t *__restrict__ pflags,
                                                     double *__restrict__ partials)
{
    constexpr int NC = kPartialCols;
    __shared__ double red[8][NC];
    const ParticleParams &pp = *ppd;
    const float *__restrict__ X = (*d_step & 1) ? X1 : X0;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] = 0.0;
    if (p < N && brow) {
        float e = 0.f, vir[6] = {0, 0, 0, 0, 0, 0};
        for (int k = brow[p]; k < brow[p + 1]; k++) {
            const int o = partner[k], t = btype[k];
            float dr[3], mdr2 = 0.f, mf = 0.f;
            for (int j = 0; j < 3; j++) {
                dr[j] = X[3 * p + j] - X[3 * o + j];
                // the reference's threshold of 0.5*Lh here (ps_deviceBonds.cu:132-133)
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
    if (p < N && aa.na) {
        float e = 0.f, vir[6] = {0, 0, 0, 0, 0, 0};
        for (int i = 0; i < aa.na[p]; i++) {
            const int b = (p * pp.maxa + i) * 3;
            float rij[3], rkj[3], fi[3], fk[3], ea;
            if (!angle_terms(g, pp, X, aa.ang[b], aa.ang[b + 1], aa.ang[b + 2], aa.atype[p * pp.maxa + i], rij, rkj,
                             fi, fk, ea))
                continue;
            e += ea;
            vir[0] += fi[0] * rij[0] + fk[0] * rkj[0];
            vir[1] += fi[1] * rij[1] + fk[1] * rkj[1];
            vir[2] += fi[2] * rij[2] + fk[2] * rkj[2];
            vir[3] += fi[0] * rij[1] + fk[0] * rkj[1];
            vir[4] += fi[0] * rij[2] + fk[0] * rkj[2];
            vir[5] += fi[1] * rij[2] + fk[1] * rkj[2];
        }
        acc[7] = e;
        for (int c = 0; c < 6; c++) acc[8 + c] = vir[c];
    }
    if (p < N && pp.nwall) {   // d_wallHarmonicEnergy (ps_potentialWall.cu:114-131)
        const float xp[3] = {X[3 * p], X[3 * p + 1], X[3 * p + 2]};
        float ew[kMaxWalls] = {0.f, 0.f, 0.f, 0.f};
        wall_terms(pp, pflags[p], xp, nullptr, ew);
#pragma unroll
        for (int w = 0; w < kMaxWalls; w++) acc[14 + w] = ew[w];
    }
    // blow-up check: a particle whose position is not finite (NaN or inf) is counted
    if (p < N && !(isfinite(X[3 * p]) && isfinite(X[3 * p + 1]) && isfinite(X[3 * p + 2])))
        acc[14 + kMaxWalls] = 1.0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = 0; c < NC; c++) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < NC) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w][threadIdx.x];
        partials[(long long)blockIdx.x * NC + threadIdx.x] = s;
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


constexpr size_t kPartSmemMax = 128 + kPartBox * sizeof(float4);
constexpr size_t kPairSmemMax = 200 * 1024;   // a paired box of up to 8,500 points

// shared memory of the paired tile gather for boxes of te[] points: the planes' boxes, the
// dealing table and the barrier (the layout of gather_paired_body)
static size_t paired_smem(const int *te, int nfg)
{
    const size_t V = (size_t)te[0] * te[1] * te[2];
    return ((V * 16 + 127) & ~(size_t)127) + (nfg == 2 ? ((V * 8 + 15) & ~(size_t)15) : 0) + kPartThreadsMax + 8;
}

template <int P>
static cudaError_t gather_launch(const Geom &g, const ParticleParams &pp, const ParticleParams *ppd, const float *X0,
                                 const float *X1, const uint32_t *pflags, const float *q, const float4 *rec,
                                 const RecLayout &rl, const long long *d_step, float *fgrid, const TileCfg &tc0,
                                 const CUtensorMap *rec_map, const CUtensorMap *pmapA, const CUtensorMap *pmapB,
                                 int *err, cudaStream_t st)
{
    const int N = pp.N;
    TileCfg tc = tc0;
    const int nbk = tc.start ? tile_ctas(tc) : (N + kPartWindow - 1) / kPartWindow;
    const int threads = tc.start ? std::min(tc.threads, kPartThreadsMax) : 256;
    if (rl.paired) {   // the host lays the records out in pairs only for sorted tiles it holds maps for
        if (!tc.start || !tc.paired || !pmapA || (rl.nfg == 2 && !pmapB) || g.nz < 2) return cudaErrorInvalidValue;
        const size_t smem = paired_smem(tc.te, rl.nfg);
        if (smem > kPairSmemMax) return cudaErrorInvalidValue;
        if (rl.nfg == 2)
            k_gather_paired<P, 2><<<nbk, threads, smem, st>>>(g, ppd, N, X0, X1, pflags, q, rl, d_step, fgrid, tc,
                                                              *pmapA, *pmapB, err);
        else
            k_gather_paired<P, 1><<<nbk, threads, smem, st>>>(g, ppd, N, X0, X1, pflags, q, rl, d_step, fgrid, tc,
                                                              *pmapA, *pmapA, err);
        return cudaGetLastError();
    }
    CUtensorMap none;
    std::memset(&none, 0, sizeof(none));
    if (!rec_map || tc.direct) tc.te[0] = tc.te[1] = tc.te[2] = 0;   // no TMA descriptor: cp.async staging
    const CUtensorMap &rm = rec_map ? *rec_map : none;
    const int cap = (tc.start && !tc.direct) ? std::min(tc.pbox, kPartBox) : 0;
    const size_t smem = 128 + (size_t)cap * sizeof(float4);
    // TMA staging needs the descriptor and the whole fixed box inside the shared-memory box
    const bool tma = tc.start && tc.te[0] > 0 && (long long)tc.te[0] * tc.te[1] * tc.te[2] <= cap;
    if (tma)
        k_gather_planar<P, true><<<nbk, threads, smem, st>>>(g, ppd, N, X0, X1, pflags, q, rec, d_step, fgrid, tc, cap,
                                                             rm, err);
    else
        k_gather_planar<P, false><<<nbk, threads, smem, st>>>(g, ppd, N, X0, X1, pflags, q, rec, d_step, fgrid, tc,
                                                              cap, rm, err);
    return cudaGetLastError();
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no driver library link).
typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiled tensor_map_encoder()
{
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult qr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &qr) != cudaSuccess ||
            qr != cudaDriverEntryPointSuccess || !p) {
            cudaGetLastError();
            return nullptr;
        }
        fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

bool build_record_map(CUtensorMap *map, const float4 *rec, const Geom &g, int nfg, const int *te)
{
    EncodeTiled fn = tensor_map_encoder();
    if (!fn) return false;
    if (te[0] <= 0 || te[0] > 256 || te[1] > 256 || te[2] > 256 || g.nz < 2) return false;
    // float4 records as 4 floats: (component, x, y, z, group); a box is one group's te[] points
    const cuuint64_t dims[5] = {4, (cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, (cuuint64_t)nfg};
    // byte strides of dimensions 1..4 (the components are contiguous)
    const cuuint64_t st[4] = {16, 16ull * g.nx, 16ull * g.nx * g.ny, 16ull * (cuuint64_t)g.M};
    const cuuint32_t box[5] = {4, (cuuint32_t)te[0], (cuuint32_t)te[1], (cuuint32_t)te[2], 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<float4 *>(rec), dims, st, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t rec_layout_bytes(const Geom &g, int nfg, int gl, const int *gh)
{
    const long long px = ((long long)g.nx + gl + gh[0] + 1) & ~1ll, py = (long long)g.ny + gl + gh[1],
                    pz = (long long)g.nz + gl + gh[2];
    const size_t pM = (size_t)(px * py * pz);
    return ((pM * 16 + 255) & ~(size_t)255) + (nfg == 2 ? pM * 8 : 0);
}

RecLayout make_rec_layout(const Geom &g, int nfg, int gl, const int *gh, void *base)
{
    RecLayout r{};
    r.paired = 1;
    r.nfg = nfg;
    r.gl = gl;
    for (int j = 0; j < 3; j++) r.gh[j] = gh[j];
    r.px = (g.nx + gl + gh[0] + 1) & ~1;   // even: plane B's rows of 2 px floats stay 16-byte multiples
    r.gh[0] = r.px - g.nx - gl;
    r.py = g.ny + gl + gh[1];
    r.pz = g.nz + gl + gh[2];
    r.pM = (long long)r.px * r.py * r.pz;
    r.A = reinterpret_cast<float4 *>(base);
    r.B = nfg == 2 ? reinterpret_cast<float2 *>(reinterpret_cast<char *>(base) + (((size_t)r.pM * 16 + 255) & ~(size_t)255))
                   : nullptr;
    return r;
}

// Plane A as a 4-D tensor of floats (component, x, y, z), boxes (4, te0, te1, te2); plane B
// as rows of 2 px floats (x, y, z), boxes (2 te0, te1, te2), which needs te0 even so that
// a box row is a multiple of 16 bytes (its x coordinate, 2 (lo + gl) with lo + gl a
// multiple of 4, is always aligned).
bool build_paired_maps(CUtensorMap *mapA, CUtensorMap *mapB, const RecLayout &rl, const int *te)
{
    EncodeTiled fn = tensor_map_encoder();
    if (!fn || !rl.paired) return false;
    if (te[0] <= 0 || (te[0] & 1) || 2 * te[0] > 256 || te[1] <= 0 || te[1] > 256 || te[2] <= 0 || te[2] > 256)
        return false;
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const cuuint64_t dA[4] = {4, (cuuint64_t)rl.px, (cuuint64_t)rl.py, (cuuint64_t)rl.pz};
    const cuuint64_t sA[3] = {16, 16ull * rl.px, 16ull * rl.px * rl.py};
    const cuuint32_t bA[4] = {4, (cuuint32_t)te[0], (cuuint32_t)te[1], (cuuint32_t)te[2]};
    if (fn(mapA, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, rl.A, dA, sA, bA, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    if (rl.nfg != 2) return true;
    const cuuint64_t dB[3] = {2ull * rl.px, (cuuint64_t)rl.py, (cuuint64_t)rl.pz};
    const cuuint64_t sB[2] = {8ull * rl.px, 8ull * rl.px * rl.py};
    const cuuint32_t bB[3] = {(cuuint32_t)(2 * te[0]), (cuuint32_t)te[1], (cuuint32_t)te[2]};
    return fn(mapB, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, rl.B, dB, sB, bB, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

void init_particle_attributes()
{
#define TILD_PA(P)                                                                                        \
    cudaFuncSetAttribute(k_gather_planar<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPartSmemMax); \
    cudaFuncSetAttribute(k_gather_planar<P, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPartSmemMax);  \
    cudaFuncSetAttribute(k_gather_paired<P, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmemMax);     \
    cudaFuncSetAttribute(k_gather_paired<P, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmemMax);     \
    cudaFuncSetAttribute(k_gather_batch<P, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmemMax);      \
    cudaFuncSetAttribute(k_gather_batch<P, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmemMax)
    TILD_PA(0);
    TILD_PA(1);
    TILD_PA(2);
    TILD_PA(3);
    TILD_PA(4);
#undef TILD_PA
}

bool paired_box_fits(const int *te, int nfg) { return paired_smem(te, nfg) <= kPairSmemMax; }

cudaError_t launch_gather(const Geom &g, const ParticleParams &pp, const ParticleParams *ppd, const float *X0,
                          const float *X1, const uint32_t *pflags, const float *q, const float4 *rec,
                          const RecLayout &rl, const long long *d_step, float *fgrid, const TileCfg &tc,
                          const CUtensorMap *rec_map, const CUtensorMap *pmapA, const CUtensorMap *pmapB, int *err,
                          cudaStream_t st)
{
    if (pp.N == 0) return cudaSuccess;
    if (pp.nfg == 0) return cudaMemsetAsync(fgrid, 0, sizeof(float) * 3 * (size_t)pp.N, st);
    cudaError_t e = cudaSuccess;
#define TILD_PL(P) e = gather_launch<P>(g, pp, ppd, X0, X1, pflags, q, rec, rl, d_step, fgrid, tc, rec_map, pmapA, pmapB, err, st)
    switch (pp.order) {
        case 0: TILD_PL(0); break;
        case 1: TILD_PL(1); break;
        case 2: TILD_PL(2); break;
        case 3: TILD_PL(3); break;
        default: TILD_PL(4); break;
    }
#undef TILD_PL
    return e;
}

template <int P>
static void integrate_launch(const Geom &g, const ParticleParams &pp, const ParticleParams *ppd, float *X0, float *X1,
                             float *noise, const uint32_t *pflags, const float *q, const int *brow, const int *partner,
                             const uint8_t *btype, AngleArrays aa, const float *fgrid, const RecLayout &rl,
                             const int *orig_id, curandState *rs, const long long *d_step, float *fout, int integrate,
                             cudaStream_t st)
{
    const bool extra = aa.na != nullptr || pp.nwall > 0;
    const int nb = (pp.N + 255) / 256;
    if (extra)
        k_integrate<P, true><<<nb, 256, 0, st>>>(g, ppd, pp.N, X0, X1, noise, pflags, q, brow, partner, btype, aa, fgrid,
                                                 rl, orig_id, rs, d_step, fout, integrate);
    else
        k_integrate<P, false><<<nb, 256, 0, st>>>(g, ppd, pp.N, X0, X1, noise, pflags, q, brow, partner, btype, aa,
                                                  fgrid, rl, orig_id, rs, d_step, fout, integrate);
}

cudaError_t launch_integrate(const Geom &g, const ParticleParams &pp, const ParticleParams *ppd, float *X0, float *X1,
                             float *noise, const uint32_t *pflags, const float *q, const int *brow, const int *partner,
                             const uint8_t *btype, AngleArrays aa, const float *fgrid, const RecLayout &rl,
                             const int *orig_id, void *rng_states, const long long *d_step, float *fout, int integrate,
                             cudaStream_t st)
{
    if (pp.N == 0) return cudaSuccess;
    curandState *rs = reinterpret_cast<curandState *>(rng_states);
#define TILD_IL(P) integrate_launch<P>(g, pp, ppd, X0, X1, noise, pflags, q, brow, partner, btype, aa, fgrid, rl, orig_id, \
                                       rs, d_step, fout, integrate, st)
    switch (pp.order) {
        case 0: TILD_IL(0); break;
        case 1: TILD_IL(1); break;
        case 2: TILD_IL(2); break;
        case 3: TILD_IL(3); break;
        default: TILD_IL(4); break;
    }
#undef TILD_IL
    return cudaGetLastError();
}

void particles_batch_shape(int stage, const BatchRep &r, int *blocks, int *threads, size_t *smem)
{
    if (stage == BS_GATHER) {
        *blocks = tile_ctas(r.tiles);
        *threads = std::min(r.tiles.threads, kPartThreadsMax);
        *smem = paired_smem(r.tiles.te, r.nfg);
    } else {   // BS_INTEGRATE
        *blocks = (r.N + 255) / 256;
        *threads = 256;
        *smem = 0;
    }
}

cudaError_t launch_particles_batch(int stage, const BatchRep *reps, int R, const BatchLaunch &bl, int order, int nfg,
                                   int extra, cudaStream_t st)
{
#define TILD_GB(P)                                                                                              \
    do {                                                                                                        \
        if (stage == BS_GATHER) {                                                                               \
            if (nfg == 2) k_gather_batch<P, 2><<<bl.blocks, bl.threads, bl.smem, st>>>(reps, bl.pre, R);        \
            else k_gather_batch<P, 1><<<bl.blocks, bl.threads, bl.smem, st>>>(reps, bl.pre, R);                 \
        } else {                                                                                                \
            if (extra) k_integrate_batch<P, true><<<bl.blocks, 256, 0, st>>>(reps, bl.pre, R);                  \
            else k_integrate_batch<P, false><<<bl.blocks, 256, 0, st>>>(reps, bl.pre, R);                       \
        }                                                                                                       \
    } while (0)
    switch (order) {
        case 0: TILD_GB(0); break;
        case 1: TILD_GB(1); break;
        case 2: TILD_GB(2); break;
        case 3: TILD_GB(3); break;
        default: TILD_GB(4); break;
    }
#undef TILD_GB
    return cudaGetLastError();
}

cudaError_t launch_batch_tick(const BatchRep *reps, int R, cudaStream_t st)
{
    k_tick_batch<<<(R + 127) / 128, 128, 0, st>>>(reps, R);
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
                               const float *X1, const long long *d_step, const int *brow, const int *partner,
                               const uint8_t *btype, AngleArrays aa, const uint32_t *pflags, double *partials,
                               int *nblocks_out, cudaStream_t st)
{
    const int nbk = pp.N > 0 ? (pp.N + 255) / 256 : 1;
    k_bond_energy<<<nbk, 256, 0, st>>>(g, ppd, pp.N, X0, X1, d_step, brow, partner, btype, aa, pflags, partials);
    if (nblocks_out) *nblocks_out = nbk;
    return cudaGetLastError();
}

cudaError_t launch_reduce_partials(const double *partials, int nblocks, int ncols, double *out, cudaStream_t st)
{
    k_reduce_partials<<<1, 256, 0, st>>>(partials, nblocks, ncols, out);
    return cudaGetLastError();
}

}  // namespace tild
