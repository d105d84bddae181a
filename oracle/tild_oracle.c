/*
 * tild_oracle.c -- CPU restatement of the MATILDA.FT TILD particle-mesh step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product in
 * matilda.ft_b200/ and the timed CPU baseline in bench.py.  Nothing in the product
 * links, loads or calls it.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference arm may use it.
 *
 * Every routine restates one reference kernel (paths relative to the MATILDA.FT
 * source tree).  The file is compiled twice:
 *   -DORC_F32  -> liborc32.so : FP32, mimicking the reference's float arithmetic,
 *                               including the fused multiply-adds that nvcc forms
 *                               by default (-fmad=true), so stencil indices and
 *                               weights are bit-comparable with the reference.
 *   (default)  -> liborc64.so : FP64 accuracy oracle.
 * Built with -ffp-contract=off so that only the explicit FMA() calls fuse.
 *
 * The spectral stage (FFT, k-space tables, energies) lives in oracle.py (numpy).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_F32
typedef float real;
#define FMA(a, b, c) fmaf((a), (b), (c))
#define SQRT(a) sqrtf(a)
#define K(c) (c##f)
#define SYM(name) orc32_##name
#else
typedef double real;
#define FMA(a, b, c) ((a) * (b) + (c))
#define SQRT(a) sqrt(a)
#define K(c) (c)
#define SYM(name) orc64_##name
#endif

/* ---------------------------------------------------------------------------
 * spline_get_weights -- ps_grid_utils.cu:17-67 (Deserno & Holm 1998 appendix).
 * quirk4 != 0 reproduces ps_grid_utils.cu:57 (sx3 = sx2*sx2 at order 4); with
 * quirk4 == 0 order 4 uses the true quartic B-spline (sx3 = sx2*sx).
 * ------------------------------------------------------------------------- */
static void spline_weights(real dx, real H, real *W, int order, int quirk4)
{
    real sx = dx / H;
    real sx2, sx3, sx4;
    if (order == 0) {
        W[0] = K(1.0);
    } else if (order == 1) {
        W[0] = K(0.5) - sx;
        W[1] = K(0.5) + sx;
    } else if (order == 2) {
        sx2 = sx * sx;
        W[0] = FMA(K(0.5), sx2, FMA(K(-0.5), sx, K(0.125)));
        W[1] = K(0.75) - sx2;
        W[2] = FMA(K(0.5), sx2, FMA(K(0.5), sx, K(0.125)));
    } else if (order == 3) {
        sx2 = sx * sx;
        sx3 = sx2 * sx;
        W[0] = FMA(K(-8.0), sx3, FMA(K(12.0), sx2, FMA(K(-6.0), sx, K(1.0)))) / K(48.0);
        W[1] = FMA(K(24.0), sx3, FMA(K(-12.0), sx2, FMA(K(-30.0), sx, K(23.0)))) / K(48.0);
        W[2] = FMA(K(-24.0), sx3, FMA(K(-12.0), sx2, FMA(K(30.0), sx, K(23.0)))) / K(48.0);
        W[3] = FMA(K(8.0), sx3, FMA(K(12.0), sx2, FMA(K(6.0), sx, K(1.0)))) / K(48.0);
    } else {
        sx2 = sx * sx;
        sx3 = quirk4 ? sx2 * sx2 : sx2 * sx;
        sx4 = sx2 * sx2;
        W[0] = FMA(K(16.0), sx4, FMA(K(-32.0), sx3, FMA(K(24.0), sx2, FMA(K(-8.0), sx, K(1.0))))) / K(384.0);
        W[1] = FMA(K(-16.0), sx4, FMA(K(16.0), sx3, FMA(K(24.0), sx2, FMA(K(-44.0), sx, K(19.0))))) / K(96.0);
        W[2] = FMA(K(48.0), sx4, FMA(K(-120.0), sx2, K(115.0))) / K(192.0);
        W[3] = FMA(K(-16.0), sx4, FMA(K(-16.0), sx3, FMA(K(24.0), sx2, FMA(K(44.0), sx, K(19.0))))) / K(96.0);
        W[4] = FMA(K(16.0), sx4, FMA(K(32.0), sx3, FMA(K(24.0), sx2, FMA(K(8.0), sx, K(1.0))))) / K(384.0);
    }
}

/* ---------------------------------------------------------------------------
 * d_calcGridWeights -- ps_grid_utils.cu:74-204.
 * x[n*Dim]; Nx[Dim]; dxf[Dim] = (float)(L/Nx); out inds/W [n*G], G = (order+1)^Dim.
 * Flat index x-fastest: nn0 + (nn1 + nn2*Nx1)*Nx0 (ps_grid_utils.cu:186), 2-D:
 * nn1*Nx0 + nn0 (:139).  W already divided by gvol = prod(dxf) (:97-101,188).
 * ------------------------------------------------------------------------- */
void SYM(grid_weights)(int n, const real *x, int Dim, const int *Nx, const real *dxf,
                       int order, int quirk4, int *inds, real *Wout)
{
    int G = 1;
    real gvol = K(1.0);
    for (int j = 0; j < Dim; j++) {
        gvol *= dxf[j];
        G *= order + 1;
    }
#pragma omp parallel for schedule(static)
    for (int id = 0; id < n; id++) {
        real W[3][6];
        int g[3];
        for (int j = 0; j < Dim; j++) {
            real xj = x[id * Dim + j], d = dxf[j], gdx;
            if (order % 2 == 0) {
                g[j] = (int)(FMA(K(0.5), d, xj) / d);
                gdx = FMA(-(real)g[j], d, xj);
            } else {
                g[j] = (int)(xj / d);
                gdx = FMA(-((real)g[j] + K(0.5)), d, xj);
            }
            spline_weights(gdx, d, W[j], order, quirk4);
        }
        int shift = order / 2, ct = 0;
        if (Dim == 2) {
            for (int ix = 0; ix <= order; ix++) {
                int n0 = (g[0] + ix - shift + Nx[0]) % Nx[0];
                for (int iy = 0; iy <= order; iy++) {
                    int n1 = (g[1] + iy - shift + Nx[1]) % Nx[1];
                    inds[id * G + ct] = n1 * Nx[0] + n0;
                    Wout[id * G + ct] = W[0][ix] * W[1][iy] / gvol;
                    ct++;
                }
            }
        } else {
            for (int ix = 0; ix <= order; ix++) {
                int n0 = (g[0] + ix - shift + Nx[0]) % Nx[0];
                for (int iy = 0; iy <= order; iy++) {
                    int n1 = (g[1] + iy - shift + Nx[1]) % Nx[1];
                    for (int iz = 0; iz <= order; iz++) {
                        int n2 = (g[2] + iz - shift + Nx[2]) % Nx[2];
                        inds[id * G + ct] = n0 + (n1 + n2 * Nx[1]) * Nx[0];
                        Wout[id * G + ct] = W[0][ix] * W[1][iy] * W[2][iz] / gvol;
                        ct++;
                    }
                }
            }
        }
    }
}

/* ---------------------------------------------------------------------------
 * d_fillDensityGrid / d_fillChargeDensityGrid -- device_utils.cu:282-352.
 * rho[M] += W over the group's sites; if rhoq != NULL also rhoq += q*W.
 * Serial (fixed particle order) unless nthreads > 1, in which case the adds are
 * atomic like the reference's (order then varies run to run).
 * ------------------------------------------------------------------------- */
void SYM(deposit)(int ns, const int *sites, int G, const int *inds, const real *W,
                  const real *q, real *rho, real *rhoq, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 1) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (int s = 0; s < ns; s++) {
            int p = sites[s];
            real qp = q ? q[p] : K(0.0);
            for (int i = 0; i < G; i++) {
                int m = inds[p * G + i];
                real w = W[p * G + i];
#pragma omp atomic
                rho[m] += w;
                if (rhoq) {
                    real qw = w * qp;
#pragma omp atomic
                    rhoq[m] += qw;
                }
            }
        }
        return;
    }
#endif
    (void)nthreads;
    for (int s = 0; s < ns; s++) {
        int p = sites[s];
        real qp = q ? q[p] : K(0.0);
        for (int i = 0; i < G; i++) {
            int m = inds[p * G + i];
            real w = W[p * G + i];
            rho[m] += w;
            if (rhoq) rhoq[m] += w * qp;
        }
    }
}

/* ---------------------------------------------------------------------------
 * d_mapGridForcesToPartics / d_mapGridChargeForcesToPartics --
 * device_utils.cu:358-461.  f[p*Dim+j] += (sum_i gridF[m_i*Dim+j]*W_i*gvol) [* q_p].
 * gvol is the float-converted double grid volume (ps_groups.cu:186-193).
 * ------------------------------------------------------------------------- */
void SYM(gather)(int ns, const int *sites, int G, const int *inds, const real *W, real gvol,
                 const real *gridF, const real *q, int Dim, real *f)
{
#pragma omp parallel for schedule(static)
    for (int s = 0; s < ns; s++) {
        int p = sites[s];
        for (int j = 0; j < Dim; j++) {
            real floc = K(0.0);
            for (int i = 0; i < G; i++) {
                int m = inds[p * G + i];
                floc = FMA(gridF[m * Dim + j] * W[p * G + i], gvol, floc);
            }
            if (q)
                f[p * Dim + j] = FMA(floc, q[p], f[p * Dim + j]);
            else
                f[p * Dim + j] += floc;
        }
    }
}

/* ---------------------------------------------------------------------------
 * d_bonds -- ps_deviceBonds.cu:7-79.  Padded partner list [n*maxb] storing both
 * directions; style 0 harmonic mf = 2k(r-req)/r, style 1 FENE; skipped for
 * r^2 <= 1e-4.  Minimum image with Lh = L/2.
 * ------------------------------------------------------------------------- */
void SYM(bonds)(int n, int Dim, const real *x, const int *nb, const int *partner,
                const int *btype, int maxb, const real *bk, const real *breq,
                const int *bstyle, const real *L, real *f)
{
#pragma omp parallel for schedule(static)
    for (int p = 0; p < n; p++) {
        real lf[3] = {0, 0, 0}, dr[3];
        for (int b = 0; b < nb[p]; b++) {
            int o = partner[p * maxb + b], t = btype[p * maxb + b];
            real mdr2 = K(0.0), mf = K(0.0);
            for (int j = 0; j < Dim; j++) {
                real Lh = K(0.5) * L[j];
                dr[j] = x[p * Dim + j] - x[o * Dim + j];
                if (dr[j] > Lh) dr[j] -= L[j];
                else if (dr[j] < -Lh) dr[j] += L[j];
                mdr2 = FMA(dr[j], dr[j], mdr2);
            }
            if (mdr2 > K(1.0e-4)) {
                real mdr = SQRT(mdr2);
                if (bstyle[t] == 0)
                    mf = K(2.0) * bk[t] * (mdr - breq[t]) / mdr;
                else {
                    real u = mdr / breq[t];
                    mf = K(2.0) * bk[t] * mdr / (K(1.0) - u * u) / mdr;
                }
            }
            for (int j = 0; j < Dim; j++) lf[j] = FMA(-mf, dr[j], lf[j]);
        }
        for (int j = 0; j < Dim; j++) f[p * Dim + j] += lf[j];
    }
}

/* ---------------------------------------------------------------------------
 * d_bondStressEnergy -- ps_deviceBonds.cu:85-171.  Per-particle energy (double
 * counted; the caller halves the sum, PS_Box.cu:292) and 6 (3-D) or 3 (2-D)
 * virial components.  Keeps the reference's minimum-image threshold of 0.5*Lh
 * (ps_deviceBonds.cu:132-133).
 * ------------------------------------------------------------------------- */
void SYM(bond_energy)(int n, int Dim, const real *x, const int *nb, const int *partner,
                      const int *btype, int maxb, const real *bk, const real *breq,
                      const int *bstyle, const real *L, real *e, real *vir)
{
    int npc = Dim == 2 ? 3 : 6;
#pragma omp parallel for schedule(static)
    for (int p = 0; p < n; p++) {
        real dr[3] = {0, 0, 0};
        e[p] = K(0.0);
        for (int c = 0; c < npc; c++) vir[p * npc + c] = K(0.0);
        for (int b = 0; b < nb[p]; b++) {
            int o = partner[p * maxb + b], t = btype[p * maxb + b];
            real mdr2 = K(0.0), mf = K(0.0);
            for (int j = 0; j < Dim; j++) {
                real Lh = K(0.5) * L[j];
                dr[j] = x[p * Dim + j] - x[o * Dim + j];
                if (dr[j] > K(0.5) * Lh) dr[j] -= L[j];
                else if (dr[j] < -K(0.5) * Lh) dr[j] += L[j];
                mdr2 = FMA(dr[j], dr[j], mdr2);
            }
            if (mdr2 > K(1.0e-4)) {
                real mdr = SQRT(mdr2);
                if (bstyle[t] == 0) {
                    real arg = mdr - breq[t];
                    mf = K(2.0) * bk[t] * arg / mdr;
                    e[p] += bk[t] * arg * arg;
                } else if (mdr / breq[t] < K(1.0)) {
                    real u = mdr / breq[t];
                    real arg = K(1.0) / (K(1.0) - u * u);
                    mf = K(2.0) * bk[t] * arg;
                    e[p] += mf * mdr;
                }
            }
            vir[p * npc + 0] += -mf * dr[0] * dr[0];
            vir[p * npc + 1] += -mf * dr[1] * dr[1];
            if (Dim == 2)
                vir[p * npc + 2] += -mf * dr[0] * dr[1];
            else {
                vir[p * npc + 2] += -mf * dr[2] * dr[2];
                vir[p * npc + 3] += -mf * dr[0] * dr[1];
                vir[p * npc + 4] += -mf * dr[0] * dr[2];
                vir[p * npc + 5] += -mf * dr[1] * dr[2];
            }
        }
    }
}

/* ---------------------------------------------------------------------------
 * GJF -- ps_integratorGJF.cu:43-95 (coefficients) and :102-163 (update), with
 * the unit normals injected by the caller (noise[s*Dim+j] for site s).
 * ------------------------------------------------------------------------- */
void SYM(gjf)(int ns, const int *sites, int Dim, const int *typ, const real *mass,
              const real *mobility, real delt, const real *L, const real *f,
              const real *noise, real *x, real *xo, real *old_noise)
{
#pragma omp parallel for schedule(static)
    for (int s = 0; s < ns; s++) {
        int p = sites[s], t = typ[p];
        real m = mass[t], Di = mobility[t];
        real b = m / (m + delt / (K(2.0) * Di));
        real a = (K(1.0) - delt / (K(2.0) * Di * m)) / (K(1.0) + delt / (K(2.0) * Di * m));
        real noiseMag = SQRT(K(2.0) * delt) / SQRT(Di);
        real bdt2m = b * (delt * delt) / m;
        real bdt2m2 = b * delt / (K(2.0) * m);
        for (int j = 0; j < Dim; j++) {
            int ai = p * Dim + j;
            real nn = noiseMag * noise[s * Dim + j];
            real xt = x[ai], xoj = xo[ai];
            if (xoj - xt > L[j] / K(2.0)) xoj -= L[j];
            else if (xoj - xt < -L[j] / K(2.0)) xoj += L[j];
            real xn = K(2.0) * b * xt - a * xoj + bdt2m * f[ai] + bdt2m2 * (nn + old_noise[ai]);
            xo[ai] = xt;
            old_noise[ai] = nn;
            if (xn > L[j]) xn -= L[j];
            else if (xn < K(0.0)) xn += L[j];
            x[ai] = xn;
        }
    }
}

/* EM -- ps_integratorEM.cu:39-82: x += delt*f + sqrt(2 delt)*xi, wrap.          */
void SYM(em)(int ns, const int *sites, int Dim, real delt, const real *L, const real *f,
             const real *noise, real *x)
{
    real nm = SQRT(K(2.0) * delt);
#pragma omp parallel for schedule(static)
    for (int s = 0; s < ns; s++) {
        int p = sites[s];
        for (int j = 0; j < Dim; j++) {
            int ai = p * Dim + j;
            real xt = x[ai] + delt * f[ai] + nm * noise[s * Dim + j];
            if (xt > L[j]) xt -= L[j];
            else if (xt < K(0.0)) xt += L[j];
            x[ai] = xt;
        }
    }
}

#ifndef ORC_F32
/* ---------------------------------------------------------------------------
 * Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, SC'11,
 * "Parallel random numbers: as easy as 1, 2, 3"), restated from the paper.
 * The CUDA product draws its GJF/EM noise with the same definition:
 *   key = (seed & 0xffffffff, seed >> 32), counter = (step, particle, 0, 0)
 *   u_i = (r_i + 0.5) * 2^-32,  Box-Muller in FP64:
 *   n0 = sqrt(-2 ln u0) cos(2 pi u1), n1 = sqrt(-2 ln u0) sin(2 pi u1),
 *   n2 = sqrt(-2 ln u2) cos(2 pi u3), rounded to float.
 * ------------------------------------------------------------------------- */
static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

/* Raw generator, exported for the known-answer test against the paper's vectors. */
void orc_philox4x32_10(uint32_t *ctr, const uint32_t *key)
{
    philox4x32_10(ctr, key[0], key[1]);
}

void orc_philox_normals(uint64_t seed, uint32_t step, int n, const int *ids, float *out)
{
    const double TWO_PI = 6.283185307179586476925286766559;
    for (int s = 0; s < n; s++) {
        uint32_t c[4] = {step, (uint32_t)ids[s], 0u, 0u};
        philox4x32_10(c, (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32));
        double u[4];
        for (int i = 0; i < 4; i++) u[i] = ((double)c[i] + 0.5) * 2.3283064365386963e-10;
        double r0 = sqrt(-2.0 * log(u[0])), r1 = sqrt(-2.0 * log(u[2]));
        out[3 * s + 0] = (float)(r0 * cos(TWO_PI * u[1]));
        out[3 * s + 1] = (float)(r0 * sin(TWO_PI * u[1]));
        out[3 * s + 2] = (float)(r1 * cos(TWO_PI * u[3]));
    }
}
#endif
