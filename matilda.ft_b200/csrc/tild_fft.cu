// tild_fft.cu -- hand-written mixed-radix Stockham 3-D FFT passes fused with the
// k-space potential/gradient multiply (sm_100a).
#include "tild_stencil.cuh"

#include <cmath>
#include <cstdio>
#include <vector>

namespace tild {

// =====================================================================================
// Shared-memory Stockham FFT of L lines of length n (mixed radix, natural order in and
// out).  Element t of line l lives at l*lp + t*ls.  Radix-R pass with p = product of the
// earlier radices: butterfly i reads i + q*n/R, twiddles by W_{pR}^{q*(i mod p)}, writes
// (i - i mod p)*R + i mod p + q*p.  Returns the buffer holding the result.
// =====================================================================================
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

template <bool INV>
__device__ __forceinline__ float2 twid(const float2 *tw, int t)
{
    float2 w = tw[t];
    if (INV) w.y = -w.y;
    return w;
}

__device__ __forceinline__ FastDiv make_fastdiv_dev(unsigned d)
{
    FastDiv f;
    f.d = d;
    f.m = d <= 1 ? 0u : (unsigned)((0x100000000ull + d - 1) / d);
    return f;
}

__device__ __forceinline__ unsigned fdiv(unsigned i, const FastDiv &f)
{
    return f.d == 1 ? i : __umulhi(i, f.m);
}

template <bool INV>
__device__ float2 *fft_lines(float2 *a, float2 *b, int L, int lp, int ls, const FftLine &pl,
                             const float2 *tw, bool line_fast, const FastDiv &dL)
{
    const int n = pl.n;
    for (int s = 0; s < pl.ns; ++s) {
        const int R = pl.R[s], p = pl.P[s], nb = n / R, stride = n / (p * R);
        const int total = L * nb;
        const FastDiv dp = pl.dP[s], dnb = pl.dNB[s];
        for (int w = threadIdx.x; w < total; w += blockDim.x) {
            int l, i;
            if (line_fast) {
                i = (int)fdiv((unsigned)w, dL);
                l = w - i * L;
            } else {
                l = (int)fdiv((unsigned)w, dnb);
                i = w - l * nb;
            }
            const int k = i - p * (int)fdiv((unsigned)i, dp);
            const float2 *src = a + l * lp;
            float2 *dst = b + l * lp;
            const int j = (i - k) * R + k;
            if (R == 2) {
                float2 a0 = src[i * ls], a1 = src[(i + nb) * ls];
                if (k) a1 = cmul(a1, twid<INV>(tw, k * stride));
                dst[j * ls] = cadd(a0, a1);
                dst[(j + p) * ls] = csub(a0, a1);
            } else if (R == 4) {
                float2 a0 = src[i * ls], a1 = src[(i + nb) * ls], a2 = src[(i + 2 * nb) * ls],
                       a3 = src[(i + 3 * nb) * ls];
                if (k) {
                    a1 = cmul(a1, twid<INV>(tw, k * stride));
                    a2 = cmul(a2, twid<INV>(tw, 2 * k * stride));
                    a3 = cmul(a3, twid<INV>(tw, 3 * k * stride));
                }
                const float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = csub(a1, a3);
                // forward: b1 = t1 - i t3, b3 = t1 + i t3; inverse swaps them
                const float2 mi = INV ? make_float2(-t3.y, t3.x) : make_float2(t3.y, -t3.x);
                dst[j * ls] = cadd(t0, t2);
                dst[(j + p) * ls] = cadd(t1, mi);
                dst[(j + 2 * p) * ls] = csub(t0, t2);
                dst[(j + 3 * p) * ls] = csub(t1, mi);
            } else if (R == 3) {
                float2 a0 = src[i * ls], a1 = src[(i + nb) * ls], a2 = src[(i + 2 * nb) * ls];
                if (k) {
                    a1 = cmul(a1, twid<INV>(tw, k * stride));
                    a2 = cmul(a2, twid<INV>(tw, 2 * k * stride));
                }
                const float s3 = INV ? 0.86602540378443865f : -0.86602540378443865f;
                const float2 t = cadd(a1, a2), u = csub(a1, a2);
                const float2 m = make_float2(a0.x - 0.5f * t.x, a0.y - 0.5f * t.y);
                // b1 = m + i*s3*u, b2 = m - i*s3*u
                const float2 iu = make_float2(-s3 * u.y, s3 * u.x);
                dst[j * ls] = cadd(a0, t);
                dst[(j + p) * ls] = cadd(m, iu);
                dst[(j + 2 * p) * ls] = csub(m, iu);
            } else if (R == 5) {
                float2 a0 = src[i * ls], a1 = src[(i + nb) * ls], a2 = src[(i + 2 * nb) * ls],
                       a3 = src[(i + 3 * nb) * ls], a4 = src[(i + 4 * nb) * ls];
                if (k) {
                    a1 = cmul(a1, twid<INV>(tw, k * stride));
                    a2 = cmul(a2, twid<INV>(tw, 2 * k * stride));
                    a3 = cmul(a3, twid<INV>(tw, 3 * k * stride));
                    a4 = cmul(a4, twid<INV>(tw, 4 * k * stride));
                }
                const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
                const float s1 = INV ? -0.95105651629515357f : 0.95105651629515357f;
                const float s2 = INV ? -0.58778525229247313f : 0.58778525229247313f;
                const float2 t1 = cadd(a1, a4), t2 = cadd(a2, a3), t3 = csub(a1, a4), t4 = csub(a2, a3);
                const float2 m1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
                const float2 m2 = make_float2(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
                // n1 = s1 t3 + s2 t4, n2 = s2 t3 - s1 t4; b1 = m1 - i n1, b4 = m1 + i n1,
                // b2 = m2 - i n2, b3 = m2 + i n2
                const float2 n1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
                const float2 n2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
                dst[j * ls] = make_float2(a0.x + t1.x + t2.x, a0.y + t1.y + t2.y);
                dst[(j + p) * ls] = make_float2(m1.x + n1.y, m1.y - n1.x);
                dst[(j + 4 * p) * ls] = make_float2(m1.x - n1.y, m1.y + n1.x);
                dst[(j + 2 * p) * ls] = make_float2(m2.x + n2.y, m2.y - n2.x);
                dst[(j + 3 * p) * ls] = make_float2(m2.x - n2.y, m2.y + n2.x);
            } else {
                // generic radix: b_q = sum_s a_s W_{pR}^{s k} W_R^{q s}
                const int nR = n / R;
                for (int qq = 0; qq < R; qq++) {
                    float2 acc = make_float2(0.f, 0.f);
                    for (int ss = 0; ss < R; ss++) {
                        float2 v = src[(i + ss * nb) * ls];
                        if (k && ss) v = cmul(v, twid<INV>(tw, ss * k * stride));
                        const int e = (qq * ss) % R;
                        if (e) v = cmul(v, twid<INV>(tw, e * nR));
                        acc = cadd(acc, v);
                    }
                    dst[(j + qq * p) * ls] = acc;
                }
            }
        }
        __syncthreads();
        float2 *t = a;
        a = b;
        b = t;
    }
    return a;
}

template <typename T>
static void set_max_smem(T *fn, size_t bytes)
{
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

static int lines_per_block(int n)
{
    int L = 2048 / n;
    if (L < 1) L = 1;
    if (L > 16) L = 16;
    return L;
}

// -------------------------------------------------------------------------------------
// Asynchronous tile loads: 16-byte cp.async copies (two complex values each), all in
// flight at once; bytes past the valid part of a row are zero-filled without a read.
// -------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc, int src_bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// rows x cols complex tile: smem dst[r*dpitch + c] <- src[r*spitch + c] for c < valid;
// cols and dpitch even; src and spitch 16-byte aligned (even element offsets).
__device__ __forceinline__ void tile_load_async(float2 *dst, int dpitch, const float2 *src, long long spitch, int rows,
                                                int cols, int valid)
{
    const int cpr = cols >> 1;   // 16-byte chunks per row
    for (int e = threadIdx.x; e < rows * cpr; e += blockDim.x) {
        const int r = e / cpr, c2 = (e - r * cpr) << 1;
        const int nv = valid - c2;
        const int bytes = nv >= 2 ? 16 : (nv == 1 ? 8 : 0);
        const float2 *s = bytes ? src + r * spitch + c2 : src;
        cp_async16(dst + r * dpitch + c2, s, bytes);
    }
}

// -------------------------------------------------------------------------------------
// x-axis forward pass.  Fields 2t and 2t+1 are packed as z = a + i b; after the complex
// FFT A(k) = (Z(k) + conj Z(n-k))/2 and B(k) = (Z(k) - conj Z(n-k))/(2i), k in [0, n/2].
// -------------------------------------------------------------------------------------
template <bool FIXED>
__global__ void __launch_bounds__(256) k_xfwd(Geom g, FftLine lx, int nd, const float2 *__restrict__ dep,
                                              const unsigned long long *__restrict__ depfix,
                                              double fscale, float2 *__restrict__ H, int L)
{
    extern __shared__ __align__(16) float2 sm[];
    const int n = g.nx;
    float2 *A = sm, *B = sm + L * n, *tw = sm + 2 * L * n;
    const int pair = blockIdx.y;
    const long long nlines = (long long)g.ny * g.nz;
    const long long line0 = (long long)blockIdx.x * L;
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = lx.tw[t];
    const int lv = (int)min((long long)L, nlines - line0);   // lines present in this block
    if (!FIXED && (n % 2) == 0) {
        tile_load_async(A, n, dep + pair * g.M + line0 * n, n, lv, n, n);
        for (int e = lv * n + threadIdx.x; e < L * n; e += blockDim.x) A[e] = make_float2(0.f, 0.f);
        cp_async_wait_all();
    } else {
        for (int e = threadIdx.x; e < L * n; e += blockDim.x) {
            const int l = e / n;
            const long long gl = line0 + l;
            float2 v = make_float2(0.f, 0.f);
            if (gl < nlines) {
                const long long idx = gl * n + (e - l * n);
                if (FIXED) {
                    v.x = (float)((double)(long long)depfix[(2 * pair) * g.M + idx] * fscale);
                    if (2 * pair + 1 < nd)
                        v.y = (float)((double)(long long)depfix[(2 * pair + 1) * g.M + idx] * fscale);
                } else {
                    v = dep[pair * g.M + idx];
                }
            }
            A[e] = v;
        }
    }
    __syncthreads();
    const float2 *R = fft_lines<false>(A, B, L, n, 1, lx, tw, false, make_fastdiv_dev(L));
    const int nxh = g.nxh;
    for (int e = threadIdx.x; e < L * nxh; e += blockDim.x) {
        const int l = e / nxh, k = e - l * nxh;
        const long long gl = line0 + l;
        if (gl >= nlines) continue;
        const float2 zk = R[l * n + k], zm = R[l * n + (k == 0 ? 0 : n - k)];
        const long long o = gl * g.hp + k;
        H[(2 * pair) * g.hstride + o] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        if (2 * pair + 1 < nd)
            H[(2 * pair + 1) * g.hstride + o] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
}

// y-axis pass over TX half-spectrum columns of one z plane of field blockIdx.z.
template <bool INV>
__global__ void __launch_bounds__(256) k_ypass(Geom g, FftLine ly, float2 *__restrict__ H, int TX)
{
    extern __shared__ __align__(16) float2 sm[];
    const int ny = g.ny;
    float2 *A = sm, *B = sm + ny * TX, *tw = sm + 2 * ny * TX;
    const int kx0 = blockIdx.x * TX;
    const long long base = (long long)blockIdx.z * g.hstride + (long long)blockIdx.y * ny * g.hp + kx0;
    for (int t = threadIdx.x; t < ny; t += blockDim.x) tw[t] = ly.tw[t];
    tile_load_async(A, TX, H + base, g.hp, ny, TX, g.nxh - kx0);
    cp_async_wait_all();
    __syncthreads();
    const float2 *R = fft_lines<INV>(A, B, TX, 1, TX, ly, tw, true, make_fastdiv_dev(TX));
    for (int e = threadIdx.x; e < ny * TX; e += blockDim.x) {
        const int y = e / TX, c = e - y * TX;
        if (kx0 + c < g.nxh) H[base + (long long)y * g.hp + c] = R[e];
    }
}

// û(k) of each potential kind, FP64 (ps_potentialGaussian.cu:38-46,
// ps_potentialErf2.cu:111-124, ps_potentialErfG.cu:177-190, ps_potentialCharges.cu:241-258).
__device__ double uk_eval(const PotDev &p, double k2)
{
    const double PI4 = 12.566370614359172953850573533118;
    if (p.kind == POT_GAUSSIAN) return p.amp * exp(-0.5 * k2 * p.sig2);
    if (p.kind == POT_CHARGES) return k2 > 0.0 ? PI4 * p.lB * exp(-k2 * p.sig2) / k2 : 0.0;
    const double R = p.Rp;
    double t;
    if (k2 == 0.0) {
        t = PI4 * R * R * R / 3.0;
        return p.kind == POT_ERF2 ? p.amp * t * t : p.amp * t;
    }
    const double k = sqrt(k2);
    double sn, cs;
    sincos(R * k, &sn, &cs);
    t = PI4 * (sn - R * k * cs) / (k2 * k);
    const double gs = exp(-0.5 * k2 * p.sig2);
    return p.kind == POT_ERF2 ? p.amp * gs * t * t : p.amp * gs * t;
}

__device__ __forceinline__ int signed_index(int i, int n) { return (i < n - i) ? i : i - n; }

// Fused z pass: forward z FFT of every density field, k-space combine, gradient and
// inverse z FFT of each gradient field; FP64 energies on request.
__global__ void __launch_bounds__(256) k_kspace_z(Geom g, FftLine lz, const KSpace *__restrict__ ksp, const float2 *__restrict__ H,
                                                  float2 *__restrict__ Hg, double *__restrict__ epart,
                                                  int energy, int forces, int TX)
{
    extern __shared__ __align__(16) float2 sm[];
    const KSpace &ks = *ksp;
    const int nz = g.nz, nd = ks.nd;
    const int ndb = nd < 2 ? 2 : nd;
    float2 *Rho = sm, *S = sm + ndb * nz * TX, *Phi = sm + 2 * ndb * nz * TX, *tw = Phi + nz * TX;
    double *red = reinterpret_cast<double *>(tw + nz);
    const int kx0 = blockIdx.x * TX, y = blockIdx.y;
    for (int t = threadIdx.x; t < nz; t += blockDim.x) tw[t] = lz.tw[t];
    for (int d = 0; d < nd; d++)
        tile_load_async(Rho + d * TX, nd * TX, H + d * g.hstride + (long long)y * g.hp + kx0, (long long)g.ny * g.hp,
                        nz, TX, g.nxh - kx0);
    cp_async_wait_all();
    __syncthreads();
    float2 *R = fft_lines<false>(Rho, S, nd * TX, 1, nd * TX, lz, tw, true, make_fastdiv_dev(nd * TX));
    float2 *Wk = (R == Rho) ? S : Rho;  // free buffer: two halves of nz*TX for the outputs
    const int ky = signed_index(y, g.ny);
    const double kyv = ks.twopi_over_L[1] * ky;
    const bool nyq_y = (g.ny % 2 == 0) && (y == g.ny / 2);

    if (energy) {
        double acc[kMaxPots];
        for (int t = 0; t < ks.neterms; t++) acc[t] = 0.0;
        for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
            const int z = e / TX, c = e - z * TX, kx = kx0 + c;
            if (kx >= g.nxh) continue;
            const double kxv = ks.twopi_over_L[0] * signed_index(kx, g.nx);
            const double kzv = ks.twopi_over_L[2] * signed_index(z, g.nz);
            const double k2 = kxv * kxv + kyv * kyv + kzv * kzv;
            const double wgt = (kx == 0 || (g.nx % 2 == 0 && kx == g.nx / 2)) ? 1.0 : 2.0;
            for (int t = 0; t < ks.neterms; t++) {
                const ETerm &et = ks.eterms[t];
                const float2 rI = R[z * nd * TX + et.dI * TX + c], rJ = R[z * nd * TX + et.dJ * TX + c];
                const double re = (double)rJ.x * rI.x + (double)rJ.y * rI.y;
                acc[t] += wgt * et.fac * uk_eval(ks.pots[et.pot], k2) * re;
            }
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        const long long blin = (long long)blockIdx.y * gridDim.x + blockIdx.x;
        for (int t = 0; t < ks.neterms; t++) {
            double v = acc[t];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp] = v;
            __syncthreads();
            if (threadIdx.x == 0) {
                double s = 0.0;
                for (int w = 0; w < nw; w++) s += red[w];
                epart[blin * ks.neterms + t] = s;
            }
            __syncthreads();
        }
    }
    if (!forces) return;

    for (int f = 0; f < ks.nfg; f++) {
        for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
            const int z = e / TX, c = e - z * TX, kx = kx0 + c;
            double px = 0.0, py = 0.0;
            if (kx < g.nxh) {
                const double kxv = ks.twopi_over_L[0] * signed_index(kx, g.nx);
                const double kzv = ks.twopi_over_L[2] * signed_index(z, g.nz);
                const double k2 = kxv * kxv + kyv * kyv + kzv * kzv;
                for (int t = 0; t < ks.nterms; t++) {
                    const KTerm &kt = ks.terms[t];
                    if (kt.fgroup != f) continue;
                    const double u = kt.mult * uk_eval(ks.pots[kt.pot], k2);
                    const float2 r = R[z * nd * TX + kt.dfield * TX + c];
                    px += u * r.x;
                    py += u * r.y;
                }
            }
            Phi[e] = make_float2((float)px, (float)py);
        }
        __syncthreads();
        // x and y are fixed along a z line, so IFFT_z(-i k_x phi) = -i k_x IFFT_z(phi) and the
        // same for y: one transform serves both; -i k_z phi needs its own.
        float2 *W1 = Wk, *W2 = Wk + nz * TX;
        for (int pass = 0; pass < 2; pass++) {
            for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
                const float2 ph = Phi[e];
                if (pass == 0) {
                    W1[e] = ph;
                } else {
                    const int z = e / TX;
                    const float kz = (g.nz % 2 == 0 && z == g.nz / 2)
                                         ? 0.f : (float)(ks.twopi_over_L[2] * signed_index(z, g.nz));
                    W1[e] = make_float2(kz * ph.y, -kz * ph.x);   // -i k_z phi
                }
            }
            __syncthreads();
            const float2 *O = fft_lines<true>(W1, W2, TX, 1, TX, lz, tw, true, make_fastdiv_dev(TX));
            for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
                const int z = e / TX, c = e - z * TX, kx = kx0 + c;
                if (kx >= g.nxh) continue;
                const long long o = ((long long)z * g.ny + y) * g.hp + kx;
                const float2 v = O[e];
                if (pass == 0) {
                    const float kxv = (g.nx % 2 == 0 && kx == g.nx / 2)
                                          ? 0.f : (float)(ks.twopi_over_L[0] * signed_index(kx, g.nx));
                    const float kyf = nyq_y ? 0.f : (float)kyv;
                    Hg[(long long)(3 * f) * g.hstride + o] = make_float2(kxv * v.y, -kxv * v.x);
                    Hg[(long long)(3 * f + 1) * g.hstride + o] = make_float2(kyf * v.y, -kyf * v.x);
                } else {
                    Hg[(long long)(3 * f + 2) * g.hstride + o] = v;
                }
            }
            __syncthreads();
        }
    }
}

// x-axis inverse pass: gradient fields 2t, 2t+1 packed as Z = G1 + i G2 (Hermitian
// completion of both half spectra), one complex inverse FFT, real -> field 2t,
// imaginary -> field 2t+1; then float4 records (x, y, z, 0) per force group.
__global__ void __launch_bounds__(256) k_xinv(Geom g, FftLine lx, int nfg, const float2 *__restrict__ Hg,
                                              float4 *__restrict__ rec, int L)
{
    extern __shared__ __align__(16) float2 sm[];
    const int n = g.nx, nf = 3 * nfg, nxh = g.nxh, hp = g.hp;
    float2 *A = sm, *B = sm + L * n, *tw = sm + 2 * L * n, *St = tw + n + (n & 1);
    float *Out = reinterpret_cast<float *>(St + 2 * L * hp);
    const long long nlines = (long long)g.ny * g.nz;
    const long long line0 = (long long)blockIdx.x * L;
    const int lv = (int)min((long long)L, nlines - line0);
    const FastDiv dL = make_fastdiv_dev(L), dn = make_fastdiv_dev(n);
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = lx.tw[t];
    for (int pr = 0; pr < (nf + 1) / 2; pr++) {
        const int f1 = 2 * pr, f2 = 2 * pr + 1;
        // consecutive lines are consecutive rows of pitch hp: stage both fields' rows
        tile_load_async(St, hp, Hg + f1 * g.hstride + line0 * hp, hp, lv, hp, nxh);
        if (f2 < nf) tile_load_async(St + L * hp, hp, Hg + f2 * g.hstride + line0 * hp, hp, lv, hp, nxh);
        cp_async_wait_all();
        __syncthreads();
        for (int e = threadIdx.x; e < L * n; e += blockDim.x) {
            const int l = (int)fdiv((unsigned)e, dn), x = e - l * n;
            float2 v = make_float2(0.f, 0.f);
            if (l < lv) {
                const bool direct = x < nxh;
                const int kk = direct ? x : n - x;
                float2 g1 = St[l * hp + kk];
                float2 g2 = (f2 < nf) ? St[L * hp + l * hp + kk] : make_float2(0.f, 0.f);
                if (kk == 0 || (n % 2 == 0 && kk == n / 2)) {
                    g1.y = 0.f;
                    g2.y = 0.f;
                }
                if (!direct) {
                    g1.y = -g1.y;
                    g2.y = -g2.y;
                }
                v = make_float2(g1.x - g2.y, g1.y + g2.x);
            }
            A[e] = v;
        }
        __syncthreads();
        const float2 *R = fft_lines<true>(A, B, L, n, 1, lx, tw, false, dL);
        for (int e = threadIdx.x; e < L * n; e += blockDim.x) {
            Out[f1 * L * n + e] = R[e].x;
            if (f2 < nf) Out[f2 * L * n + e] = R[e].y;
        }
        __syncthreads();
    }
    for (int f = 0; f < nfg; f++) {
        float4 *rf = rec + f * g.M + line0 * n;
        for (int e = threadIdx.x; e < lv * n; e += blockDim.x)
            rf[e] = make_float4(Out[(3 * f) * L * n + e], Out[(3 * f + 1) * L * n + e], Out[(3 * f + 2) * L * n + e], 0.f);
    }
}


// ---- plans and launchers ----
void init_fft_attributes()
{
    set_max_smem(k_xfwd<true>, 200 * 1024);
    set_max_smem(k_xfwd<false>, 200 * 1024);
    set_max_smem(k_ypass<false>, 200 * 1024);
    set_max_smem(k_ypass<true>, 200 * 1024);
    set_max_smem(k_kspace_z, 220 * 1024);
    set_max_smem(k_xinv, 200 * 1024);
}

void build_fft_line(int n, FftLine &pl, float2 *dev_tw_dst)
{
    pl.n = n;
    pl.ns = 0;
    int m = n, p = 1;
    auto push = [&](int r) {
        pl.R[pl.ns] = r;
        pl.P[pl.ns] = p;
        pl.dP[pl.ns] = make_fastdiv((unsigned)p);
        pl.dNB[pl.ns] = make_fastdiv((unsigned)(n / r));
        pl.ns++;
        p *= r;
        m /= r;
    };
    while (m % 4 == 0) push(4);
    while (m % 2 == 0) push(2);
    while (m % 3 == 0) push(3);
    while (m % 5 == 0) push(5);
    for (int r = 7; m > 1; r += 2)
        while (m % r == 0) push(r);
    std::vector<float2> tw(n);
    for (int t = 0; t < n; t++) {
        const double a = -2.0 * M_PI * (double)t / (double)n;
        tw[t] = make_float2((float)cos(a), (float)sin(a));
    }
    cudaMemcpy(dev_tw_dst, tw.data(), n * sizeof(float2), cudaMemcpyHostToDevice);
    pl.tw = dev_tw_dst;
}

cudaError_t launch_xfwd(const Geom &g, const FftLine &lx, int npair, int nd, const float2 *dep,
                        const unsigned long long *dep_fixed, float2 *H, cudaStream_t st)
{
    const int L = lines_per_block(g.nx);
    const long long nlines = (long long)g.ny * g.nz;
    dim3 gx((unsigned)((nlines + L - 1) / L), npair);
    const size_t smx = (size_t)(2 * L * g.nx + g.nx) * sizeof(float2);
    if (dep_fixed)
        k_xfwd<true><<<gx, 256, smx, st>>>(g, lx, nd, dep, dep_fixed, 1.0 / kFixScale, H, L);
    else
        k_xfwd<false><<<gx, 256, smx, st>>>(g, lx, nd, dep, dep_fixed, 1.0, H, L);
    return cudaGetLastError();
}

cudaError_t launch_ypass(const Geom &g, const FftLine &ly, int nfields, int inverse, float2 *H, cudaStream_t st)
{
    const int TX = 16;
    dim3 gy((g.nxh + TX - 1) / TX, g.nz, nfields);
    const size_t smy = (size_t)(2 * g.ny * TX + g.ny) * sizeof(float2);
    if (inverse) k_ypass<true><<<gy, 256, smy, st>>>(g, ly, H, TX);
    else k_ypass<false><<<gy, 256, smy, st>>>(g, ly, H, TX);
    return cudaGetLastError();
}

cudaError_t launch_kspace_z(const Geom &g, const FftLine &lz, const KSpace &ks, const KSpace *ks_dev,
                            const float2 *H, float2 *Hg, double *epart, int energy, int forces,
                            int *nblocks_out, cudaStream_t st)
{
    const int TX = 8;
    const int ndb = ks.nd < 2 ? 2 : ks.nd;
    dim3 grid((g.nxh + TX - 1) / TX, g.ny);
    const size_t sm = (size_t)(2 * ndb * g.nz * TX + g.nz * TX + g.nz) * sizeof(float2) + 8 * sizeof(double);
    k_kspace_z<<<grid, 256, sm, st>>>(g, lz, ks_dev, H, Hg, epart, energy, forces, TX);
    if (nblocks_out) *nblocks_out = (int)(grid.x * grid.y);
    return cudaGetLastError();
}

cudaError_t launch_xinv(const Geom &g, const FftLine &lx, int nfg, const float2 *Hg, float4 *rec, cudaStream_t st)
{
    int L = 768 / g.nx;
    L = L < 1 ? 1 : (L > 8 ? 8 : L);
    const long long nlines = (long long)g.ny * g.nz;
    const size_t smx = (size_t)(2 * L * g.nx + g.nx + (g.nx & 1) + 2 * L * g.hp) * sizeof(float2) +
                       (size_t)3 * nfg * L * g.nx * sizeof(float);
    k_xinv<<<(unsigned)((nlines + L - 1) / L), 256, smx, st>>>(g, lx, nfg, Hg, rec, L);
    return cudaGetLastError();
}

}  // namespace tild
