// tild_fft.cu -- hand-written mixed-radix Stockham 3-D FFT passes fused with the
// k-space potential/gradient multiply (sm_100a).
#include "tild_stencil.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

namespace tild {

// =====================================================================================
// Shared-memory Stockham FFT of L lines of length n (mixed radix, natural order in and
// out).  Element t of line l lives at l*lp + t*ls.  Radix-R pass with p = product of the
// earlier radices: butterfly i reads i + q*n/R, twiddles by W_{pR}^{q*(i mod p)}, writes
// (i - i mod p)*R + i mod p + q*p.  Returns the buffer holding the result.
// =====================================================================================
// complex arithmetic on paired FP32 instructions (FMUL2/FFMA2/FADD2 of sm_100)
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return __ffma2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x), __fmul2_rn(make_float2(a.x, a.x), b));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }

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

__device__ __forceinline__ float2 mul_mi(float2 v) { return make_float2(v.y, -v.x); }   // -i v
__device__ __forceinline__ float2 mul_pi(float2 v) { return make_float2(-v.y, v.x); }   // +i v

// In-register DFT of R points, v[q] <- sum_s v[s] W_R^{+-qs} (forward sign -), R = 2, 3, 4, 5, 7, 8.
template <bool INV>
__device__ __forceinline__ void dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3)
{
    const float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = csub(a1, a3);
    const float2 m = INV ? mul_pi(t3) : mul_mi(t3);
    a0 = cadd(t0, t2);
    a1 = cadd(t1, m);
    a2 = csub(t0, t2);
    a3 = csub(t1, m);
}

template <bool INV, int R>
__device__ __forceinline__ void dft_reg(float2 *v)
{
    if (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        dft4<INV>(v[0], v[1], v[2], v[3]);
    } else if (R == 8) {
        // radix-2 split into even and odd outputs, W_8 twiddles, two 4-point DFTs
        const float c = 0.70710678118654752f;
        float2 a0 = cadd(v[0], v[4]), b0 = csub(v[0], v[4]);
        float2 a1 = cadd(v[1], v[5]), b1 = csub(v[1], v[5]);
        float2 a2 = cadd(v[2], v[6]), b2 = csub(v[2], v[6]);
        float2 a3 = cadd(v[3], v[7]), b3 = csub(v[3], v[7]);
        if (INV) {
            b1 = make_float2(c * (b1.x - b1.y), c * (b1.x + b1.y));     // * W_8^-1
            b2 = mul_pi(b2);                                            // * W_8^-2
            b3 = make_float2(-c * (b3.x + b3.y), c * (b3.x - b3.y));    // * W_8^-3
        } else {
            b1 = make_float2(c * (b1.x + b1.y), c * (b1.y - b1.x));     // * W_8^1
            b2 = mul_mi(b2);                                            // * W_8^2
            b3 = make_float2(c * (b3.y - b3.x), -c * (b3.x + b3.y));    // * W_8^3
        }
        dft4<INV>(a0, a1, a2, a3);
        dft4<INV>(b0, b1, b2, b3);
        v[0] = a0; v[2] = a1; v[4] = a2; v[6] = a3;
        v[1] = b0; v[3] = b1; v[5] = b2; v[7] = b3;
    } else if (R == 3) {
        const float s3 = INV ? 0.86602540378443865f : -0.86602540378443865f;
        const float2 a0 = v[0], t = cadd(v[1], v[2]), u = csub(v[1], v[2]);
        const float2 m = make_float2(a0.x - 0.5f * t.x, a0.y - 0.5f * t.y);
        const float2 iu = make_float2(-s3 * u.y, s3 * u.x);   // i * s3 * u
        v[0] = cadd(a0, t);
        v[1] = cadd(m, iu);
        v[2] = csub(m, iu);
    } else if (R == 5) {
        const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
        const float s1 = INV ? -0.95105651629515357f : 0.95105651629515357f;
        const float s2 = INV ? -0.58778525229247313f : 0.58778525229247313f;
        const float2 a0 = v[0];
        const float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]), t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        const float2 m1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
        const float2 m2 = make_float2(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
        // n1 = s1 t3 + s2 t4, n2 = s2 t3 - s1 t4; b1 = m1 - i n1, b4 = m1 + i n1,
        // b2 = m2 - i n2, b3 = m2 + i n2
        const float2 n1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
        const float2 n2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
        v[0] = make_float2(a0.x + t1.x + t2.x, a0.y + t1.y + t2.y);
        v[1] = make_float2(m1.x + n1.y, m1.y - n1.x);
        v[4] = make_float2(m1.x - n1.y, m1.y + n1.x);
        v[2] = make_float2(m2.x + n2.y, m2.y - n2.x);
        v[3] = make_float2(m2.x - n2.y, m2.y + n2.x);
    } else if (R == 7) {
        // t_k = a_k + a_{7-k}, u_k = a_k - a_{7-k}; b_q = m_q -+ i n_q with
        // m_q = a0 + sum_k cos(2 pi qk/7) t_k, n_q = sum_k sin(2 pi qk/7) u_k
        const float c1 = 0.62348980185873359f, c2 = -0.22252093395631434f, c3 = -0.90096886790241903f;
        const float sg = INV ? -1.f : 1.f;
        const float s1 = sg * 0.78183148246802980f, s2 = sg * 0.97492791218182362f, s3 = sg * 0.43388373911755823f;
        const float2 a0 = v[0];
        const float2 t1 = cadd(v[1], v[6]), t2 = cadd(v[2], v[5]), t3 = cadd(v[3], v[4]);
        const float2 u1 = csub(v[1], v[6]), u2 = csub(v[2], v[5]), u3 = csub(v[3], v[4]);
        const float2 m1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x + c3 * t3.x, a0.y + c1 * t1.y + c2 * t2.y + c3 * t3.y);
        const float2 m2 = make_float2(a0.x + c2 * t1.x + c3 * t2.x + c1 * t3.x, a0.y + c2 * t1.y + c3 * t2.y + c1 * t3.y);
        const float2 m3 = make_float2(a0.x + c3 * t1.x + c1 * t2.x + c2 * t3.x, a0.y + c3 * t1.y + c1 * t2.y + c2 * t3.y);
        const float2 n1 = make_float2(s1 * u1.x + s2 * u2.x + s3 * u3.x, s1 * u1.y + s2 * u2.y + s3 * u3.y);
        const float2 n2 = make_float2(s2 * u1.x - s3 * u2.x - s1 * u3.x, s2 * u1.y - s3 * u2.y - s1 * u3.y);
        const float2 n3 = make_float2(s3 * u1.x - s1 * u2.x + s2 * u3.x, s3 * u1.y - s1 * u2.y + s2 * u3.y);
        v[0] = make_float2(a0.x + t1.x + t2.x + t3.x, a0.y + t1.y + t2.y + t3.y);
        v[1] = cadd(m1, mul_mi(n1));
        v[6] = csub(m1, mul_mi(n1));
        v[2] = cadd(m2, mul_mi(n2));
        v[5] = csub(m2, mul_mi(n2));
        v[3] = cadd(m3, mul_mi(n3));
        v[4] = csub(m3, mul_mi(n3));
    }
}

// One radix-R Stockham stage over L lines: butterfly i of line l reads i + q*nb, is
// twiddled by W_{pR}^{q*(i mod p)} and writes (i - i mod p)*R + i mod p + q*p.
template <bool INV, int R>
__device__ __forceinline__ void fft_stage(const float2 *__restrict__ src, float2 *__restrict__ dst, int L, int lp,
                                          int ls, int n, int p, const FastDiv &dp, const FastDiv &dsplit,
                                          bool line_fast, const float2 *tw)
{
    const int nb = n / R, stride = n / (p * R);
    const int total = L * nb, snb = nb * ls, sp = p * ls;
    for (int w = threadIdx.x; w < total; w += blockDim.x) {
        int l, i;
        if (line_fast) {
            i = (int)fdiv((unsigned)w, dsplit);
            l = w - i * L;
        } else {
            l = (int)fdiv((unsigned)w, dsplit);
            i = w - l * nb;
        }
        const int blk = (int)fdiv((unsigned)i, dp);
        const int k = i - blk * p;
        const int sb = l * lp + i * ls, db = l * lp + (blk * p * R + k) * ls;
        float2 v[R];
#pragma unroll
        for (int q = 0; q < R; q++) v[q] = src[sb + q * snb];
        if (k) {
            const int ks = k * stride;
#pragma unroll
            for (int q = 1; q < R; q++) v[q] = cmul(v[q], twid<INV>(tw, q * ks));
        }
        dft_reg<INV, R>(v);
#pragma unroll
        for (int q = 0; q < R; q++) dst[db + q * sp] = v[q];
    }
}

// Generic radix stage: b_q = sum_s a_s W_{pR}^{s k} W_R^{q s}, R an odd prime (11, 13,
// ...: the plan takes 2, 3, 5 and 7 first).  One thread per output pair (q, R - q) of a
// butterfly, so that a prime line (one butterfly of radix n) still spreads over (n+1)/2
// threads: W_R^{(R-q) s} = conj W_R^{q s}, so both outputs share each term's loads and
// products; each sums its R terms in order s = 0..R-1.
template <bool INV>
__device__ void fft_stage_generic(const float2 *__restrict__ src, float2 *__restrict__ dst, int L, int lp, int ls,
                                  int n, int R, int p, const FastDiv &dp, const FastDiv &dsplit, bool line_fast,
                                  const float2 *tw)
{
    const int nb = n / R, stride = n / (p * R), nR = n / R, items = L * nb, half = (R + 1) / 2;
    for (int w = threadIdx.x; w < items * half; w += blockDim.x) {
        const int qq = w / items, wi = w - qq * items;
        int l, i;
        if (line_fast) {
            i = (int)fdiv((unsigned)wi, dsplit);
            l = wi - i * L;
        } else {
            l = (int)fdiv((unsigned)wi, dsplit);
            i = wi - l * nb;
        }
        const int k = i - p * (int)fdiv((unsigned)i, dp);
        const float2 *s = src + l * lp;
        const int j = (i - k) * R + k;
        float2 acc = make_float2(0.f, 0.f), acm = make_float2(0.f, 0.f);   // b_q, b_{R-q}
        int e = 0;   // (qq * ss) mod R
        for (int ss = 0; ss < R; ss++) {
            float2 v = s[(i + ss * nb) * ls];
            if (k && ss) v = cmul(v, twid<INV>(tw, ss * k * stride));
            if (e) {
                const float2 t = twid<INV>(tw, e * nR);
                const float xr = v.x * t.x, yi = v.y * t.y, xi = v.x * t.y, yr = v.y * t.x;
                acc.x += xr - yi;
                acc.y += xi + yr;
                acm.x += xr + yi;
                acm.y += yr - xi;
            } else {
                acc = cadd(acc, v);
                acm = cadd(acm, v);
            }
            e += qq;
            if (e >= R) e -= R;
        }
        dst[l * lp + (j + qq * p) * ls] = acc;
        if (qq) dst[l * lp + (j + (R - qq) * p) * ls] = acm;
    }
}

// Shared-memory Stockham FFT of L lines of length n (mixed radix, natural order in and
// out).  Element t of line l lives at l*lp + t*ls.  line_fast: consecutive threads take
// consecutive lines (lines interleaved, ls = L), else consecutive butterflies of a line.
// dL divides by L.  Returns the buffer holding the result.
template <bool INV>
__device__ float2 *fft_lines(float2 *a, float2 *b, int L, int lp, int ls, const FftLine &pl,
                             const float2 *tw, bool line_fast, const FastDiv &dL)
{
    const int n = pl.n;
    for (int s = 0; s < pl.ns; ++s) {
        const int R = pl.R[s], p = pl.P[s];
        const FastDiv &dsplit = line_fast ? dL : pl.dNB[s];
        switch (R) {
            case 8: fft_stage<INV, 8>(a, b, L, lp, ls, n, p, pl.dP[s], dsplit, line_fast, tw); break;
            case 4: fft_stage<INV, 4>(a, b, L, lp, ls, n, p, pl.dP[s], dsplit, line_fast, tw); break;
            case 2: fft_stage<INV, 2>(a, b, L, lp, ls, n, p, pl.dP[s], dsplit, line_fast, tw); break;
            case 3: fft_stage<INV, 3>(a, b, L, lp, ls, n, p, pl.dP[s], dsplit, line_fast, tw); break;
            case 5: fft_stage<INV, 5>(a, b, L, lp, ls, n, p, pl.dP[s], dsplit, line_fast, tw); break;
            case 7: fft_stage<INV, 7>(a, b, L, lp, ls, n, p, pl.dP[s], dsplit, line_fast, tw); break;
            default: fft_stage_generic<INV>(a, b, L, lp, ls, n, R, p, pl.dP[s], dsplit, line_fast, tw); break;
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
    const FastDiv dc = make_fastdiv_dev((unsigned)cpr);
    for (int e = threadIdx.x; e < rows * cpr; e += blockDim.x) {
        const int r = (int)fdiv((unsigned)e, dc), c2 = (e - r * cpr) << 1;
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
__device__ __forceinline__ void xfwd_body(const Geom &g, const FftLine &lx, int nd, const float2 *__restrict__ dep,
                                          const unsigned long long *__restrict__ depfix, double fscale,
                                          float2 *__restrict__ H, int L, unsigned vbx, unsigned vby)
{
    extern __shared__ __align__(16) float2 sm[];
    const int n = g.nx;
    float2 *A = sm, *B = sm + L * n, *tw = sm + 2 * L * n;
    const int pair = vby;
    const long long nlines = (long long)g.ny * g.nz;
    const long long line0 = (long long)vbx * L;
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
    const FastDiv dh = make_fastdiv_dev((unsigned)nxh);
    for (int e = threadIdx.x; e < L * nxh; e += blockDim.x) {
        const int l = (int)fdiv((unsigned)e, dh), k = e - l * nxh;
        const long long gl = line0 + l;
        if (gl >= nlines) continue;
        const float2 zk = R[l * n + k], zm = R[l * n + (k == 0 ? 0 : n - k)];
        const long long o = gl * g.hp + k;
        H[(2 * pair) * g.hstride + o] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        if (2 * pair + 1 < nd)
            H[(2 * pair + 1) * g.hstride + o] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
}
template <bool FIXED>
__global__ void __launch_bounds__(256) k_xfwd(Geom g, FftLine lx, int nd, const float2 *__restrict__ dep,
                                              const unsigned long long *__restrict__ depfix,
                                              double fscale, float2 *__restrict__ H, int L)
{
    xfwd_body<FIXED>(g, lx, nd, dep, depfix, fscale, H, L, blockIdx.x, blockIdx.y);
}

// the x forward pass over several replicas: CTA b of replica r takes (b % gx, b / gx) of
// the replica's grid (gx line blocks, one row per field pair)
// The batch forms of the x forward and y passes read their replica's geometry from the
// device table, which costs registers; bounded to six CTAs per SM (40 registers), like the
// single-box kernels (C3: 4.99 -> 4.94 ms per batch step).
template <bool FIXED>
__global__ void __launch_bounds__(256, 6) k_xfwd_batch(const BatchRep *__restrict__ reps, const int *__restrict__ pre, int R)
{
    const int r = batch_replica(pre, R, blockIdx.x);
    const BatchRep &b = reps[r];
    const unsigned lb = blockIdx.x - pre[r];
    const unsigned gx = (unsigned)(((long long)b.g.ny * b.g.nz + b.Lx - 1) / b.Lx);
    xfwd_body<FIXED>(b.g, b.lx, b.nd, b.dep, b.depfix, FIXED ? 1.0 / kFixScale : 1.0, b.H, b.Lx, lb % gx, lb / gx);
}

// y-axis pass over TX half-spectrum columns of one z plane of field blockIdx.z.
template <bool INV, int TX>
__device__ __forceinline__ void ypass_body(const Geom &g, const FftLine &ly, float2 *__restrict__ H, unsigned vbx,
                                           unsigned vby, unsigned vbz)
{
    extern __shared__ __align__(16) float2 sm[];
    const int ny = g.ny;
    float2 *A = sm, *B = sm + ny * TX, *tw = sm + 2 * ny * TX;
    const int kx0 = vbx * TX;
    const long long base = (long long)vbz * g.hstride + (long long)vby * ny * g.hp + kx0;
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
template <bool INV, int TX>
__global__ void __launch_bounds__(256) k_ypass(Geom g, FftLine ly, float2 *__restrict__ H)
{
    ypass_body<INV, TX>(g, ly, H, blockIdx.x, blockIdx.y, blockIdx.z);
}

// the y pass over several replicas: CTA b of replica r takes (x, z plane, field) of the
// replica's grid of ceil(nxh / TX) x nz x fields (density fields forward, 3F inverse)
template <bool INV, int TX>
__global__ void __launch_bounds__(256, 6) k_ypass_batch(const BatchRep *__restrict__ reps, const int *__restrict__ pre, int R)
{
    const int r = batch_replica(pre, R, blockIdx.x);
    const BatchRep &b = reps[r];
    const unsigned lb = blockIdx.x - pre[r];
    const unsigned gx = (unsigned)((b.g.nxh + TX - 1) / TX), gy = (unsigned)b.g.nz;
    ypass_body<INV, TX>(b.g, b.ly, INV ? b.Hg : b.H, lb % gx, (lb / gx) % gy, lb / (gx * gy));
}

// û(k) of each potential kind, FP64 (ps_potentialGaussian.cu:38-46,
// ps_potentialErf2.cu:111-124, ps_potentialErfG.cu:177-190, ps_potentialCharges.cu:241-258),
// as amplitude x shape: the shape is fixed for a box, the amplitude follows the ramp.
__device__ double uk_shape(const PotDev &p, double k2)
{
    const double PI4 = 12.566370614359172953850573533118;
    if (p.kind == POT_WALL) return 0.0;   // a per-particle term, nothing in k-space
    if (p.kind == POT_GAUSSIAN) return exp(-0.5 * k2 * p.sig2);
    if (p.kind == POT_CHARGES) return k2 > 0.0 ? PI4 * p.lB * exp(-k2 * p.sig2) / k2 : 0.0;
    const double R = p.Rp;
    double t;
    if (k2 == 0.0) {
        t = PI4 * R * R * R / 3.0;
        return p.kind == POT_ERF2 ? t * t : t;
    }
    const double k = sqrt(k2);
    double sn, cs;
    sincos(R * k, &sn, &cs);
    t = PI4 * (sn - R * k * cs) / (k2 * k);
    const double gs = exp(-0.5 * k2 * p.sig2);
    return p.kind == POT_ERF2 ? gs * t * t : gs * t;
}

__device__ __forceinline__ double uk_amp(const PotDev &p) { return p.kind == POT_CHARGES ? 1.0 : p.amp; }

__device__ __forceinline__ double uk_eval(const PotDev &p, double k2) { return uk_amp(p) * uk_shape(p, k2); }

// (d û / d k) / k for k > 0, FP64, amplitude included: the strain derivative of the pair
// energy.  gaussian: -sigma^2 û; charges: û (-2 sigma^2 - 2/k^2); erf2/erfG with
// t = 4 pi (sin Rk - Rk cos Rk)/k^3: A g t^(p-1) (-sigma^2 t + p t'/k),
// t'/k = 4 pi (R^2 sin(Rk)/k^3 - 3 (sin Rk - Rk cos Rk)/k^5).
__device__ double uk_dk_over_k(const PotDev &p, double k2)
{
    if (k2 <= 0.0 || p.kind == POT_WALL) return 0.0;
    if (p.kind == POT_GAUSSIAN) return -p.sig2 * uk_eval(p, k2);
    if (p.kind == POT_CHARGES) return uk_eval(p, k2) * (-2.0 * p.sig2 - 2.0 / k2);
    const double PI4 = 12.566370614359172953850573533118;
    const double R = p.Rp, k = sqrt(k2);
    double sn, cs;
    sincos(R * k, &sn, &cs);
    const double f = sn - R * k * cs;
    const double t = PI4 * f / (k2 * k);
    const double dt_k = PI4 * (R * R * sn / (k2 * k) - 3.0 * f / (k2 * k2 * k));
    const double gs = exp(-0.5 * k2 * p.sig2);
    return p.kind == POT_ERF2 ? p.amp * gs * t * (-p.sig2 * t + 2.0 * dt_k) : p.amp * gs * (-p.sig2 * t + dt_k);
}

__device__ __forceinline__ int signed_index(int i, int n) { return (i < n - i) ? i : i - n; }

// FP32 shape table of every potential over the half spectrum, layout of one density field
// (the reference keeps û(k) as a precomputed FP32 array, ps_potential.cu:41-78).
__global__ void k_uk_table(Geom g, const KSpace *__restrict__ ksp, float *__restrict__ tab)
{
    const KSpace &ks = *ksp;
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= g.hstride) return;
    const int kx = (int)(o % g.hp);
    const long long zy = o / g.hp;
    const int y = (int)(zy % g.ny), z = (int)(zy / g.ny);
    double k2 = 0.0;
    if (kx < g.nxh) {
        const double kxv = ks.twopi_over_L[0] * signed_index(kx, g.nx);
        const double kyv = ks.twopi_over_L[1] * signed_index(y, g.ny);
        const double kzv = ks.twopi_over_L[2] * signed_index(z, g.nz);
        k2 = kxv * kxv + kyv * kyv + kzv * kzv;
    }
    for (int p = 0; p < ks.npots; p++)
        tab[(long long)p * g.hstride + o] = kx < g.nxh ? (float)uk_shape(ks.pots[p], k2) : 0.f;
}

__device__ __forceinline__ size_t kspace_uk_offset_dev(int nz, int nsets, int tx)
{
    const size_t b = (size_t)(2 * nsets * nz * tx + nz) * sizeof(float2) + 8 * sizeof(double);
    return (b + 15) & ~(size_t)15;
}

// Fused z pass: forward z FFT of every density field, k-space combine, gradient and
// inverse z FFT of each gradient field; FP64 energies on request.
template <int TX>
__device__ __forceinline__ void kspace_body(const Geom &g, const FftLine &lz, const KSpace *__restrict__ ksp,
                                            const float2 *__restrict__ H, const float *__restrict__ uk,
                                            float2 *__restrict__ Hg, double *__restrict__ epart, int energy, int forces,
                                            unsigned vbx, unsigned vby, unsigned vgx)
{
    extern __shared__ __align__(16) float2 sm[];
    const KSpace &ks = *ksp;
    const int nz = g.nz, nd = ks.nd;
    const int ndb = nd < 2 ? 2 : nd;
    // two buffers of nsets line sets (nsets = max(density fields, 2 x force groups)),
    // each set TX lines of nz points, sets interleaved per z row
    const int nsets = ndb > 2 * ks.nfg ? ndb : 2 * ks.nfg;
    float2 *Rho = sm, *S = sm + nsets * nz * TX, *tw = sm + 2 * nsets * nz * TX;
    double *red = reinterpret_cast<double *>(tw + nz);
    const int kx0 = vbx * TX, y = vby;
    for (int t = threadIdx.x; t < nz; t += blockDim.x) tw[t] = lz.tw[t];
    for (int d = 0; d < nd; d++)
        tile_load_async(Rho + d * TX, nd * TX, H + d * g.hstride + (long long)y * g.hp + kx0, (long long)g.ny * g.hp,
                        nz, TX, g.nxh - kx0);
    // the u(k) rows of the block's columns, for the combine: whole rows of TX floats (the
    // table's row pitch hp covers every block's TX columns)
    const size_t ukoff = kspace_uk_offset_dev(nz, nsets, TX);
    float *ukt = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(sm) + ukoff);
    if (forces)
        for (int e = threadIdx.x; e < ks.npots * nz; e += blockDim.x) {
            const int pt = e / nz, z = e - pt * nz;
            const float *src = uk + pt * g.hstride + ((long long)z * g.ny + y) * g.hp + kx0;
            const unsigned s = (unsigned)__cvta_generic_to_shared(ukt + e * TX);
            if (TX == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
            else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(src) : "memory");
        }
    cp_async_wait_all();
    __syncthreads();
    float2 *R = fft_lines<false>(Rho, S, nd * TX, 1, nd * TX, lz, tw, true, make_fastdiv_dev(nd * TX));
    float2 *Wk = (R == Rho) ? S : Rho;  // the other buffer, free for the inverse transforms
    const int ky = signed_index(y, g.ny);
    const double kyv = ks.twopi_over_L[1] * ky;
    const bool nyq_y = (g.ny % 2 == 0) && (y == g.ny / 2);

    if (energy) {
        // per potential U_t = fac sum_k u(k) Re(rho_I* rho_J) (Parseval); the summed
        // virial W_ab = sum_t [U_t delta_ab + fac sum_k (u'(k)/k) k_a k_b Re(...)] keeps only
        // the second part here (the host adds the first)
        double acc[kMaxPots];
        double vir[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int t = 0; t < ks.neterms; t++) acc[t] = 0.0;
        for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
            const int z = e / TX, c = e - z * TX, kx = kx0 + c;
            if (kx >= g.nxh) continue;
            const double kxv = ks.twopi_over_L[0] * signed_index(kx, g.nx);
            const double kzv = ks.twopi_over_L[2] * signed_index(z, g.nz);
            const double k2 = kxv * kxv + kyv * kyv + kzv * kzv;
            const double wgt = (kx == 0 || (g.nx % 2 == 0 && kx == g.nx / 2)) ? 1.0 : 2.0;
            double sv = 0.0;
            for (int t = 0; t < ks.neterms; t++) {
                const ETerm &et = ks.eterms[t];
                const float2 rI = R[z * nd * TX + et.dI * TX + c], rJ = R[z * nd * TX + et.dJ * TX + c];
                const double re = (double)rJ.x * rI.x + (double)rJ.y * rI.y;
                acc[t] += wgt * et.fac * uk_eval(ks.pots[et.pot], k2) * re;
                sv += wgt * et.fac * uk_dk_over_k(ks.pots[et.pot], k2) * re;
            }
            vir[0] += sv * kxv * kxv;
            vir[1] += sv * kyv * kyv;
            vir[2] += sv * kzv * kzv;
            vir[3] += sv * kxv * kyv;
            vir[4] += sv * kxv * kzv;
            vir[5] += sv * kyv * kzv;
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        const long long blin = (long long)vby * vgx + vbx;
        const int ncol = ks.neterms + 6;
        for (int t = 0; t < ncol; t++) {
            double v = t < ks.neterms ? acc[t] : sel<5>(vir, t - ks.neterms);
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp] = v;
            __syncthreads();
            if (threadIdx.x == 0) {
                double s = 0.0;
                for (int w = 0; w < nw; w++) s += red[w];
                epart[blin * ncol + t] = s;
            }
            __syncthreads();
        }
    }
    if (!forces) return;

    __shared__ float tcoef[kMaxTerms];
    __shared__ int tfg[kMaxTerms], tpot[kMaxTerms], tdf[kMaxTerms];
    const int nterms = ks.nterms;
    for (int t = threadIdx.x; t < nterms; t += blockDim.x) {
        const KTerm &kt = ks.terms[t];
        tcoef[t] = (float)(kt.mult * uk_amp(ks.pots[kt.pot]));
        tfg[t] = kt.fgroup;
        tpot[t] = kt.pot;
        tdf[t] = kt.dfield;
    }
    __syncthreads();
    // line set 2f: phi_f = sum c u rho; set 2f+1: -i k_z phi_f.  x and y are fixed along a z
    // line, so IFFT_z(-i k_x phi) = -i k_x IFFT_z(phi) and the same for y: one transform of
    // phi serves both, -i k_z phi needs its own.  All 2F sets go through one transform.
    const int nf2 = 2 * ks.nfg, pitch = nf2 * TX;
    for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
        const int z = e / TX, c = e - z * TX, kx = kx0 + c;
        const float kz = (g.nz % 2 == 0 && z == g.nz / 2) ? 0.f : (float)(ks.twopi_over_L[2] * signed_index(z, g.nz));
        for (int f = 0; f < ks.nfg; f++) {
            float px = 0.f, py = 0.f;
            if (kx < g.nxh) {
                for (int t = 0; t < nterms; t++) {
                    if (tfg[t] != f) continue;
                    const float u = tcoef[t] * ukt[(tpot[t] * nz + z) * TX + c];
                    const float2 r = R[z * nd * TX + tdf[t] * TX + c];
                    px = fmaf(u, r.x, px);
                    py = fmaf(u, r.y, py);
                }
            }
            Wk[z * pitch + (2 * f) * TX + c] = make_float2(px, py);
            Wk[z * pitch + (2 * f + 1) * TX + c] = make_float2(kz * py, -kz * px);
        }
    }
    __syncthreads();
    float2 *other = (Wk == Rho) ? S : Rho;
    const float2 *O = fft_lines<true>(Wk, other, nf2 * TX, 1, nf2 * TX, lz, tw, true, make_fastdiv_dev(nf2 * TX));
    const float kyf = nyq_y ? 0.f : (float)kyv;
    for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
        const int z = e / TX, c = e - z * TX, kx = kx0 + c;
        if (kx >= g.nxh) continue;
        const long long o = ((long long)z * g.ny + y) * g.hp + kx;
        const float kxv = (g.nx % 2 == 0 && kx == g.nx / 2) ? 0.f : (float)(ks.twopi_over_L[0] * signed_index(kx, g.nx));
        for (int f = 0; f < ks.nfg; f++) {
            const float2 v = O[z * pitch + (2 * f) * TX + c], w = O[z * pitch + (2 * f + 1) * TX + c];
            Hg[(long long)(3 * f) * g.hstride + o] = make_float2(kxv * v.y, -kxv * v.x);
            Hg[(long long)(3 * f + 1) * g.hstride + o] = make_float2(kyf * v.y, -kyf * v.x);
            Hg[(long long)(3 * f + 2) * g.hstride + o] = w;
        }
    }
}
template <int TX>
__global__ void __launch_bounds__(256) k_kspace_z(Geom g, FftLine lz, const KSpace *__restrict__ ksp, const float2 *__restrict__ H,
                                                  const float *__restrict__ uk, float2 *__restrict__ Hg,
                                                  double *__restrict__ epart, int energy, int forces)
{
    kspace_body<TX>(g, lz, ksp, H, uk, Hg, epart, energy, forces, blockIdx.x, blockIdx.y, gridDim.x);
}

// the k-space z pass over several replicas (forces only: no energy partials)
template <int TX>
__global__ void __launch_bounds__(256) k_kspace_batch(const BatchRep *__restrict__ reps, const int *__restrict__ pre, int R)
{
    const int r = batch_replica(pre, R, blockIdx.x);
    const BatchRep &b = reps[r];
    const unsigned lb = blockIdx.x - pre[r];
    const unsigned gx = (unsigned)((b.g.nxh + TX - 1) / TX);
    kspace_body<TX>(b.g, b.lz, b.ks, b.H, b.uk, b.Hg, nullptr, 0, 1, lb % gx, lb / gx, gx);
}

// Structure factor pass (after the x and y forward passes of one field): z FFT of a
// column block, then |rho^(k)|^2 * scale binned by |k| in FP64 over the full grid (the
// half spectrum's interior kx columns stand for their Hermitian partners too).
// bins[3b] += S, bins[3b+1] += |k|, bins[3b+2] += count.
template <int TX>
__global__ void __launch_bounds__(256) k_sk_z(Geom g, FftLine lz, const float2 *__restrict__ H, double tx,
                                              double ty, double tz, double scale, int nbins, double inv_dk,
                                              double *__restrict__ bins)
{
    extern __shared__ __align__(16) float2 sm[];
    const int nz = g.nz;
    float2 *A = sm, *B = sm + nz * TX, *tw = sm + 2 * nz * TX;
    const int kx0 = blockIdx.x * TX, y = blockIdx.y;
    for (int t = threadIdx.x; t < nz; t += blockDim.x) tw[t] = lz.tw[t];
    tile_load_async(A, TX, H + (long long)y * g.hp + kx0, (long long)g.ny * g.hp, nz, TX, g.nxh - kx0);
    cp_async_wait_all();
    __syncthreads();
    const float2 *R = fft_lines<false>(A, B, TX, 1, TX, lz, tw, true, make_fastdiv_dev(TX));
    const double kyv = ty * signed_index(y, g.ny);
    for (int e = threadIdx.x; e < nz * TX; e += blockDim.x) {
        const int z = e / TX, c = e - z * TX, kx = kx0 + c;
        if (kx >= g.nxh) continue;
        const double kxv = tx * signed_index(kx, g.nx), kzv = tz * signed_index(z, g.nz);
        const double k = sqrt(kxv * kxv + kyv * kyv + kzv * kzv);
        const int b = (int)(k * inv_dk);
        if (b >= nbins) continue;
        const double w = (kx == 0 || (g.nx % 2 == 0 && kx == g.nx / 2)) ? 1.0 : 2.0;
        const float2 v = R[e];
        atomicAdd(bins + 3 * b, w * scale * ((double)v.x * v.x + (double)v.y * v.y));
        atomicAdd(bins + 3 * b + 1, w * k);
        atomicAdd(bins + 3 * b + 2, w);
    }
}

// x-axis inverse pass: gradient fields 2t, 2t+1 packed as Z = G1 + i G2 (Hermitian
// completion of both half spectra), one complex inverse FFT, real -> field 2t,
// imaginary -> field 2t+1; then float4 records (x, y, z, 0) per force group.  A block
// takes L lines of every field: all rows are staged at once, every pair is transformed
// in one pass over npair*L lines, and the records are written from the transform.  The
// transform's lines are interleaved (element x of line j at x*ls + j, ls = npair*L made
// odd): each radix stage then reads and writes consecutive lines of one element in
// consecutive lanes, and the record writes, which step along x, read rows ls apart --
// distinct bank pairs for every half warp, where lines stored one after another put the
// first stages' outputs R complex values apart (a 16-way conflict at R = 8).
__host__ __device__ inline int xinv_pitch(int nf, int L)
{
    const int lines = ((nf + 1) / 2) * L;
    return lines | 1;
}

__device__ __forceinline__ void xinv_body(const Geom &g, const FftLine &lx, int nfg, const float2 *__restrict__ Hg,
                                          float4 *__restrict__ rec, const RecLayout &rl, int L, unsigned vbx)
{
    extern __shared__ __align__(16) float2 sm[];
    const int n = g.nx, nf = 3 * nfg, npair = (nf + 1) / 2, nxh = g.nxh, hp = g.hp;
    const int lines = npair * L, ls = xinv_pitch(nf, L);
    const int stsz = nf * L * hp, bsz = n * ls;
    // St receives 16-byte cp.async copies: start it on an even complex offset
    float2 *A = sm, *St = sm + ((bsz + 1) & ~1), *tw = St + (stsz > bsz ? stsz : bsz);
    const long long nlines = (long long)g.ny * g.nz;
    const long long line0 = (long long)vbx * L;
    const int lv = (int)min((long long)L, nlines - line0);
    const FastDiv dn = make_fastdiv_dev(n), dL = make_fastdiv_dev(L), dlines = make_fastdiv_dev(lines);
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = lx.tw[t];
    // consecutive lines are consecutive rows of pitch hp: stage every field's rows
    for (int f = 0; f < nf; f++)
        tile_load_async(St + f * L * hp, hp, Hg + f * g.hstride + line0 * hp, hp, lv, hp, nxh);
    cp_async_wait_all();
    __syncthreads();
    // transform line j = pr * L + l holds pair pr of line l; element x of it sits at x*ls + j
    // (lanes step along x: contiguous reads of the staged rows, writes ls apart)
    for (int e = threadIdx.x; e < n * lines; e += blockDim.x) {
        const int j = (int)fdiv((unsigned)e, dn), x = e - j * n;
        const int pr = (int)fdiv((unsigned)j, dL), l = j - pr * L;
        const int f1 = 2 * pr, f2 = 2 * pr + 1;
        float2 v = make_float2(0.f, 0.f);
        if (l < lv) {
            const bool direct = x < nxh;
            const int kk = direct ? x : n - x;
            float2 g1 = St[(f1 * L + l) * hp + kk];
            float2 g2 = (f2 < nf) ? St[(f2 * L + l) * hp + kk] : make_float2(0.f, 0.f);
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
        A[x * ls + j] = v;
    }
    __syncthreads();
    const float2 *R = fft_lines<true>(A, St, lines, 1, ls, lx, tw, true, dlines);
    // field k is component k % 2 of pair k / 2
    auto comp = [&](int k, int l, int x) {
        const float2 v = R[x * ls + (k >> 1) * L + l];
        return (k & 1) ? v.y : v.x;
    };
    if (rl.paired) {
        // plane A (g0.x, g0.y, g1.x, g1.y) or (x, y, z, 0), plane B (g0.z, g1.z), at the
        // point and at every ghost of it: the padded coordinates c' in [-gl, n + gh) with
        // c' = c mod n along each axis
        const FastDiv dny = make_fastdiv_dev(g.ny);
        for (int e = threadIdx.x; e < lv * n; e += blockDim.x) {
            const int l = (int)fdiv((unsigned)e, dn), x = e - l * n;
            const int line = (int)line0 + l, z = (int)fdiv((unsigned)line, dny), y = line - z * g.ny;
            float4 a;
            float2 b = make_float2(0.f, 0.f);
            if (nfg == 2) {
                a = make_float4(comp(0, l, x), comp(1, l, x), comp(3, l, x), comp(4, l, x));
                b = make_float2(comp(2, l, x), comp(5, l, x));
            } else {
                a = make_float4(comp(0, l, x), comp(1, l, x), comp(2, l, x), 0.f);
            }
            const int gl = rl.gl;
            const long long r0 = ((long long)(z + gl) * rl.py + (y + gl)) * rl.px + gl + x;
            rl.A[r0] = a;
            if (nfg == 2) rl.B[r0] = b;
            // ghosts: only points within gl of the top or gh of the bottom of an axis have any
            if (x < rl.gh[0] || x >= n - gl || y < rl.gh[1] || y >= g.ny - gl || z < rl.gh[2] || z >= g.nz - gl) {
                // the lowest copy: c itself unless c sits within gl of the top (then c - n,
                // or lower still on a grid of fewer than gl points)
                auto low = [gl](int c, int m) { return c + gl < m ? c : c - m * ((c + gl) / m); };
                for (int zz = low(z, g.nz); zz < g.nz + rl.gh[2]; zz += g.nz)
                    for (int yy = low(y, g.ny); yy < g.ny + rl.gh[1]; yy += g.ny) {
                        const long long rb = ((long long)(zz + gl) * rl.py + (yy + gl)) * rl.px + gl;
                        for (int xx = low(x, n); xx < n + rl.gh[0]; xx += n) {
                            if (zz == z && yy == y && xx == x) continue;
                            rl.A[rb + xx] = a;
                            if (nfg == 2) rl.B[rb + xx] = b;
                        }
                    }
            }
        }
        return;
    }
    for (int f = 0; f < nfg; f++) {
        float4 *rf = rec + f * g.M + line0 * n;
        for (int e = threadIdx.x; e < lv * n; e += blockDim.x) {
            const int l = (int)fdiv((unsigned)e, dn), x = e - l * n;
            rf[e] = make_float4(comp(3 * f, l, x), comp(3 * f + 1, l, x), comp(3 * f + 2, l, x), 0.f);
        }
    }
}
__global__ void __launch_bounds__(256) k_xinv(Geom g, FftLine lx, int nfg, const float2 *__restrict__ Hg,
                                              float4 *__restrict__ rec, RecLayout rl, int L)
{
    xinv_body(g, lx, nfg, Hg, rec, rl, L, blockIdx.x);
}

// the x inverse pass over several replicas
__global__ void __launch_bounds__(256) k_xinv_batch(const BatchRep *__restrict__ reps, const int *__restrict__ pre, int R)
{
    const int r = batch_replica(pre, R, blockIdx.x);
    const BatchRep &b = reps[r];
    xinv_body(b.g, b.lx, b.nfg, b.Hg, b.rec, b.rl, b.Lxi, blockIdx.x - pre[r]);
}


// ---- plans and launchers ----
constexpr int kTXy = 16;   // half-spectrum columns per y-pass block
constexpr int kTXz = 8;    // half-spectrum columns per structure-factor z block
constexpr size_t kKspaceSmemMax = 220 * 1024;
void init_fft_attributes()
{
    set_max_smem(k_xfwd<true>, 200 * 1024);
    set_max_smem(k_xfwd<false>, 200 * 1024);
    set_max_smem(k_ypass<false, kTXy>, 200 * 1024);
    set_max_smem(k_ypass<true, kTXy>, 200 * 1024);
    set_max_smem(k_kspace_z<8>, kKspaceSmemMax);
    set_max_smem(k_kspace_z<4>, kKspaceSmemMax);
    set_max_smem(k_kspace_z<2>, kKspaceSmemMax);
    set_max_smem(k_sk_z<kTXz>, 200 * 1024);
    set_max_smem(k_xinv, 200 * 1024);
    set_max_smem(k_xfwd_batch<true>, 200 * 1024);
    set_max_smem(k_xfwd_batch<false>, 200 * 1024);
    set_max_smem(k_ypass_batch<false, kTXy>, 200 * 1024);
    set_max_smem(k_ypass_batch<true, kTXy>, 200 * 1024);
    set_max_smem(k_kspace_batch<4>, kKspaceSmemMax);
    set_max_smem(k_kspace_batch<2>, kKspaceSmemMax);
    set_max_smem(k_xinv_batch, 200 * 1024);
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
    while (m % 8 == 0) push(8);
    while (m % 4 == 0) push(4);
    while (m % 2 == 0) push(2);
    while (m % 3 == 0) push(3);
    while (m % 5 == 0) push(5);
    while (m % 7 == 0) push(7);
    for (int r = 11; m > 1; r += 2)
        while (m % r == 0) push(r);
    // the generic stage computes output pairs (q, R - q) and so needs an odd radix
    for (int s = 0; s < pl.ns; s++)
        if (pl.R[s] != 2 && pl.R[s] != 4 && pl.R[s] != 8 && pl.R[s] % 2 == 0) {
            std::fprintf(stderr, "tild: FFT plan of length %d has an even radix %d outside {2,4,8}\n", n, pl.R[s]);
            std::abort();
        }
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
    constexpr int TX = kTXy;
    dim3 gy((g.nxh + TX - 1) / TX, g.nz, nfields);
    const size_t smy = (size_t)(2 * g.ny * TX + g.ny) * sizeof(float2);
    if (inverse) k_ypass<true, TX><<<gy, 256, smy, st>>>(g, ly, H);
    else k_ypass<false, TX><<<gy, 256, smy, st>>>(g, ly, H);
    return cudaGetLastError();
}

// two line-set buffers and the twiddles (float2), the reduction slots, then the staged
// u(k) rows of every potential (float, 16-byte aligned)
static size_t kspace_uk_offset(const Geom &g, int nsets, int tx)
{
    const size_t b = (size_t)(2 * nsets * g.nz * tx + g.nz) * sizeof(float2) + 8 * sizeof(double);
    return (b + 15) & ~(size_t)15;
}

static size_t kspace_smem(const Geom &g, int nd, int nfg, int npots, int tx)
{
    const int ndb = nd < 2 ? 2 : nd;
    const int nsets = ndb > 2 * nfg ? ndb : 2 * nfg;   // as in the kernel
    return kspace_uk_offset(g, nsets, tx) + (size_t)npots * g.nz * tx * sizeof(float);
}

int kspace_tile_width(const Geom &g, int nd, int nfg, int npots)
{
    for (int tx : {4, 2})   // 4 columns: four blocks per SM at C2 sizes, better than 8 at two
        if (kspace_smem(g, nd, nfg, npots, tx) <= kKspaceSmemMax) return tx;
    return 0;
}

cudaError_t launch_kspace_z(const Geom &g, const FftLine &lz, const KSpace &ks, const KSpace *ks_dev,
                            const float2 *H, const float *uk, float2 *Hg, double *epart, int energy, int forces,
                            int *nblocks_out, cudaStream_t st)
{
    const int tx = kspace_tile_width(g, ks.nd, ks.nfg, ks.npots);
    if (tx == 0) return cudaErrorInvalidConfiguration;
    dim3 grid((g.nxh + tx - 1) / tx, g.ny);
    const size_t sm = kspace_smem(g, ks.nd, ks.nfg, ks.npots, tx);
    if (tx == 8) k_kspace_z<8><<<grid, 256, sm, st>>>(g, lz, ks_dev, H, uk, Hg, epart, energy, forces);
    else if (tx == 4) k_kspace_z<4><<<grid, 256, sm, st>>>(g, lz, ks_dev, H, uk, Hg, epart, energy, forces);
    else k_kspace_z<2><<<grid, 256, sm, st>>>(g, lz, ks_dev, H, uk, Hg, epart, energy, forces);
    if (nblocks_out) *nblocks_out = (int)(grid.x * grid.y);
    return cudaGetLastError();
}

// lines per block of the x inverse pass (at most 4k complex points: three blocks per SM
// on a 192-point line) and its shared memory
static int xinv_lines(const Geom &g, int nfg)
{
    const int npair = (3 * nfg + 1) / 2;
    const int L = 4096 / (npair * g.nx);
    return L < 1 ? 1 : (L > 16 ? 16 : L);
}

static size_t xinv_smem(const Geom &g, int nfg, int L)
{
    const int nf = 3 * nfg;
    const size_t bsz = (size_t)g.nx * xinv_pitch(nf, L), stsz = (size_t)nf * L * g.hp;
    return (((bsz + 1) & ~(size_t)1) + std::max(bsz, stsz) + g.nx) * sizeof(float2);
}

cudaError_t launch_xinv(const Geom &g, const FftLine &lx, int nfg, const float2 *Hg, float4 *rec, const RecLayout &rl,
                        cudaStream_t st)
{
    if (rl.paired && (rl.nfg != nfg || nfg < 1 || nfg > 2)) return cudaErrorInvalidValue;
    const int L = xinv_lines(g, nfg);
    const long long nlines = (long long)g.ny * g.nz;
    k_xinv<<<(unsigned)((nlines + L - 1) / L), 256, xinv_smem(g, nfg, L), st>>>(g, lx, nfg, Hg, rec, rl, L);
    return cudaGetLastError();
}

// ---- batched replicas: shapes and launches of the transform stages ----
int fft_batch_lines(int stage, const Geom &g, int nfg)
{
    return stage == BS_XFWD ? lines_per_block(g.nx) : xinv_lines(g, nfg);
}

void fft_batch_shape(int stage, const BatchRep &r, int *blocks, int *threads, size_t *smem)
{
    const Geom &g = r.g;
    const long long nlines = (long long)g.ny * g.nz;
    *threads = 256;
    switch (stage) {
        case BS_XFWD:
            *blocks = (int)((nlines + r.Lx - 1) / r.Lx) * ((r.nd + 1) / 2);
            *smem = (size_t)(2 * r.Lx * g.nx + g.nx) * sizeof(float2);
            break;
        case BS_YFWD:
        case BS_YINV:
            *blocks = ((g.nxh + kTXy - 1) / kTXy) * g.nz * (stage == BS_YFWD ? r.nd : 3 * r.nfg);
            *smem = (size_t)(2 * g.ny * kTXy + g.ny) * sizeof(float2);
            break;
        case BS_KSPACE:
            *blocks = ((g.nxh + r.txz - 1) / r.txz) * g.ny;
            *smem = kspace_smem(g, r.nd, r.nfg, r.ks_npots, r.txz);
            break;
        default:   // BS_XINV
            *blocks = (int)((nlines + r.Lxi - 1) / r.Lxi);
            *smem = xinv_smem(g, r.nfg, r.Lxi);
            break;
    }
}

cudaError_t launch_fft_batch(int stage, const BatchRep *reps, int R, const BatchLaunch &bl, int deterministic, int txz,
                             cudaStream_t st)
{
    switch (stage) {
        case BS_XFWD:
            if (deterministic) k_xfwd_batch<true><<<bl.blocks, 256, bl.smem, st>>>(reps, bl.pre, R);
            else k_xfwd_batch<false><<<bl.blocks, 256, bl.smem, st>>>(reps, bl.pre, R);
            break;
        case BS_YFWD: k_ypass_batch<false, kTXy><<<bl.blocks, 256, bl.smem, st>>>(reps, bl.pre, R); break;
        case BS_YINV: k_ypass_batch<true, kTXy><<<bl.blocks, 256, bl.smem, st>>>(reps, bl.pre, R); break;
        case BS_KSPACE:
            if (txz == 4) k_kspace_batch<4><<<bl.blocks, 256, bl.smem, st>>>(reps, bl.pre, R);
            else if (txz == 2) k_kspace_batch<2><<<bl.blocks, 256, bl.smem, st>>>(reps, bl.pre, R);
            else return cudaErrorInvalidValue;
            break;
        case BS_XINV: k_xinv_batch<<<bl.blocks, 256, bl.smem, st>>>(reps, bl.pre, R); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_uk_table(const Geom &g, const KSpace *ks_dev, float *tab, cudaStream_t st)
{
    k_uk_table<<<(unsigned)((g.hstride + 255) / 256), 256, 0, st>>>(g, ks_dev, tab);
    return cudaGetLastError();
}

cudaError_t launch_structure_factor(const Geom &g, const FftLine &lx, const FftLine &ly, const FftLine &lz,
                                   const double *twopi_over_L, const float2 *rho_pair, float2 *Hs, int nbins,
                                   double dk, double *bins, cudaStream_t st)
{
    cudaError_t e = launch_xfwd(g, lx, 1, 1, rho_pair, nullptr, Hs, st);
    if (e == cudaSuccess) e = launch_ypass(g, ly, 1, 0, Hs, st);
    if (e != cudaSuccess) return e;
    constexpr int TX = kTXz;
    dim3 grid((g.nxh + TX - 1) / TX, g.ny);
    const size_t sm = (size_t)(2 * g.nz * TX + g.nz) * sizeof(float2);
    const double M = (double)g.M;
    k_sk_z<TX><<<grid, 256, sm, st>>>(g, lz, Hs, twopi_over_L[0], twopi_over_L[1], twopi_over_L[2],
                                      1.0 / (M * M), nbins, 1.0 / dk, bins);
    return cudaGetLastError();
}

}  // namespace tild
