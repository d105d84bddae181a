// tild_grid.cu -- density deposit and reference-exact stencil tables (sm_100a).
#include "tild_stencil.cuh"

#include <type_traits>

#include <algorithm>
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

// Reference-exact stencil table (d_calcGridWeights, ps_grid_utils.cu:74-204): (P+1)^3
// entries per particle, or (P+1)^2 for a 2-D box (nz == 1; index n1*nx + n0, :139).
template <int P>
__global__ void k_grid_weights(Geom g, int quirk4, const float *X, int N, int *inds, float *W)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    float Wx[P + 1], Wy[P + 1], Wz[P + 1];
    const int gx = stencil_axis<P>(X[3 * p], g.dxf[0], quirk4, Wx);
    const int gy = stencil_axis<P>(X[3 * p + 1], g.dxf[1], quirk4, Wy);
    const int gz = stencil_axis_z<P>(X[3 * p + 2], g.dxf[2], quirk4, Wz, g.nz);
    const float gvol = __fmul_rn(__fmul_rn(__fmul_rn(1.0f, g.dxf[0]), g.dxf[1]), g.dxf[2]);
    const bool flat = g.nz == 1;
    const int G = flat ? (P + 1) * (P + 1) : (P + 1) * (P + 1) * (P + 1), ez = flat ? 0 : P;
    int ct = 0;
    for (int a = 0; a <= P; a++) {
        const int n0 = wrapi(gx + a, g.nx);
        for (int b = 0; b <= P; b++) {
            const int n1 = wrapi(gy + b, g.ny);
            for (int e = 0; e <= ez; e++) {
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
    const int gz = stencil_axis_z<P>(X[3 * p + 2], g.dxf[2], quirk4, Wz, g.nz);
    const float gvol = __fmul_rn(__fmul_rn(g.dxf[0], g.dxf[1]), g.dxf[2]);
    const float c = charge ? q[p] : 1.f;
    for (int a = 0; a <= P; a++)
        for (int b = 0; b <= P; b++)
            for (int e = 0; e <= P; e++) {
                const long long m = wrapi(gx + a, g.nx) + (long long)g.nx * (wrapi(gy + b, g.ny) + (long long)g.ny * wrapi(gz + e, g.nz));
                atomicAdd(rho + m, __fdiv_rn(__fmul_rn(__fmul_rn(Wx[a], Wy[b]), Wz[e]), gvol) * c);
            }
}


// Field frames of every group at once (PS_Group::makeDensityField, ps_groups.cu:147-158,
// written by writeDensityFieldBinary, :257-262): each particle computes its stencil once
// and adds the reference weight (/gvol) to the field of every group in its mask.  The
// 'charges' group's frame is its particle density d_rho, not the charge density.
template <int P>
__global__ void k_group_density_frames(Geom g, int quirk4, const float *X0, const float *X1,
                                       const long long *d_step, const int *orig,
                                       const unsigned long long *mask, int N, float *rho)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N) return;
    const unsigned long long bits = mask[orig[s]];
    if (!bits) return;
    const float *X = (*d_step & 1) ? X1 : X0;
    float Wx[P + 1], Wy[P + 1], Wz[P + 1];
    const int gx = stencil_axis<P>(X[3 * s], g.dxf[0], quirk4, Wx);
    const int gy = stencil_axis<P>(X[3 * s + 1], g.dxf[1], quirk4, Wy);
    const int gz = stencil_axis_z<P>(X[3 * s + 2], g.dxf[2], quirk4, Wz, g.nz);
    const float gvol = __fmul_rn(__fmul_rn(g.dxf[0], g.dxf[1]), g.dxf[2]);
    for (int a = 0; a <= P; a++)
        for (int b = 0; b <= P; b++)
            for (int e = 0; e <= P; e++) {
                const long long m = wrapi(gx + a, g.nx) + (long long)g.nx * (wrapi(gy + b, g.ny) + (long long)g.ny * wrapi(gz + e, g.nz));
                const float w = __fdiv_rn(__fmul_rn(__fmul_rn(Wx[a], Wy[b]), Wz[e]), gvol);
                for (unsigned long long r = bits; r; r &= r - 1)
                    atomicAdd(rho + (long long)(__ffsll((long long)r) - 1) * g.M + m, w);
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
constexpr int kDepSmemFast = 96 * 1024;   // a box of 21^3 points x 2 fields (64-brick tiles)
constexpr int kDepSmemFixed = 128 * 1024;

// Coefficient of field f for a particle: membership bit, charge channel -> q.
__device__ __forceinline__ float field_coef(uint32_t dm, unsigned dq, int f, float qp)
{
    return ((dm >> f) & 1u) ? (((dq >> f) & 1u) ? qp : 1.f) : 0.f;
}

// Shared-memory accumulation of one contribution.  Deterministic mode: 64-bit fixed
// point (kFixScale), exact and order-independent.  Fast mode: 32-bit fixed point (integer
// shared atomics, about twice the speed of FP32 ones) in tiles whose particle count keeps
// every sum inside int32 (`ia`), else FP32 atomics.  The scale is 2^24 per unit weight for
// tiles within the count bound int_tile_max (a contribution rounded once to 3e-8, below the
// FP32 rounding of a running sum of order one), 2^23 or 2^22 for tiles of up to two or four
// times as many particles (1.2e-7 at most), so that large deposit tiles stay in integers.
constexpr int kTileFixLog2 = 24;
constexpr int kTileFixSteps = 2;   // the scale may drop to 2^22
template <bool FIXED>
__device__ __forceinline__ void smem_add(float *tf, unsigned long long *tu, int i, float v, bool ia, float tfix)
{
    if (FIXED) atomicAdd(tu + i, (unsigned long long)__double2ll_rn((double)v * kFixScale));
    else if (ia) atomicAdd(reinterpret_cast<int *>(tf) + i, __float2int_rn(v * tfix));
    else atomicAdd(tf + i, v);
}

// The contribution v to every field f with sgn[f] != 0, as sgn[f] * v: one conversion to
// fixed point for all of them (exact: the conversions round to nearest even, so the value
// of -v is minus that of v).
template <bool FIXED, bool IB, int NC>
__device__ __forceinline__ void smem_add_signed(float *tf, unsigned long long *tu, int V, int i, float v,
                                                const int *sgn)
{
    if (FIXED) {
        const long long k = __double2ll_rn((double)v * kFixScale);
#pragma unroll
        for (int f = 0; f < NC; f++)
            if (sgn[f]) atomicAdd(tu + f * V + i, (unsigned long long)(sgn[f] > 0 ? k : -k));
    } else if (IB) {   // v carries the tile's fixed-point scale already (see the caller)
        const int k = __float2int_rn(v);
#pragma unroll
        for (int f = 0; f < NC; f++)
            if (sgn[f]) atomicAdd(reinterpret_cast<int *>(tf) + f * V + i, sgn[f] > 0 ? k : -k);
    } else {
#pragma unroll
        for (int f = 0; f < NC; f++)
            if (sgn[f]) atomicAdd(tf + f * V + i, sgn[f] > 0 ? v : -v);
    }
}

template <bool FIXED>
__device__ __forceinline__ void global_add(float2 *dep, unsigned long long *depfix, long long M, int f, long long m,
                                           float v)
{
    if (FIXED) atomicAdd(depfix + f * M + m, (unsigned long long)__double2ll_rn((double)v * kFixScale));
    else atomicAdd(FIELD_PTR(dep, f, M) + 2 * m, v);
}

// Deposit of one tile of sorted particles (or a window of slots).  The box of grid points
// is accumulated in shared memory, each thread adding its particle's (P+1)^3 points with
// shared-memory atomics (the atomics have throughput to spare; what bounds the deposit
// is instruction issue, so a particle's stencil is computed once, by its own thread, and
// converted to fixed point once per point).  Each touched point is flushed once.
// NF: number of density fields when 1 or 2 (unrolled), 0 = any.
template <int P, int NF, bool FIXED>
__device__ __forceinline__ void deposit_body(const Geom &g, int N, int quirk4, int nd, unsigned dq,
                                             const float *__restrict__ X0, const float *__restrict__ X1,
                                             const long long *__restrict__ d_step,
                                             const uint32_t *__restrict__ pflags,
                                             const float *__restrict__ q, float2 *__restrict__ dep,
                                             unsigned long long *__restrict__ depfix, int cap_bytes,
                                             const TileCfg &tc, int int_tile_max, unsigned bx)
{
    constexpr int P1 = P + 1;
    constexpr int NC = NF ? NF : kMaxFields;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ TileShared ts;
    const float *__restrict__ X = (*d_step & 1) ? X1 : X0;
    int b0, b1;
    tile_range(tc, N, kDepPB, b0, b1, bx);
    if (b1 <= b0) return;
    const int nn[3] = {g.nx, g.ny, g.nz};
    // sorted tiles: the fixed box of the tile's bricks plus the drift margin; particles
    // whose stencil left it deposit with global atomics (windows of unsorted slots: all)
    int lo[3] = {0, 0, 0}, span[3] = {-1, -1, -1}, E[3] = {0, 0, 0};
    if (tc.start) tile_box<P>(tc, nn, lo, span, E, bx);
    const int nfields = NF ? NF : nd;
    const size_t esz = FIXED ? sizeof(unsigned long long) : sizeof(float);
    const long long Vl = (long long)E[0] * E[1] * E[2];
    const bool staged = tc.start && E[0] <= kMaxBoxEdge && E[1] <= kMaxBoxEdge && E[2] <= kMaxBoxEdge &&
                        Vl * nfields * (long long)esz <= cap_bytes;
    const int V = staged ? (int)Vl : 0, E0 = E[0], E01 = E[0] * E[1];
    // int32 fixed-point box: the scale 2^(24 - k) with the least k <= 2 whose count bound
    // int_tile_max 2^k covers the tile (powers of two: exact scalings)
    int ksh = 0;
    while (ksh < kTileFixSteps && (long long)(b1 - b0) > ((long long)int_tile_max << ksh)) ksh++;
    const bool ia = !FIXED && staged && (long long)(b1 - b0) <= ((long long)int_tile_max << ksh);
    const float tfix = __int_as_float((127 + kTileFixLog2 - ksh) << 23);      // 2^(24 - k)
    const float tinv = __int_as_float((127 - kTileFixLog2 + ksh) << 23);      // 2^-(24 - k)
    float *tf = reinterpret_cast<float *>(smraw);
    unsigned long long *tu = reinterpret_cast<unsigned long long *>(smraw);
    if (staged) {
        if (threadIdx.x < 3) {
            ts.ref[threadIdx.x] = lo[threadIdx.x];
            ts.lo[threadIdx.x] = 0;
        }
        __syncthreads();
        tile_tables(ts, g.nx, g.ny, g.nz, E);
        // 16-byte stores (the box and its capacity are multiples of 16 bytes)
        const int n16 = (int)(((long long)V * nfields * (long long)esz + 15) / 16);
        uint4 *z4 = reinterpret_cast<uint4 *>(smraw);
        for (int v = threadIdx.x; v < n16; v += blockDim.x) z4[v] = make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    if (staged) {
        // One particle per thread, all its (P+1)^3 points.  A particle's field coefficients
        // are c0 (its first non-zero one) times s_f in {-1, 0, +1} (a density field and a
        // charge channel of charge +-1, or one field of each block of a copolymer), so one
        // conversion per stencil point serves every field: the fixed-point value of
        // -c0 * w is minus that of c0 * w (round to nearest even is symmetric).  A warp
        // holding a particle with any other coefficients converts per field.
        for (int base = b0 + (threadIdx.x & ~31); base < b1; base += blockDim.x) {
            const int p = base + lane;
            uint32_t dm = p < b1 ? (pflags[p] & 0xffu) : 0u;
            float Wx[P1], Wy[P1], Wz[P1], cf[NC];
            int o = 0;
#pragma unroll
            for (int i = 0; i < P1; i++) Wx[i] = Wy[i] = Wz[i] = 0.f;
#pragma unroll
            for (int f = 0; f < NC; f++) cf[f] = 0.f;
            if (dm) {
                const int gs[3] = {stencil_fast<P>(X[3 * p + 0], g, 0, quirk4, Wx),
                                   stencil_fast<P>(X[3 * p + 1], g, 1, quirk4, Wy),
                                   stencil_fast_z<P>(X[3 * p + 2], g, quirk4, Wz)};
                int d[3];
                bool in = true;
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    d[j] = wrapi(gs[j] - lo[j], nn[j]);
                    in = in && d[j] <= span[j];
                }
                const float qp = q ? q[p] : 0.f;
                if (!in) {   // drifted out of the tile box: straight to global memory
#pragma unroll 1
                    for (int e = 0; e < P1; e++) {
                        const float wz = sel<P>(Wz, e);
                        const long long mz = (long long)g.nx * g.ny * wrapi(gs[2] + e, g.nz);
#pragma unroll 1
                        for (int bb = 0; bb < P1; bb++) {
                            const float wyz = sel<P>(Wy, bb) * wz;
                            const long long my = mz + (long long)g.nx * wrapi(gs[1] + bb, g.ny);
#pragma unroll
                            for (int a = 0; a < P1; a++) {
                                const float w = Wx[a] * wyz;
                                for (int f = 0; f < nfields; f++) {
                                    const float v = field_coef(dm, dq, f, qp) * w;
                                    if (v != 0.f) global_add<FIXED>(dep, depfix, g.M, f, my + wrapi(gs[0] + a, g.nx), v);
                                }
                            }
                        }
                    }
                } else {
                    o = d[2] * E01 + d[1] * E0 + d[0];
#pragma unroll
                    for (int f = 0; f < NC; f++) cf[f] = f < nfields ? field_coef(dm, dq, f, qp) : 0.f;
                }
            }
            float c0 = 0.f;
            int sgn[NC];
            bool general = false;
#pragma unroll
            for (int f = 0; f < NC; f++) {
                if (c0 == 0.f) c0 = cf[f];
                sgn[f] = cf[f] == 0.f ? 0 : (cf[f] == c0 ? 1 : (cf[f] == -c0 ? -1 : 2));
                general = general || sgn[f] == 2;
            }
            // in an int32 box the conversion's scale rides on the coefficient: an exact
            // power-of-two scaling, so c0 2^s w rounds to the same value as (c0 w) 2^s
            const float c0v = (!FIXED && ia) ? c0 * tfix : c0;
            // Wx * (Wy * Wz), then the coefficient: the association of the unstaged path,
            // so that the deterministic mode's fixed-point values do not depend on staging
            auto points = [&](auto int_box, auto gen) {
                constexpr bool IB = decltype(int_box)::value, GN = decltype(gen)::value;
#pragma unroll
                for (int e = 0; e < P1; e++)
#pragma unroll
                    for (int bb = 0; bb < P1; bb++) {
                        const float wyz = Wy[bb] * Wz[e];
                        const int row = o + e * E01 + bb * E0;
#pragma unroll
                        for (int a = 0; a < P1; a++) {
                            const float w = Wx[a] * wyz;
                            if (GN) {
#pragma unroll
                                for (int f = 0; f < NC; f++)
                                    if (cf[f] != 0.f) smem_add<FIXED>(tf, tu, f * V + row + a, cf[f] * w, IB, tfix);
                            } else {
                                smem_add_signed<FIXED, IB, NC>(tf, tu, V, row + a, c0v * w, sgn);
                            }
                        }
                    }
            };
            // the box's number type is fixed for the tile, the conversion per warp
            if (__any_sync(full, general)) {
                if (ia) points(std::true_type{}, std::true_type{});
                else points(std::false_type{}, std::true_type{});
            } else {
                if (ia) points(std::true_type{}, std::false_type{});
                else points(std::false_type{}, std::false_type{});
            }
        }
    } else {
        for (int p = b0 + threadIdx.x; p < b1; p += blockDim.x) {
            const uint32_t dm = pflags[p] & 0xffu;
            if (!dm) continue;
            float Wx[P1], Wy[P1], Wz[P1];
            const int gx = stencil_fast<P>(X[3 * p + 0], g, 0, quirk4, Wx);
            const int gy = stencil_fast<P>(X[3 * p + 1], g, 1, quirk4, Wy);
            const int gz = stencil_fast_z<P>(X[3 * p + 2], g, quirk4, Wz);
            const float qp = q ? q[p] : 0.f;
            int ix[P1], iy[P1], iz[P1];
#pragma unroll
            for (int i = 0; i < P1; i++) {
                ix[i] = wrapi(gx + i, g.nx);
                iy[i] = wrapi(gy + i, g.ny);
                iz[i] = wrapi(gz + i, g.nz);
            }
#pragma unroll 1
            for (int e = 0; e < P1; e++) {
                const float wz = sel<P>(Wz, e);
                const long long mz = (long long)g.nx * g.ny * sel<P>(iz, e);
#pragma unroll
                for (int b = 0; b < P1; b++) {
                    const float wyz = Wy[b] * wz;
                    const long long my = mz + (long long)g.nx * iy[b];
#pragma unroll
                    for (int a = 0; a < P1; a++) {
                        const float w = Wx[a] * wyz;
                        for (int f = 0; f < nd; f++) {
                            const float v = field_coef(dm, dq, f, qp) * w;
                            if (v != 0.f) global_add<FIXED>(dep, depfix, g.M, f, my + ix[a], v);
                        }
                    }
                }
            }
        }
    }
    if (!staged) return;
    __syncthreads();
    const int npair = (nfields + 1) >> 1;
    tile_for_each(ts, E, E[0], E[0] * E[1], [&](int v, int m) {
        if (FIXED) {
            for (int f = 0; f < nfields; f++) {
                const unsigned long long u = tu[f * V + v];
                if (u) atomicAdd(depfix + f * g.M + m, u);
            }
        } else {
            for (int t = 0; t < npair; t++) {
                float a0 = tf[(2 * t) * V + v];
                float a1 = (2 * t + 1 < nfields) ? tf[(2 * t + 1) * V + v] : 0.f;
                if (ia) {
                    a0 = (float)__float_as_int(a0) * tinv;
                    a1 = (float)__float_as_int(a1) * tinv;
                }
                if (a0 != 0.f && a1 != 0.f) atomicAdd(dep + t * g.M + m, make_float2(a0, a1));
                else if (a0 != 0.f) atomicAdd(&dep[t * g.M + m].x, a0);
                else if (a1 != 0.f) atomicAdd(&dep[t * g.M + m].y, a1);
            }
        }
    });
}

template <int P, int NF, bool FIXED>
__global__ void __launch_bounds__(512) k_deposit_tiled(Geom g, int N, int quirk4, int nd, unsigned dq,
                                                       const float *__restrict__ X0, const float *__restrict__ X1,
                                                       const long long *__restrict__ d_step,
                                                       const uint32_t *__restrict__ pflags,
                                                       const float *__restrict__ q, float2 *__restrict__ dep,
                                                       unsigned long long *__restrict__ depfix, int cap_bytes,
                                                       TileCfg tc, int int_tile_max)
{
    deposit_body<P, NF, FIXED>(g, N, quirk4, nd, dq, X0, X1, d_step, pflags, q, dep, depfix, cap_bytes, tc,
                               int_tile_max, blockIdx.x);
}

// the deposit over several replicas (one launch; see BatchRep)
template <int P, int NF, bool FIXED>
__global__ void __launch_bounds__(512) k_deposit_batch(const BatchRep *__restrict__ reps, const int *__restrict__ pre,
                                                       int R)
{
    const int r = batch_replica(pre, R, blockIdx.x);
    const BatchRep &b = reps[r];
    deposit_body<P, NF, FIXED>(b.g, b.N, b.quirk4, b.nd, b.dq, b.X0, b.X1, b.d_step, b.flags, b.q, b.dep, b.depfix,
                               b.dep_cap, b.dtiles, b.int_tile_max, blockIdx.x - pre[r]);
}

// the deposit's box capacity in bytes (the host's estimate for sorted tiles, capped)
static int deposit_cap(const TileCfg &tc, int nf, bool fixed)
{
    int cap = tc.start ? (int)((size_t)tc.pbox * nf * (fixed ? 8 : 4)) : 0;
    cap = std::min(cap, fixed ? kDepSmemFixed : kDepSmemFast);
    return (cap + 15) & ~15;
}

template <int P, int NF>
static void dep_launch_nf(int nb, int threads, const Geom &g, const ParticleParams &pp, const float *X0,
                          const float *X1, const long long *d_step, const uint32_t *pflags, const float *q,
                          float2 *dep, unsigned long long *depfix, const TileCfg &tc, cudaStream_t st)
{
    // box capacity: the host's estimate for sorted tiles (no staging unsorted), capped
    const int cap = deposit_cap(tc, NF ? NF : pp.nd, depfix != nullptr);
    if (depfix)
        k_deposit_tiled<P, NF, true><<<nb, threads, cap, st>>>(g, pp.N, pp.quirk4, pp.nd, pp.dchan_charge, X0,
                                                                       X1, d_step, pflags, q, dep, depfix, cap, tc,
                                                                       pp.int_tile_max);
    else
        k_deposit_tiled<P, NF, false><<<nb, threads, cap, st>>>(g, pp.N, pp.quirk4, pp.nd, pp.dchan_charge, X0,
                                                                        X1, d_step, pflags, q, dep, depfix, cap, tc,
                                                                        pp.int_tile_max);
}

template <int P>
static void dep_launch(const Geom &g, const ParticleParams &pp, const float *X0, const float *X1,
                       const long long *d_step, const uint32_t *pflags, const float *q, float2 *dep,
                       unsigned long long *depfix, const TileCfg &tc, cudaStream_t st)
{
    const int nb = tc.start ? tile_ctas(tc) : (pp.N + kDepPB - 1) / kDepPB;
    const int threads = tc.start ? tc.threads : 256;
    if (pp.nd == 1)
        dep_launch_nf<P, 1>(nb, threads, g, pp, X0, X1, d_step, pflags, q, dep, depfix, tc, st);
    else if (pp.nd == 2)
        dep_launch_nf<P, 2>(nb, threads, g, pp, X0, X1, d_step, pflags, q, dep, depfix, tc, st);
    else
        dep_launch_nf<P, 0>(nb, threads, g, pp, X0, X1, d_step, pflags, q, dep, depfix, tc, st);
}

// zero every replica's deposit target: 8-byte words (float2 pairs, or 64-bit fixed point
// in deterministic mode), 2048 per CTA
__global__ void k_zero_batch(const BatchRep *__restrict__ reps, const int *__restrict__ pre, int R, int fixed)
{
    const int r = batch_replica(pre, R, blockIdx.x);
    const BatchRep &b = reps[r];
    const long long words = (long long)(fixed ? 2 : 1) * ((b.nd + 1) / 2) * b.g.M;
    unsigned long long *p = fixed ? b.depfix : reinterpret_cast<unsigned long long *>(b.dep);
    const long long i0 = (long long)(blockIdx.x - pre[r]) * 2048 + threadIdx.x;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const long long i = i0 + k * 256;
        if (i < words) p[i] = 0ull;
    }
}

void zero_batch_shape(const BatchRep &r, int deterministic, int *blocks)
{
    const long long words = (long long)(deterministic ? 2 : 1) * ((r.nd + 1) / 2) * r.g.M;
    *blocks = (int)((words + 2047) / 2048);
}

cudaError_t launch_zero_batch(const BatchRep *reps, int R, const BatchLaunch &bl, int deterministic, cudaStream_t st)
{
    k_zero_batch<<<bl.blocks, 256, 0, st>>>(reps, bl.pre, R, deterministic);
    return cudaGetLastError();
}

void deposit_batch_shape(const BatchRep &r, int deterministic, int *blocks, int *threads, size_t *smem, int *cap)
{
    *cap = deposit_cap(r.dtiles, r.nd, deterministic != 0);
    *blocks = tile_ctas(r.dtiles);
    *threads = r.dtiles.threads;
    *smem = (size_t)*cap;
}

cudaError_t launch_deposit_batch(const BatchRep *reps, int R, const BatchLaunch &bl, int order, int nd,
                                 int deterministic, cudaStream_t st)
{
#define TILD_DB(P, NF)                                                                                      \
    do {                                                                                                    \
        if (deterministic) k_deposit_batch<P, NF, true><<<bl.blocks, bl.threads, bl.smem, st>>>(reps, bl.pre, R); \
        else k_deposit_batch<P, NF, false><<<bl.blocks, bl.threads, bl.smem, st>>>(reps, bl.pre, R);         \
    } while (0)
#define TILD_DBP(P) do { if (nd == 1) TILD_DB(P, 1); else TILD_DB(P, 2); } while (0)
    switch (order) {
        case 0: TILD_DBP(0); break;
        case 1: TILD_DBP(1); break;
        case 2: TILD_DBP(2); break;
        case 3: TILD_DBP(3); break;
        default: TILD_DBP(4); break;
    }
#undef TILD_DBP
#undef TILD_DB
    return cudaGetLastError();
}

void init_deposit_attributes()
{
#define TILD_DA1(P, NF)                                                                                        \
    cudaFuncSetAttribute(k_deposit_tiled<P, NF, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDepSmemFixed); \
    cudaFuncSetAttribute(k_deposit_tiled<P, NF, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDepSmemFast); \
    cudaFuncSetAttribute(k_deposit_batch<P, NF, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDepSmemFixed);  \
    cudaFuncSetAttribute(k_deposit_batch<P, NF, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDepSmemFast)
#define TILD_DA(P) TILD_DA1(P, 0); TILD_DA1(P, 1); TILD_DA1(P, 2)
    TILD_DA(0);
    TILD_DA(1);
    TILD_DA(2);
    TILD_DA(3);
    TILD_DA(4);
#undef TILD_DA
#undef TILD_DA1
}

cudaError_t launch_deposit(const Geom &g, const ParticleParams &pp, const float *X0, const float *X1,
                           const long long *d_step, const uint32_t *pflags, const float *q, float2 *dep,
                           unsigned long long *dep_fixed, int deterministic, const TileCfg &tc, cudaStream_t st)
{
    if (pp.N == 0) return cudaSuccess;
    unsigned long long *df = deterministic ? dep_fixed : nullptr;
#define TILD_DL(P) dep_launch<P>(g, pp, X0, X1, d_step, pflags, q, dep, df, tc, st)
    switch (pp.order) {
        case 0: TILD_DL(0); break;
        case 1: TILD_DL(1); break;
        case 2: TILD_DL(2); break;
        case 3: TILD_DL(3); break;
        default: TILD_DL(4); break;
    }
#undef TILD_DL
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

__global__ void k_to_pairs(const float *__restrict__ rho, float2 *__restrict__ out, long long M)
{
    const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m < M) out[m] = make_float2(rho[m], 0.f);
}

cudaError_t launch_group_density_frames(const Geom &g, const ParticleParams &pp, const float *X0, const float *X1,
                                        const long long *d_step, const int *orig,
                                        const unsigned long long *mask, int N, float *rho, cudaStream_t st)
{
    if (N == 0) return cudaSuccess;
    const int nbk = (N + 255) / 256;
    switch (pp.order) {
        case 0: k_group_density_frames<0><<<nbk, 256, 0, st>>>(g, pp.quirk4, X0, X1, d_step, orig, mask, N, rho); break;
        case 1: k_group_density_frames<1><<<nbk, 256, 0, st>>>(g, pp.quirk4, X0, X1, d_step, orig, mask, N, rho); break;
        case 2: k_group_density_frames<2><<<nbk, 256, 0, st>>>(g, pp.quirk4, X0, X1, d_step, orig, mask, N, rho); break;
        case 3: k_group_density_frames<3><<<nbk, 256, 0, st>>>(g, pp.quirk4, X0, X1, d_step, orig, mask, N, rho); break;
        default: k_group_density_frames<4><<<nbk, 256, 0, st>>>(g, pp.quirk4, X0, X1, d_step, orig, mask, N, rho); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_to_pairs(const float *rho, float2 *out, long long M, cudaStream_t st)
{
    k_to_pairs<<<(unsigned)((M + 255) / 256), 256, 0, st>>>(rho, out, M);
    return cudaGetLastError();
}

}  // namespace tild
