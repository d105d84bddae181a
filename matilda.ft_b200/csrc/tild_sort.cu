// tild_sort.cu -- periodic spatial re-sort of the particle arrays (sm_100a).
//
// Particles are ordered by the Morton code of their 4x4x4-cell brick so that the
// particles of one CTA (and one warp) touch a compact block of grid points: the deposit
// stages that block in shared memory and the gathers hit L1.  The reference keeps
// particles in input order (PS_Box_initialization.cu:862-884); order changes nothing in
// the physics: every per-particle array moves together, bond partners are renumbered,
// and the original id travels along for the Philox counter and the C ABI.
//
// Counting sort: brick key per particle with an atomic rank inside its bin, exclusive
// scan of the bin counts, new slot = start[key] + rank, one permute kernel.
#include "tild_stencil.cuh"

#include <curand_kernel.h>

namespace tild {

__device__ __forceinline__ uint32_t spread3(uint32_t v)   // 10-bit -> every third bit
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ int cell_of(float x, float d, int n)
{
    int c = (int)floorf(x / d);
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

__global__ void k_sort_keys(Geom g, int N, const float *__restrict__ X0, const float *__restrict__ X1,
                            const long long *__restrict__ d_step, uint32_t *__restrict__ key,
                            int *__restrict__ rank, uint32_t *__restrict__ count)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const float *X = (*d_step & 1) ? X1 : X0;
    const uint32_t bx = cell_of(X[3 * p], g.dxf[0], g.nx) >> 2;
    const uint32_t by = cell_of(X[3 * p + 1], g.dxf[1], g.ny) >> 2;
    const uint32_t bz = cell_of(X[3 * p + 2], g.dxf[2], g.nz) >> 2;
    const uint32_t k = spread3(bx) | (spread3(by) << 1) | (spread3(bz) << 2);
    key[p] = k;
    rank[p] = (int)atomicAdd(count + k, 1u);
}

// Exclusive scan in three kernels: per-block totals, scan of the totals, local scan + add.
constexpr int kScanBlock = 1024;

__global__ void k_scan_totals(const uint32_t *__restrict__ in, int n, uint32_t *__restrict__ totals)
{
    __shared__ uint32_t red[32];
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    uint32_t v = i < n ? in[i] : 0u;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t w = red[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) totals[blockIdx.x] = w;
    }
}

__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *total)
{
    __shared__ uint32_t ws[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        ws[lane] = s;
    }
    __syncthreads();
    const uint32_t before = warp ? ws[warp - 1] : 0u;
    if (total) *total = ws[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}

// Single block: exclusive scan of nb totals (loops over chunks of kScanBlock).
__global__ void k_scan_partials(uint32_t *__restrict__ totals, int nb)
{
    uint32_t carry = 0;
    for (int base = 0; base < nb; base += kScanBlock) {
        const int i = base + threadIdx.x;
        const uint32_t v = i < nb ? totals[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(v, &tot);
        if (i < nb) totals[i] = carry + ex;
        carry += tot;
        __syncthreads();
    }
}

__global__ void k_scan_apply(const uint32_t *__restrict__ in, int n, const uint32_t *__restrict__ offsets,
                             uint32_t *__restrict__ out)
{
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    const uint32_t v = i < n ? in[i] : 0u;
    const uint32_t ex = block_exclusive_scan(v, nullptr);
    if (i < n) out[i] = offsets[blockIdx.x] + ex;
}

__global__ void k_newpos(int N, const uint32_t *__restrict__ key, const int *__restrict__ rank,
                         const uint32_t *__restrict__ start, int *__restrict__ newpos)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    newpos[p] = (int)start[key[p]] + rank[p];
}

struct PermArrays {
    const float *X0, *X1, *noise, *q;
    const uint32_t *flags;
    const int *orig, *brow;
    const curandState *rng;
    const uint8_t *na, *atype;
    const int *ang;
    float *X0n, *X1n, *noisen, *qn;
    uint32_t *flagsn;
    int *orign;
    uint32_t *degn;   // bond count of every new slot (the CSR rows' lengths in the new order)
    curandState *rngn;
    uint8_t *nan, *atypen;
    int *angn;
};

__global__ void k_permute(int N, int maxa, PermArrays a, const int *__restrict__ newpos)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const int s = newpos[p];
#pragma unroll
    for (int j = 0; j < 3; j++) {
        a.X0n[3 * s + j] = a.X0[3 * p + j];
        a.X1n[3 * s + j] = a.X1[3 * p + j];
        a.noisen[3 * s + j] = a.noise[3 * p + j];
    }
    a.flagsn[s] = a.flags[p];
    a.orign[s] = a.orig[p];
    if (a.q) a.qn[s] = a.q[p];
    if (a.brow) a.degn[s] = (uint32_t)(a.brow[p + 1] - a.brow[p]);
    if (a.rng) a.rngn[s] = a.rng[p];
    if (a.na) {   // angles: all three particle slots renumbered
        const int nap = a.na[p];
        a.nan[s] = (uint8_t)nap;
        for (int k = 0; k < maxa; k++) {
            for (int r = 0; r < 3; r++)
                a.angn[(s * maxa + k) * 3 + r] = k < nap ? newpos[a.ang[(p * maxa + k) * 3 + r]] : 0;
            a.atypen[s * maxa + k] = a.atype[p * maxa + k];
        }
    }
}

// CSR bond rows in the new slot order: row p moves to the new row of slot newpos[p]
// (offsets from the scan of the new order's bond counts), its partners renumbered.
__global__ void k_permute_bonds(int N, const int *__restrict__ brow, const int *__restrict__ partner,
                                const uint8_t *__restrict__ btype, const int *__restrict__ newpos,
                                const int *__restrict__ brown, int *__restrict__ partnern, uint8_t *__restrict__ btypen)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= N) return;
    const int k0 = brow[p], k1 = brow[p + 1], d = brown[newpos[p]];
    for (int k = k0; k < k1; k++) {
        partnern[d + k - k0] = newpos[partner[k]];
        btypen[d + k - k0] = btype[k];
    }
}

// out[orig[s]] = in[s] for rows of `width` floats (slot order -> original order)
__global__ void k_unpermute_rows(int N, int width, const int *__restrict__ orig, const float *__restrict__ in,
                                 float *__restrict__ out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)N * width) return;
    const int s = (int)(i / width), c = (int)(i - (long long)s * width);
    out[(long long)orig[s] * width + c] = in[i];
}

// out[s] = in[orig[s]] (original order -> slot order), rows of `width` floats
__global__ void k_permute_rows(int N, int width, const int *__restrict__ orig, const float *__restrict__ in,
                               float *__restrict__ out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)N * width) return;
    const int s = (int)(i / width), c = (int)(i - (long long)s * width);
    out[i] = in[(long long)orig[s] * width + c];
}

uint32_t sort_key_count(const Geom &g)
{
    const int b = std::max(std::max((g.nx + 3) / 4, (g.ny + 3) / 4), (g.nz + 3) / 4);
    int bits = 0;
    while ((1 << bits) < b) bits++;
    return 1u << (3 * bits);
}

cudaError_t launch_sort(const Geom &g, int N, int maxa, const SortScratch &w, const PermIn &in, cudaStream_t st)
{
    if (N == 0) return cudaSuccess;
    const uint32_t nk = sort_key_count(g);
    const int nbk = (N + 255) / 256;
    cudaMemsetAsync(w.count, 0, sizeof(uint32_t) * nk, st);
    k_sort_keys<<<nbk, 256, 0, st>>>(g, N, in.X0, in.X1, in.d_step, w.key, w.rank, w.count);
    const int nsb = (int)((nk + kScanBlock - 1) / kScanBlock);
    k_scan_totals<<<nsb, kScanBlock, 0, st>>>(w.count, (int)nk, w.totals);
    k_scan_partials<<<1, kScanBlock, 0, st>>>(w.totals, nsb);
    k_scan_apply<<<nsb, kScanBlock, 0, st>>>(w.count, (int)nk, w.totals, w.start);
    k_newpos<<<nbk, 256, 0, st>>>(N, w.key, w.rank, w.start, w.newpos);
    PermArrays a;
    a.X0 = in.X0; a.X1 = in.X1; a.noise = in.noise; a.q = in.q; a.flags = in.flags; a.orig = in.orig;
    a.brow = in.brow;
    a.rng = reinterpret_cast<const curandState *>(in.rng);
    a.X0n = w.X0; a.X1n = w.X1; a.noisen = w.noise; a.qn = w.q; a.flagsn = w.flags; a.orign = w.orig;
    // the ranks are spent once the new slots exist: their array takes the new bond counts
    a.degn = reinterpret_cast<uint32_t *>(w.rank);
    a.rngn = reinterpret_cast<curandState *>(w.rng);
    a.na = in.na;
    a.atype = in.atype;
    a.ang = in.ang;
    a.nan = w.na;
    a.atypen = w.atype;
    a.angn = w.ang;
    k_permute<<<nbk, 256, 0, st>>>(N, maxa, a, w.newpos);
    if (in.brow) {   // new CSR rows: exclusive scan of the counts (brow[N] never changes), then the rows
        const int nsn = (N + kScanBlock - 1) / kScanBlock;
        k_scan_totals<<<nsn, kScanBlock, 0, st>>>(a.degn, N, w.totalsN);
        k_scan_partials<<<1, kScanBlock, 0, st>>>(w.totalsN, nsn);
        k_scan_apply<<<nsn, kScanBlock, 0, st>>>(a.degn, N, w.totalsN, reinterpret_cast<uint32_t *>(w.brow));
        k_permute_bonds<<<nbk, 256, 0, st>>>(N, in.brow, in.partner, in.btype, w.newpos, w.brow, w.partner, w.btype);
    }
    return cudaGetLastError();
}

cudaError_t launch_unpermute_rows(int N, int width, const int *orig, const float *in, float *out, cudaStream_t st)
{
    const long long n = (long long)N * width;
    if (n == 0) return cudaSuccess;
    k_unpermute_rows<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(N, width, orig, in, out);
    return cudaGetLastError();
}

// positions of the current buffer (chosen by the step parity) in original order
__global__ void k_snapshot_positions(int N, const int *__restrict__ orig, const float *__restrict__ X0,
                                     const float *__restrict__ X1, const long long *__restrict__ d_step,
                                     float *__restrict__ out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3LL * N) return;
    const float *X = (*d_step & 1) ? X1 : X0;
    const int s = (int)(i / 3), c = (int)(i - 3LL * s);
    out[3LL * orig[s] + c] = X[i];
}

cudaError_t launch_snapshot_positions(int N, const int *orig, const float *X0, const float *X1,
                                      const long long *d_step, float *out, cudaStream_t st)
{
    const long long n = 3LL * N;
    if (n == 0) return cudaSuccess;
    k_snapshot_positions<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(N, orig, X0, X1, d_step, out);
    return cudaGetLastError();
}

cudaError_t launch_permute_rows(int N, int width, const int *orig, const float *in, float *out, cudaStream_t st)
{
    const long long n = (long long)N * width;
    if (n == 0) return cudaSuccess;
    k_permute_rows<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(N, width, orig, in, out);
    return cudaGetLastError();
}

}  // namespace tild
