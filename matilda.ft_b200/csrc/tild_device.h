// tild_device.h -- device-side data layout and kernel launchers of the TILD step.
//
// Layout in HBM (one box):
//   X[2][N*3]      float   positions, ping-pong: x_t in X[t&1], x_{t-1} in X[(t+1)&1]
//   noise[N*3]     float   GJF previous noise
//   pflags[N]      uint32  bits 0-7 density-field membership, 8-15 force-group
//                          membership, 16-19 integrator slot (15 = none), 20-23 type
//   q[N]           float   charges (only with doCharges)
//   brow[N+1], partner[nnz], btype[nnz]     bonds in CSR, both directions (readDataConfig);
//                          particle p's partners are partner[brow[p] .. brow[p+1])
//   dep[npair][M]  float2  deposit target: field 2i in .x, 2i+1 in .y
//   H[D][Nz][Ny][hp]  float2  density half spectra (kx in [0, Nx/2])
//   Hg[3F][Nz][Ny][hp] float2 gradient half spectra
//   rec[F][M]      float4  grid force of each force group (x, y, z, 0) ("planar"), or for
//                          one or two force groups the "paired" planes of RecLayout
//   fgrid[N*3]     float   grid force of each particle (sum over its force groups)
#pragma once
#include <cstdint>
#include <cuda.h>            // CUtensorMap (a host-built TMA descriptor; no driver library linked)
#include <cuda_runtime.h>

namespace tild {

constexpr int kMaxFields = 8;     // density fields D
constexpr int kMaxFGroups = 4;    // force groups F (3F gradient fields)
constexpr int kMaxPots = 16;
constexpr int kMaxTerms = 32;
// FP64 results of the energy reductions: pair energy of each potential at [0, npots),
// the summed pair virial W_ab (xx, yy, zz, xy, xz, yz) right after them, the bond energy
// and bond virial at kResBond
constexpr int kResBond = kMaxPots + 6;
constexpr int kResAngle = kResBond + 7;   // angle energy and virial (each angle on 3 particles)
constexpr int kMaxWalls = 4;              // `potential wall` terms (per-particle, flag bits 24..27)
constexpr int kResWall = kResAngle + 7;   // energy of each wall
constexpr int kResNonFinite = kResWall + kMaxWalls;   // particles whose position is not finite
constexpr int kResSize = kResNonFinite + 1;
constexpr int kPartialCols = 15 + kMaxWalls;   // per-block columns of the bond/angle/wall reduction
constexpr int kMaxTypes = 16;
constexpr int kMaxBondTypes = 16;
constexpr int kMaxAngleTypes = 16;
constexpr int kMaxStages = 20;
constexpr int kNoIntegrator = 15;
constexpr double kFixScale = 4294967296.0;  // deterministic deposit: 2^32 per unit weight

enum PotKind { POT_GAUSSIAN = 0, POT_ERF2 = 1, POT_ERFG = 2, POT_CHARGES = 3, POT_WALL = 4 };

// Division by a runtime constant d through a multiply: exact for i * d < 2^32.
struct FastDiv {
    unsigned d, m;        // m = ceil(2^32 / d); d == 1 handled separately
};
inline FastDiv make_fastdiv(unsigned d)
{
    FastDiv f;
    f.d = d;
    f.m = d <= 1 ? 0u : (unsigned)((0x100000000ull + d - 1) / d);
    return f;
}

struct FftLine {          // Stockham mixed-radix plan of one line length
    int n;
    int ns;
    int R[kMaxStages];
    int P[kMaxStages];
    FastDiv dP[kMaxStages];   // division by P[s]
    FastDiv dNB[kMaxStages];  // division by n / R[s]
    const float2 *tw;     // device twiddles W_n^t, t in [0, n)  (forward sign)
};

struct Geom {
    int nx, ny, nz, nxh, hp;   // grid, half-spectrum width nx/2+1, row pitch (complex)
    long long M;               // nx*ny*nz
    long long hstride;         // elements per half-spectrum field = nz*ny*hp
    float dxf[3];              // (float)(L/Nx)
    float dlo[3];              // (float)(L/Nx - dxf): the FP32 remainder of the cell width
    float inv[3];              // 1.f / dxf (IEEE FP32 division)
    float L[3];
    float Lh[3];
};

struct PotDev {
    int kind;
    double amp;    // effective amplitude (after any ramp update)
    double sig2;   // sigma^2
    double Rp;
    double lB;
};

struct KTerm {      // phi_f += mult * u_pot(k) * rhohat_d(k)
    int fgroup;
    int pot;
    int dfield;
    double mult;
};

struct ETerm {      // U_pot = fac * sum_k u_pot(k) Re(rhohat_J conj rhohat_I)
    int pot;
    int dI, dJ;
    double fac;
};

struct KSpace {
    int npots;
    PotDev pots[kMaxPots];
    int nterms;
    KTerm terms[kMaxTerms];
    int nfg;              // force groups receiving k-space terms
    int nd;               // density fields
    int neterms;
    ETerm eterms[kMaxPots];
    double twopi_over_L[3];
};

struct TypeCoef {   // per-type integrator constants (ps_integratorGJF.cu:63-76)
    float a, b, noiseMag, bdt2m, bdt2m2;
};

struct ParticleParams {
    int N;
    int order;
    int quirk4;
    int nd;                         // density fields
    int npair;
    unsigned dchan_charge;          // bit i set: field i is a charge-weighted channel
    int int_tile_max;               // deposit: tiles of at most this many particles sum in int32 fixed point
    int nfg;
    unsigned fg_qweighted;          // bit f set: force group f gathers q-weighted
    int maxb;
    int nbtypes;
    float bk[kMaxBondTypes], breq[kMaxBondTypes];
    int bstyle[kMaxBondTypes];
    int maxa;                       // angle slots per particle (0: no angles)
    float ak[kMaxAngleTypes], atheq[kMaxAngleTypes];
    int astyle[kMaxAngleTypes];     // 0 wlc, 1 harmonic
    int integ_kind[4];              // 0 GJF, 1 EM per integrator slot
    float em_delt[4], em_noise[4];
    TypeCoef coef[4][kMaxTypes];
    unsigned long long seed;
    int rng_compat;
    int dim;                        // 2: z is one plane at z = 0 (no z noise), 3: full 3-D
    // harmonic walls (ps_potentialWall.cu): on particles with flag bit 24 + w, a force
    // k (pos - x_axis) along the axis while sign (pos - x_axis) > 0
    int nwall;
    int wall_axis[kMaxWalls], wall_sign[kMaxWalls];
    float wall_pos[kMaxWalls], wall_k[kMaxWalls];
};

// Work split of the particle kernels over a sorted particle order: a CTA of `threads`
// threads takes the slots of `codes` consecutive brick codes; boxes of up to `box`
// grid points are staged in shared memory.  start == nullptr: fixed windows of slots.
struct TileCfg {
    const uint32_t *start;
    const uint32_t *list;   // the tiles that meet the grid (CTA b takes tile list[b]); NULL: every tile
    int nlist;
    int nkeys;
    int codes;
    int threads;
    int box;      // deposit: shared-memory records of a tile's bounding box (estimate)
    int pbox;     // particle pass: records of the fixed tile box (odd pitches)
    int margin;   // particle pass: drift margin of the fixed box, cells per side
    int direct;   // particle pass: 1 = read every stencil through L1/L2 (no staged box)
    int te[3];    // particle pass: edges of the TMA box of force records (0: stage with cp.async)
    int paired;   // particle pass: 1 = the tile gather over the paired records (RecLayout)
};

// Force records in the "paired" layout of the tile gather (one or two force groups, 3-D
// boxes): plane A holds float4 (g0.x, g0.y, g1.x, g1.y) -- (x, y, z, 0) for one group --
// and plane B float2 (g0.z, g1.z), both over a padded grid of px x py x pz points that
// carries `gl` periodic ghost layers below and gh[] above every axis, so that no tile's
// box wraps: grid point (x, y, z) sits at ((z + gl) * py + (y + gl)) * px + x + gl, and a
// ghost holds the value of the point it wraps to.
struct RecLayout {
    int paired;
    int nfg;
    int gl;
    int gh[3];
    int px, py, pz;
    long long pM;         // px * py * pz
    float4 *A;
    float2 *B;            // nfg == 2 only
};
// layout for tiles whose boxes reach gl points below and gh[] above the grid
RecLayout make_rec_layout(const Geom &g, int nfg, int gl, const int *gh, void *base);
size_t rec_layout_bytes(const Geom &g, int nfg, int gl, const int *gh);

// TMA descriptors of the paired planes for boxes of te[] points (te[0] even): false where
// they cannot be built (the planar path is used then).
bool build_paired_maps(CUtensorMap *mapA, CUtensorMap *mapB, const RecLayout &rl, const int *te);

// TMA descriptor of the force records rec[F][nz][ny][nx] (float4) for boxes of te[] points:
// false where it cannot be built (the particle pass then stages with cp.async).
bool build_record_map(CUtensorMap *map, const float4 *rec, const Geom &g, int nfg, const int *te);

struct AngleArrays {        // angles in slot order (all NULL: the box has none)
    const uint8_t *na, *atype;  // [n] angles per particle, [n*maxa] types
    const int *ang;             // [n*maxa*3] slots of the angle's i, j (middle), k
};

// -------------------------------------------------------------------------------------
// Batched replicas: one launch per step stage over the work of several boxes.  Each box's
// step state is one entry of a device table; CTA b of a stage belongs to the replica r
// with pre[r] <= b < pre[r + 1] and works on that replica's block b - pre[r].
// -------------------------------------------------------------------------------------
struct BatchRep {
    CUtensorMap mapA, mapB;     // TMA descriptors of the paired record planes (64-byte aligned)
    Geom g;
    FftLine lx, ly, lz;
    TileCfg tiles, dtiles;      // particle-pass and deposit tiles (start and list set)
    RecLayout rl;
    AngleArrays aa;
    const ParticleParams *ppd;
    const KSpace *ks;
    const float *uk;
    int N, quirk4, nd, nfg, int_tile_max, dep_cap, Lx, Lxi, txz, ks_npots;
    unsigned dq;
    float *X0, *X1, *noise;
    const uint32_t *flags;
    const float *q;
    const int *brow, *partner;
    const uint8_t *btype;
    const int *orig;
    void *rng;
    float2 *dep;
    unsigned long long *depfix;
    float2 *H, *Hg;
    float4 *rec;
    float *fgrid;
    long long *d_step;
    int *err;
};

enum BatchStage { BS_DEPOSIT, BS_XFWD, BS_YFWD, BS_KSPACE, BS_YINV, BS_XINV, BS_GATHER, BS_INTEGRATE, BS_COUNT };

struct BatchLaunch {        // one stage's launch over all replicas
    const int *pre;         // device: exclusive prefix of the replicas' CTA counts, R + 1 entries
    int blocks, threads;
    size_t smem;
};

cudaError_t launch_batch_tick(const BatchRep *reps, int R, cudaStream_t st);
// per-file pieces of the above (tild_grid.cu, tild_fft.cu, tild_particles.cu)
void zero_batch_shape(const BatchRep &r, int deterministic, int *blocks);
cudaError_t launch_zero_batch(const BatchRep *reps, int R, const BatchLaunch &bl, int deterministic, cudaStream_t st);
void deposit_batch_shape(const BatchRep &r, int deterministic, int *blocks, int *threads, size_t *smem, int *cap);
cudaError_t launch_deposit_batch(const BatchRep *reps, int R, const BatchLaunch &bl, int order, int nd,
                                 int deterministic, cudaStream_t st);
int fft_batch_lines(int stage, const Geom &g, int nfg);   // lines per block of the x passes
void fft_batch_shape(int stage, const BatchRep &r, int *blocks, int *threads, size_t *smem);
cudaError_t launch_fft_batch(int stage, const BatchRep *reps, int R, const BatchLaunch &bl, int deterministic, int txz,
                             cudaStream_t st);
void particles_batch_shape(int stage, const BatchRep &r, int *blocks, int *threads, size_t *smem);
cudaError_t launch_particles_batch(int stage, const BatchRep *reps, int R, const BatchLaunch &bl, int order, int nfg,
                                   int extra, cudaStream_t st);

// -------------------------------------------------------------------------------------
// Launchers (tild_grid.cu, tild_fft.cu, tild_particles.cu, tild_sort.cu).  All run on `st`;
// none synchronises.
void build_fft_line(int n, FftLine &pl, float2 *dev_tw_dst);
void init_fft_attributes();      // opt the FFT kernels into large dynamic shared memory
void init_deposit_attributes();  // same for the staged deposit
cudaError_t launch_zero(void *p, size_t bytes, cudaStream_t st);
cudaError_t launch_deposit(const Geom &g, const ParticleParams &pp, const float *X0,
                           const float *X1, const long long *d_step, const uint32_t *pflags,
                           const float *q, float2 *dep, unsigned long long *dep_fixed,
                           int deterministic, const TileCfg &tc, cudaStream_t st);
cudaError_t launch_xfwd(const Geom &g, const FftLine &lx, int npair, int nd, const float2 *dep,
                        const unsigned long long *dep_fixed, float2 *H, cudaStream_t st);
cudaError_t launch_ypass(const Geom &g, const FftLine &ly, int nfields, int inverse, float2 *H,
                         cudaStream_t st);
cudaError_t launch_kspace_z(const Geom &g, const FftLine &lz, const KSpace &ks, const KSpace *ks_dev,
                            const float2 *H, const float *uk, float2 *Hg, double *epart, int energy, int forces,
                            int *nblocks_out, cudaStream_t st);
// half-spectrum columns per block of the k-space z pass (4, or 2 so that its shared
// memory fits), 0 if even 2 do not fit
int kspace_tile_width(const Geom &g, int nd, int nfg, int npots);
// FP32 table of every potential's û(k) shape (amplitude 1) over the half spectrum
cudaError_t launch_uk_table(const Geom &g, const KSpace *ks_dev, float *tab, cudaStream_t st);
// S(|k|) of one real field given as float2 pairs (field in .x): x/y forward passes into
// Hs, then the z pass bins |FFT(rho)/M|^2 into bins[3*nbins] (S, |k|, count; FP64)
// out[m] = (rho[m], 0)
cudaError_t launch_to_pairs(const float *rho, float2 *out, long long M, cudaStream_t st);
cudaError_t launch_structure_factor(const Geom &g, const FftLine &lx, const FftLine &ly, const FftLine &lz,
                                   const double *twopi_over_L, const float2 *rho_pair, float2 *Hs, int nbins,
                                   double dk, double *bins, cudaStream_t st);
// x inverse pass: the records of every force group, planar into rec, or into the paired
// planes of rl when rl.paired
cudaError_t launch_xinv(const Geom &g, const FftLine &lx, int nfg, const float2 *Hg, float4 *rec,
                        const RecLayout &rl, cudaStream_t st);
// The particle pass as two kernels.  launch_gather: the grid gather of every particle's
// force groups into fgrid[3N] (the tile gather over the paired records when rl.paired,
// else the planar gather over rec[F][M]).  launch_integrate: bonds, angles and walls plus
// fgrid, fout[3N] on request, and the GJF/EM update, one thread per particle (which also
// gathers, from the paired records, the particles the tile gather left to it).
cudaError_t launch_gather(const Geom &g, const ParticleParams &pp, const ParticleParams *ppd, const float *X0,
                          const float *X1, const uint32_t *pflags, const float *q, const float4 *rec,
                          const RecLayout &rl, const long long *d_step, float *fgrid, const TileCfg &tc,
                          const CUtensorMap *rec_map, const CUtensorMap *pmapA, const CUtensorMap *pmapB, int *err,
                          cudaStream_t st);
cudaError_t launch_integrate(const Geom &g, const ParticleParams &pp, const ParticleParams *ppd, float *X0, float *X1,
                             float *noise, const uint32_t *pflags, const float *q, const int *brow, const int *partner,
                             const uint8_t *btype, AngleArrays aa, const float *fgrid, const RecLayout &rl,
                             const int *orig_id, void *rng_states, const long long *d_step, float *fout, int integrate,
                             cudaStream_t st);
// whether the paired tile gather can stage a box of te[] points for nfg force groups
bool paired_box_fits(const int *te, int nfg);
void init_particle_attributes();
cudaError_t launch_tick(long long *d_step, cudaStream_t st);

// ---- spatial re-sort (tild_sort.cu) ----
struct PermIn {             // current particle arrays (slot order)
    const float *X0, *X1, *noise, *q;
    const uint32_t *flags;
    const int *orig;
    const int *brow, *partner;  // bonds in CSR: row p = [brow[p], brow[p+1]) of partner/btype
    const uint8_t *btype;       // (NULL brow: no bonds)
    const void *rng;
    const long long *d_step;
    const uint8_t *na, *atype;  // angles per particle and their types (may be NULL)
    const int *ang;             // [n*maxa*3] particle slots of each angle
};
struct SortScratch {        // work arrays and the permuted copies
    uint32_t *key, *count, *totals, *start;
    uint32_t *totalsN;          // per-block totals of the scan of the N bond counts
    int *rank, *newpos;
    float *X0, *X1, *noise, *q;
    uint32_t *flags;
    int *orig;
    int *brow, *partner;
    uint8_t *btype;
    void *rng;
    uint8_t *na, *atype;
    int *ang;
};
uint32_t sort_key_count(const Geom &g);
cudaError_t launch_sort(const Geom &g, int N, int maxa, const SortScratch &w, const PermIn &in, cudaStream_t st);
cudaError_t launch_unpermute_rows(int N, int width, const int *orig, const float *in, float *out,
                                  cudaStream_t st);
cudaError_t launch_permute_rows(int N, int width, const int *orig, const float *in, float *out,
                                cudaStream_t st);
cudaError_t launch_rng_init(void *states, const int *orig_id, int n, unsigned long long seed,
                            cudaStream_t st);
size_t rng_state_bytes();
// per block (kPartialCols columns): bond energy + virial (7), angle energy + virial (7),
// the energy of each wall (kMaxWalls), then the count of particles whose position is not
// finite
cudaError_t launch_bond_energy(const Geom &g, const ParticleParams &pp, const ParticleParams *ppd,
                               const float *X0, const float *X1, const long long *d_step,
                               const int *brow, const int *partner, const uint8_t *btype, AngleArrays aa,
                               const uint32_t *pflags, double *partials, int *nblocks_out, cudaStream_t st);
cudaError_t launch_reduce_partials(const double *partials, int nblocks, int ncols, double *out,
                                   cudaStream_t st);
cudaError_t launch_grid_weights(const Geom &g, int order, int quirk4, const float *X, int N,
                                int *inds, float *W, cudaStream_t st);
cudaError_t launch_density_single(const Geom &g, const ParticleParams &pp, const float *X,
                                  const int *sites, int ns, const float *q, int charge,
                                  float *rho, cudaStream_t st);
// Output snapshots, read from the current buffer of the (X0, X1) pair chosen by *d_step:
// field frames rho[g*M + m] of every group g whose bit is set in mask[original id]
// (group densities with the reference's weights), and positions in original order.
constexpr int kMaxFrameGroups = 64;
cudaError_t launch_group_density_frames(const Geom &g, const ParticleParams &pp, const float *X0, const float *X1,
                                        const long long *d_step, const int *orig,
                                        const unsigned long long *mask, int N, float *rho, cudaStream_t st);
cudaError_t launch_snapshot_positions(int N, const int *orig, const float *X0, const float *X1,
                                      const long long *d_step, float *out, cudaStream_t st);

// Static device scratch of the allocation-free density read-back (tild_noalloc.cu):
// kStaticScratchBytes in one file-scope __device__ array, address looked up once per device.
constexpr size_t kStaticScratchBytes = size_t(16) << 20;
cudaError_t static_scratch(int device, void **ptr);
// slot_of[orig[s]] = s for s < n, then sites[k] = slot_of[sites[k]] for k < ns
cudaError_t launch_slot_map(const int *orig, int n, int *slot_of, int *sites, int ns, cudaStream_t st);

}  // namespace tild
