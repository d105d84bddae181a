/*
 * tild_b200.h -- C ABI of the B200-native TILD particle-mesh step.
 *
 * One opaque box object replaces MATILDA.FT's PS_Box (PS_Box.h:19-212) together with
 * the objects it owns (PS_Group, PS_Potential and its kinds, Integrator GJF/EM,
 * PS_Species).  MATILDA.FT has no C ABI or plugin loader: its "API" is the input
 * script plus those C++ classes.  Each entry point below names the reference member
 * or code path it replaces (file:line in the MATILDA.FT source tree).
 *
 * Conventions
 *  - Every call returns an int status (TILD_OK == 0); nothing calls exit().  The
 *    reference dies instead (die.cu:7-20).  tild_last_error() returns the message of
 *    the last failing call on the calling thread.
 *  - All pointers are caller-owned HOST buffers; device memory is owned by the box.
 *  - A box is used from one host thread at a time (thread-compatible, not
 *    thread-safe) and issues its work on one CUDA stream (tild_box_set_stream).
 *  - Positions are float[n*Dim] interleaved (x fastest) as in the reference.
 */
#ifndef TILD_B200_H
#define TILD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum tild_status {
    TILD_OK = 0,
    TILD_ERR_ARG = 1,         /* bad argument / null pointer / size                  */
    TILD_ERR_PARSE = 2,       /* script or data-file error (reference: die())        */
    TILD_ERR_IO = 3,          /* file could not be opened or written                 */
    TILD_ERR_CUDA = 4,        /* a CUDA runtime call or kernel failed                */
    TILD_ERR_STATE = 5,       /* call out of order (e.g. step before endBox)         */
    TILD_ERR_UNSUPPORTED = 6, /* a script feature outside the TILD hot path          */
    TILD_ERR_DEVICE = 7       /* device-side check failed: a kernel counted particles whose
                                 position is not finite (the run blew up); reported when
                                 energies are read (log rows, thermo) */
};

typedef struct tild_box tild_box;

/* Summary of a box after endBox (PS_Box public members used by callers). */
typedef struct tild_box_info {
    int64_t nstot;        /* particles                                       */
    int32_t dim;          /* Dim                                             */
    int32_t nx[3];        /* grid                                            */
    float L[3];           /* box lengths                                     */
    int32_t pmeorder;     /* spline order                                    */
    int32_t n_groups;     /* psGroup.size()                                  */
    int32_t n_potentials; /* potentials.size()                               */
    int32_t n_density_fields; /* distinct density fields the potentials read */
    int32_t n_force_groups;   /* groups that receive grid forces             */
    int32_t n_bond_types;
    int64_t n_bonds;      /* nBondsTot                                       */
    int64_t step;         /* steps taken so far (totSteps)                   */
    int64_t device_bytes; /* device memory held by this box                  */
} tild_box_info;

/* Version / build string of the library. */
const char *tild_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char *tild_last_error(void);

/* Create an empty PS box on CUDA device `device` (reference: BoxFactory + PS_Box ctor,
 * Box.cu:491-507, PS_Box.cu:585-589).  Defaults follow PS_Box::readInput
 * (PS_Box_initialization.cu:36-62). */
int tild_box_create(int device, tild_box **out);

/* Free every device and host resource of the box (PS_Box::~PS_Box, PS_Box.cu:578). */
int tild_box_destroy(tild_box *box);

/* Use this CUDA stream (cudaStream_t passed as void*) for all work of the box; NULL
 * selects a stream the box creates itself.  The reference runs on the legacy default
 * stream (one host thread, PS_Box.cu:73-207). */
int tild_box_set_stream(tild_box *box, void *cuda_stream);

/* Set the directory that relative file names in the script (readData, datFileName)
 * resolve against.  The reference resolves them against the process working dir. */
int tild_box_set_base_dir(tild_box *box, const char *dir);

/* Feed one line of the `box ps` block, parsed word by word exactly like
 * PS_Box::readInput (PS_Box_initialization.cu:68-339).  The line "endBox" runs
 * finishInitialization (PS_Box_initialization.cu:352-569). */
int tild_box_command(tild_box *box, const char *line);

/* Feed a whole `box ps ... endBox` block (several lines; "box ps" itself optional);
 * the block must end with endBox (PS_Box::readInput, PS_Box_initialization.cu:32-345). */
int tild_box_read_input(tild_box *box, const char *text);

/* Particles supplied as arrays instead of `readData` (PS_Box::readDataConfig atoms
 * section, PS_Box_initialization.cu:858-884).  type is 0-based into the declared
 * species; mol may be NULL; q may be NULL unless doCharges was given.  Must precede
 * endBox. */
int tild_box_set_particles(tild_box *box, int64_t n, const float *x, const int32_t *type,
                           const int32_t *mol, const float *q);

/* Bonds supplied as arrays (readDataConfig bonds section,
 * PS_Box_initialization.cu:887-926): pairs[2*nbonds] 0-based particle ids,
 * btype[nbonds] 0-based bond types (NULL = all type 0).  Must precede endBox. */
int tild_box_set_bonds(tild_box *box, int64_t nbonds, const int64_t *pairs,
                       const int32_t *btype);

/* Angles supplied as arrays (readDataConfig angles section,
 * PS_Box_initialization.cu:933-993): triples[3*nangles] 0-based particle ids (i, middle
 * j, k), atype[nangles] 0-based angle types (NULL = all type 0); each angle is stored on
 * its three particles (at most MAXANGLES per particle).  Must precede endBox. */
int tild_box_set_angles(tild_box *box, int64_t nangles, const int64_t *triples, const int32_t *atype);

/* Options outside the reference grammar.  Keys:
 *   "rng"            0 = Philox4x32-10 (default), 1 = cuRAND XORWOW compatible mode
 *                    (same curand_init/curand_normal calls as device_utils.cu:465-472,
 *                    ps_integratorGJF.cu:140)
 *   "deterministic"  1 = deposit by exact fixed-point sums (bit-reproducible), 0 = fast
 *   "bspline4_exact" 1 = true quartic B-spline at pmeorder 4 instead of the
 *                    reference's weights (ps_grid_utils.cu:57)
 *   "write_files"    0 = write no files: ps_data.dat, init/final data files, and the
 *                    run's lammpstrj, GSD and density-<group>.bin outputs (default 1)
 *   "sort_interval"  steps between spatial re-sorts of the particle arrays (0 = never)
 *   "autotune"       1 = at endBox, time the force evaluation with particle tiles of
 *                    half, the same and twice the bricks per CTA, each with a staged and a
 *                    direct gather (staged cubic ones also with 64 more threads), then
 *                    the deposit's tiles (the same, twice, four and eight times the
 *                    bricks; one thread per particle or CTAs of 64, 128, 256), and keep
 *                    the fastest (default 0)
 *   "direct_gather"  1 = the particle gather reads each stencil through L1/L2 instead of
 *                    staging its tile's box in shared memory (default 0; same bits)
 *   "tile_codes"     fixed bricks per particle tile, a power of two <= 64 (0 = from the
 *                    particle density)
 *   "deposit_codes"  fixed bricks per deposit tile, a power of two in [8, 64] (0 = chosen)
 *   "deposit_threads" fixed deposit CTA size, a multiple of 32 in [64, 512] (0 = one
 *                    thread per particle of a typical tile)
 *   "gather_threads" fixed CTA size of the particle gather, a multiple of 32 in [64, 448]
 *                    (0 = about one thread per particle of a typical tile; same bits)
 * Must precede endBox except "write_files", "echo", "stage_timing" and "sort_interval". */
int tild_box_set_option(tild_box *box, const char *key, int64_t value);

/* JSON description of the parsed box (species, groups, potentials, integrators, grid,
 * box lengths) -- the state PS_Box holds after readInput.  Works before endBox and
 * without a GPU.  Writes at most size bytes including the terminating NUL; *needed
 * (may be NULL) receives the full size. */
int tild_box_describe(const tild_box *box, char *buf, int64_t size, int64_t *needed);

/* Box summary (valid after endBox). */
int tild_box_get_info(const tild_box *box, tild_box_info *out);

/* `run nvt nsteps`: PS_Box::NVT (PS_Box.cu:210-234) -- writeData(-1), nsteps calls of
 * doTimeStep with thermo logging every logFreq steps to datFileName (PS_Box.cu:339-370),
 * then the final writeData and final.input.data. */
int tild_box_run_nvt(tild_box *box, int64_t nsteps);

/* A top-level `modify` line after endBox, without the word `modify`: PS_Box::modifyBox
 * (PS_Box.cu:848-870).  "potential remove i" (or "delete") drops the i-th potential,
 * counted from 1 in script order; positions, the integrators' state, the noise streams and
 * the particle order are kept, so the next run continues the same trajectory.  Like the
 * reference, an out-of-range index or another word changes nothing. */
int tild_box_modify(tild_box *box, const char *rest);

/* nsteps time steps with no I/O and no thermo (PS_Box::doTimeStep, PS_Box.cu:73-162,
 * without the I/O branch :168-205).  Runs as replays of a captured CUDA graph. */
int tild_box_step(tild_box *box, int64_t nsteps);

/* Total force on every particle at the current positions, f[n*Dim] (PS_Box::forces,
 * PS_Box.cu:240-278, after the deposit of :97-114).  Positions are not changed. */
int tild_box_forces(tild_box *box, float *f_out);

/* Thermodynamic terms at the current positions (PS_Box::computeThermoProps,
 * PS_Box.cu:282-317) in FP64: out[0] = Upe, out[1] = Ubond, out[2+i] = energy of
 * potential i (i < npot); then three 6-component tensors in the order xx, yy, zz, xy,
 * xz, yz: the bonded virial (sum over bonds of dr_a f_b plus, over angles,
 * r_ij,a f_i,b + r_kj,a f_k,b), the pair virial -dU_pair/d(strain_ab)
 * (= U_pair delta_ab + sum_k (du/dk / k) k_a k_b Re(rho_I* rho_J), the reference has no
 * counterpart), and the pressure tensor (N kT delta_ab + W_pair + W_bonded) / V with
 * kT = 1; last the angle energy Uangle (included in Upe, PS_Box.cu:296-315).
 * Writes min(nout, 2 + npot + 19) values; *nwritten (may be NULL) receives the count. */
int tild_box_thermo(tild_box *box, double *out, int nout, int *nwritten);

/* Copy positions device -> host (x_out[n*Dim]) / host -> device (x_in[n*Dim]).  Setting
 * positions also resets the GJF old positions to them (GJF::finishInitialization,
 * ps_integratorGJF.cu:48-51).  A 2-D box (Dim 2) runs as one grid plane: its particles
 * stay at z = 0 and only x, y are read and written. */
int tild_box_get_positions(tild_box *box, float *x_out);
int tild_box_set_positions(tild_box *box, const float *x_in);

/* Density field of group `group` at the current positions (PS_Group::d_rho, or d_rhoq
 * when charge_channel != 0), rho_out[M] in the reference's x-fastest order. */
int tild_box_get_density(tild_box *box, const char *group, int charge_channel, float *rho_out);

/* Grid force of group `group` from the last force evaluation (tild_box_forces or a
 * step): PS_Group::d_gridForce after the potentials' CalcForces (ps_potential.cu:41-125,
 * ps_groups.cu:164-179), gf_out[M*Dim] interleaved per grid point in the reference's
 * x-fastest order and units (the particle force is sum_m gf[m] W_m).  A group that takes
 * no grid force reads zeros. */
int tild_box_get_grid_force(tild_box *box, const char *group, float *gf_out);

/* No counterpart in the reference.  tild_box_get_density for callers that cannot
 * allocate device memory: a host program whose pool allocator has reserved the device's
 * memory up front (so cudaMalloc fails or fragments the pool), or one that reads
 * densities between steps of other work on other streams, where cudaFree would
 * synchronise the whole device.  The device scratch (4 bytes per grid point, per
 * particle and per site of the group) comes instead from one static device array of
 * TILD_NOALLOC_SCRATCH_BYTES (16 MiB), which every GPU that loads the library holds until
 * the process exits.  A box needing more is refused with TILD_ERR_ARG ("... the static
 * scratch holds ...").  The first call on a device looks the array's address up
 * (cudaGetSymbolAddress, with that device current), which can load the library's device
 * code: make that first call before any stream capture.  Every call on a device shares
 * the array, which keeps the last call's contents; the call clears the part that must
 * start at zero (the density accumulator) itself.  Calls that overlap on one device
 * (two boxes, or two host threads) race on the array.  The call returns after the copy
 * to rho_out[M] has finished.  The looked-up address is kept for the life of the
 * process: do not call this entry point on a device after cudaDeviceReset (or any reset
 * of its primary context) in the same process. */
#define TILD_NOALLOC_SCRATCH_BYTES (16u << 20)
int tild_box_get_density_noalloc(tild_box *box, const char *group, int charge_channel, float *rho_out);

/* Structure factor of group `group`'s density (or its charge density when charge_channel
 * != 0) at the current positions: rho^(k) rho^(-k) with rho^ = FFT(rho)/M, as the
 * reference's S(k) compute defines it (ps_compute_sk.cu:18-50, which the reference never
 * initialises), over every k-vector of the grid, averaged in nbins shells of |k| of width
 * kmax/nbins, in FP64: sk_out[b], the mean |k| in the shell k_out[b] and the number of
 * k-vectors count_out[b] (any of the three may be NULL). */
int tild_box_structure_factor(tild_box *box, const char *group, int charge_channel, int32_t nbins, double kmax,
                              double *k_out, double *sk_out, double *count_out);

/* Stencil indices and weights of every particle at the current positions
 * (d_calcGridWeights, ps_grid_utils.cu:74-204): inds_out/w_out[n*(pmeorder+1)^Dim],
 * same order and float arithmetic as the reference (weights divided by gvol). */
int tild_box_grid_weights(tild_box *box, int32_t *inds_out, float *w_out);

/* Energies recorded by the runs so far (one row per logged step: step, Ubond, pot...)
 * copied to out[rows*cols]; rows and cols report the shape (the widest row; rows logged
 * while fewer potentials existed end in zeros).  Pass out=NULL to query. */
int tild_box_get_log(tild_box *box, double *out, int64_t *rows, int32_t *cols);

/* Execute a whole MATILDA.FT input script file (main.cu:21-156): `box ps` blocks,
 * `run nvt N`, `modify potential remove i`; unknown top-level words are ignored as in
 * the reference.  Output files are written next to the script. */
int tild_run_script_file(const char *path, int device);

/* Average device seconds per launch of each kernel during the last tild_box_step call
 * made with option "stage_timing" = 1 (then the steps run as individual launches with a
 * CUDA event after every kernel instead of as graph replays):
 * out[0] zero + deposit, [1] x-axis forward FFT, [2] y-axis forward FFT,
 * [3] z-axis FFT + k-space multiply + inverse z FFT, [4] y-axis inverse FFT,
 * [5] x-axis inverse FFT, [6] particle pass.  The reference has no counterpart (it keeps
 * second-resolution timers only, timing.h:8-12).  *n receives the count written. */
int tild_box_stage_times(tild_box *box, double *out, int nmax, int *n);

/* ---- Job pool: many boxes on one GPU (batched replicas, served jobs) ----------------
 * No counterpart in the reference, which runs one box per process (main.cu:21-156).  A
 * job is a box whose script and particles are given but whose endBox has NOT been
 * processed, plus a number of steps (doTimeStep without I/O, like tild_box_step).  A
 * scheduler thread admits queued jobs in arrival order while their estimated device
 * memory fits mem_budget_bytes and fewer than max_active (<= 0: no limit) are running,
 * allocates them then (stream-ordered, no device-wide synchronisation), and keeps chunks
 * of steps in flight on each job's own stream so that the jobs overlap on the GPU.  When a
 * job finishes, its positions and thermo are copied to the host and its device memory is
 * freed, so queued jobs enter while others are still running (continuous batching). */
typedef struct tild_pool tild_pool;
enum { TILD_JOB_QUEUED = 0, TILD_JOB_RUNNING = 1, TILD_JOB_DONE = 2, TILD_JOB_FAILED = 3, TILD_JOB_CANCELLED = 4 };

int tild_pool_create(int device, int64_t mem_budget_bytes, int32_t max_active, tild_pool **out);
/* Cancels queued jobs, waits for running ones, frees everything. */
int tild_pool_destroy(tild_pool *pool);
/* Hands `box` to the pool (its handle is emptied; still call tild_box_destroy on it).  The
 * script is checked and the device memory estimated here: TILD_ERR_ARG if the job alone
 * exceeds the budget, TILD_ERR_STATE if endBox was already processed; on an error the
 * caller keeps the box. */
int tild_pool_submit(tild_pool *pool, tild_box *box, int64_t nsteps, int64_t *job_id);
/* state: TILD_JOB_*; times3 (may be NULL): submit, admission and completion times in
 * seconds since the pool was created (0 until reached). */
int tild_pool_status(tild_pool *pool, int64_t job_id, int32_t *state, int64_t *steps_done, double *times3);
/* Blocks until the job is done; TILD_ERR_STATE with the job's error if it failed or was
 * cancelled. */
int tild_pool_wait(tild_pool *pool, int64_t job_id);
/* Cancels a queued or running job.  A queued job leaves the queue at once; a running one
 * stops taking new chunks of steps, its chunks already on the GPU finish, and then its
 * device memory is freed and its state becomes TILD_JOB_CANCELLED (tild_pool_wait
 * returns then, with TILD_ERR_STATE).  Other jobs are not disturbed.  TILD_ERR_STATE for a
 * job that has already finished, failed or been cancelled. */
int tild_pool_cancel(tild_pool *pool, int64_t job_id);
/* Changes the memory budget.  It applies to admissions from now on: running jobs keep
 * their memory and run to completion, queued jobs enter once the running set fits the new
 * budget, and queued jobs larger than the whole new budget fail (TILD_JOB_FAILED). */
int tild_pool_set_budget(tild_pool *pool, int64_t mem_budget_bytes);
/* Final positions x_out[n*Dim] (particle order, may be NULL) and up to nthermo values of
 * tild_box_thermo's layout at the last step. */
int tild_pool_result(tild_pool *pool, int64_t job_id, float *x_out, double *thermo_out, int32_t nthermo,
                     int32_t *nwritten);
/* Forgets a finished, failed or cancelled job. */
int tild_pool_release(tild_pool *pool, int64_t job_id);
/* out[0..6]: queued, running, done, failed, device bytes reserved by running jobs, budget,
 * cancelled. */
int tild_pool_stats(tild_pool *pool, int64_t *out, int32_t nout);

/* ---- Batch: replicas stepped together, one launch per step stage --------------------
 * No counterpart in the reference, which runs one box per process (main.cu:63-76) and
 * steps it alone (PS_Box::doTimeStep, PS_Box.cu:73-207).  A batch holds boxes whose
 * endBox has been processed and that share the kernels' compile-time settings: 3-D, the
 * same pmeorder, one or two density fields and force groups in each, the same
 * deterministic mode and sort_interval, no ramped potential, and the tile gather (sorted
 * tiles with TMA boxes).  Sizes, grids, potentials' amplitudes, tiles, integrators and
 * seeds may differ.  Each step runs every stage of the TILD step (zeroing the deposit
 * targets, the deposit, the five transform passes, the grid gather, the integrator pass,
 * the step counters) as ONE kernel launch over the work of all replicas -- their
 * geometries, FFT plans, tile lists and TMA descriptors in a device table -- and the ten
 * launches of a step are captured once in a CUDA graph; each replica's spatial re-sort
 * runs every sort_interval steps as a branch of one more graph.  A step is bit-identical to
 * tild_box_step on each replica in deterministic mode.  The boxes stay the caller's: read
 * them with tild_box_get_positions, tild_box_thermo and the like; destroy the batch before
 * its boxes (tild_box_destroy refuses a box that belongs to a batch). */
typedef struct tild_batch tild_batch;

int tild_batch_create(int device, tild_batch **out);
int tild_batch_destroy(tild_batch *batch);
/* Adds a box: TILD_ERR_STATE before its endBox or when it belongs to a batch already,
 * TILD_ERR_UNSUPPORTED (with the reason) when it does not share the batch's settings. */
int tild_batch_add(tild_batch *batch, tild_box *box);
int tild_batch_size(tild_batch *batch, int32_t *n);
/* Splits the replicas into `streams` (1..8) groups of about equal work, each stepped by
 * its own graph on its own stream: one launch per stage per group, the groups' stages
 * overlapping on the GPU.  1 (the default) is one launch per stage for the whole batch. */
int tild_batch_set_streams(tild_batch *batch, int32_t streams);
/* nsteps steps of every replica (doTimeStep without I/O, like tild_box_step); returns when
 * they are done. */
int tild_batch_step(tild_batch *batch, int64_t nsteps);

#ifdef __cplusplus
}
#endif

#endif /* TILD_B200_H */
