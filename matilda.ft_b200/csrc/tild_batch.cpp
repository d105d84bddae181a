// tild_batch.cpp -- replicas stepped together, one launch per step stage (tild_batch.h).
#include "tild_batch.h"

#include "tild_b200.h"

#include <algorithm>
#include <cstring>

namespace tild {

Batch::Batch(int dev) : device(dev)
{
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        throw BoxError{TILD_ERR_DEVICE, "batch: cannot use device " + std::to_string(device)};
    }
}

Batch::~Batch()
{
    cudaSetDevice(device);
    release();
    for (Box *b : boxes) b->inBatch = nullptr;
    for (cudaStream_t s : forks) cudaStreamDestroy(s);
}

void Batch::release()
{
    for (Group &g : groups) {
        if (g.stream) cudaStreamSynchronize(g.stream);
        if (g.gStep) cudaGraphExecDestroy(g.gStep);
        if (g.gSort) cudaGraphExecDestroy(g.gSort);
        if (g.dReps) cudaFree(g.dReps);
        if (g.dPre) cudaFree(g.dPre);
        if (g.stream) cudaStreamDestroy(g.stream);
    }
    groups.clear();
    built = false;
}

void Batch::setStreams(int k)
{
    if (k < 1 || k > 8) throw BoxError{TILD_ERR_ARG, "batch: streams must be in [1, 8]"};
    nstreams = k;
    release();
}

// The settings a batch's launches share are fixed by its first replica; each later one
// must match them.
void Batch::add(Box *b)
{
    auto refuse = [](const std::string &why) { throw BoxError{TILD_ERR_UNSUPPORTED, "batch: " + why}; };
    if (!b->ready) throw BoxError{TILD_ERR_STATE, "batch: the box's endBox has not been processed"};
    if (b->inBatch) throw BoxError{TILD_ERR_STATE, "batch: the box already belongs to a batch"};
    if (b->device != device) refuse("the box lives on device " + std::to_string(b->device));
    if (b->Dim != 3 || b->geom.nz < 2) refuse("two-dimensional boxes are stepped alone");
    const int bnd = (int)b->dfields.size(), bnfg = (int)b->fgroups.size();
    if (bnd < 1 || bnd > 2) refuse("a replica needs one or two density fields (this box has " + std::to_string(bnd) + ")");
    if (bnfg < 1 || bnfg > 2) refuse("a replica needs one or two force groups (this box has " + std::to_string(bnfg) + ")");
    for (const PS_Potential &p : b->potentials)
        if (p.ramp) refuse("ramped potentials update their amplitude between steps; step such a box alone");
    if (!b->sortedTiles || !b->tiles.paired || !b->recLayout().paired)
        refuse("the box does not use the tile gather over paired records (sorted tiles with TMA boxes)");
    if (kspace_tile_width(b->geom, bnd, bnfg, (int)b->potentials.size()) == 0) refuse("the box's k-space pass does not fit");
    const int bextra = (b->dNa != nullptr || b->ppHost.nwall > 0) ? 1 : 0;
    if (boxes.empty()) {
        order = b->pmeorder;
        nd = bnd;
        nfg = bnfg;
        deterministic = b->deterministic;
        sortInterval = b->sortInterval;
    } else {
        if (b->pmeorder != order) refuse("every replica needs the same pmeorder");
        if (bnd != nd || bnfg != nfg) refuse("every replica needs the same numbers of density fields and force groups");
        if (b->deterministic != deterministic) refuse("every replica needs the same deterministic mode");
        if (b->sortInterval != sortInterval) refuse("every replica needs the same sort_interval");
    }
    extra |= bextra;
    b->ck(cudaStreamSynchronize(b->stream), "batch add");
    boxes.push_back(b);
    b->inBatch = this;
    release();
}

static void batch_ck(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw BoxError{TILD_ERR_DEVICE, std::string("batch: ") + what + ": " + cudaGetErrorString(e)};
    }
}

// Groups of about equal work (grid points plus particles), each in dispatch order: the
// replicas whose CTAs take longest first -- largest prime factor of a grid edge (the
// generic FFT stage costs O(p) per point), then the largest grid -- so that the slow CTAs
// overlap the many short ones instead of forming each stage's tail.
void Batch::build()
{
    release();
    const int R = (int)boxes.size();
    if (R == 0) return;
    cudaSetDevice(device);
    auto maxPrime = [](int n) {
        int m = n, p = 1;
        for (int f = 2; f * f <= m; f++)
            while (m % f == 0) {
                p = std::max(p, f);
                m /= f;
            }
        return std::max(p, m);
    };
    std::vector<int> ord(R);
    std::vector<long long> key(R);
    for (int r = 0; r < R; r++) {
        const Geom &g = boxes[r]->geom;
        ord[r] = r;
        key[r] = (long long)std::max(maxPrime(g.nx), std::max(maxPrime(g.ny), maxPrime(g.nz))) * (1ll << 40) + g.M;
    }
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return key[a] > key[b]; });
    const int k = std::min(nstreams, R);
    groups.resize(k);
    std::vector<double> work(k, 0.0);
    std::vector<int> byWork(ord);
    std::stable_sort(byWork.begin(), byWork.end(), [&](int a, int b) {
        return boxes[a]->geom.M + boxes[a]->nstot > boxes[b]->geom.M + boxes[b]->nstot;
    });
    std::vector<int> groupOf(R, 0);
    for (int r : byWork) {   // the largest remaining replica to the group with the least work
        const int gi = (int)(std::min_element(work.begin(), work.end()) - work.begin());
        groupOf[r] = gi;
        work[gi] += (double)boxes[r]->geom.M + (double)boxes[r]->nstot;
    }
    for (int r : ord) groups[groupOf[r]].reps.push_back(boxes[r]);
    while ((int)forks.size() < 8) {
        cudaStream_t f;
        batch_ck(cudaStreamCreateWithFlags(&f, cudaStreamNonBlocking), "stream");
        forks.push_back(f);
    }
    for (Group &g : groups) {
        batch_ck(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking), "stream");
        buildGroup(g);
    }
    sinceSort = 0;
    for (Box *b : boxes) sinceSort = std::max(sinceSort, b->sinceSort);
    built = true;
}

void Batch::buildGroup(Group &G)
{
    const int R = (int)G.reps.size();
    G.txz = 4;
    for (Box *b : G.reps)
        G.txz = std::min(G.txz, kspace_tile_width(b->geom, nd, nfg, (int)b->potentials.size()));
    std::vector<BatchRep> h(R);
    for (int r = 0; r < R; r++) {
        Box *b = G.reps[r];
        BatchRep &e = h[r];
        std::memset(&e, 0, sizeof(e));
        const RecLayout rl = b->recLayout();
        e.mapA = b->pmapA;
        e.mapB = b->pmapB;
        e.g = b->geom;
        e.lx = b->lx;
        e.ly = b->ly;
        e.lz = b->lz;
        e.tiles = b->tileCfg();
        e.dtiles = b->depTileCfg();
        e.rl = rl;
        e.aa = AngleArrays{b->dNa, b->dAtype, b->dAng};
        e.ppd = b->dPp;
        e.ks = b->dKs;
        e.uk = b->dUk;
        e.N = (int)b->nstot;
        e.quirk4 = b->ppHost.quirk4;
        e.nd = nd;
        e.nfg = nfg;
        e.int_tile_max = b->ppHost.int_tile_max;
        e.dq = b->ppHost.dchan_charge;
        e.Lx = fft_batch_lines(BS_XFWD, b->geom, nfg);
        e.Lxi = fft_batch_lines(BS_XINV, b->geom, nfg);
        e.txz = G.txz;
        e.ks_npots = (int)b->potentials.size();
        e.X0 = b->dX[0];
        e.X1 = b->dX[1];
        e.noise = b->dNoise;
        e.flags = b->dFlags;
        e.q = b->dQ;
        e.brow = b->dBrow;
        e.partner = b->dPartner;
        e.btype = b->dBtype;
        e.orig = b->dOrig;
        e.rng = b->dRng;
        e.dep = b->dDep;
        e.depfix = b->dDepFix;
        e.H = b->dH;
        e.Hg = b->dHg;
        e.rec = b->dRec;
        e.fgrid = b->dFgrid;
        e.d_step = b->dStep;
        e.err = b->dErr;
        int blocks, threads, cap;
        size_t smem;
        deposit_batch_shape(e, deterministic, &blocks, &threads, &smem, &cap);
        e.dep_cap = cap;
    }
    // every stage's prefix table of CTA counts, its widest CTA and largest shared memory
    std::vector<int> pre((size_t)(BS_COUNT + 1) * (R + 1), 0);
    for (int s = 0; s <= BS_COUNT; s++) {
        int *ps = pre.data() + (size_t)s * (R + 1);
        BatchLaunch &bl = G.launches[s];
        bl.threads = 0;
        bl.smem = 0;
        for (int r = 0; r < R; r++) {
            int blocks = 0, threads = 256, cap = 0;
            size_t smem = 0;
            if (s == BS_COUNT) zero_batch_shape(h[r], deterministic, &blocks);
            else if (s == BS_DEPOSIT) deposit_batch_shape(h[r], deterministic, &blocks, &threads, &smem, &cap);
            else if (s == BS_GATHER || s == BS_INTEGRATE) particles_batch_shape(s, h[r], &blocks, &threads, &smem);
            else fft_batch_shape(s, h[r], &blocks, &threads, &smem);
            ps[r + 1] = ps[r] + blocks;
            bl.threads = std::max(bl.threads, threads);
            bl.smem = std::max(bl.smem, smem);
        }
        bl.blocks = ps[R];
    }
    batch_ck(cudaMalloc(&G.dReps, sizeof(BatchRep) * R), "cudaMalloc");
    batch_ck(cudaMalloc(&G.dPre, sizeof(int) * pre.size()), "cudaMalloc");
    batch_ck(cudaMemcpy(G.dReps, h.data(), sizeof(BatchRep) * R, cudaMemcpyHostToDevice), "table upload");
    batch_ck(cudaMemcpy(G.dPre, pre.data(), sizeof(int) * pre.size(), cudaMemcpyHostToDevice), "table upload");
    for (int s = 0; s <= BS_COUNT; s++) G.launches[s].pre = G.dPre + (size_t)s * (R + 1);
    // the step: zero, deposit, x/y forward, k-space, y/x inverse, gather, integrate, tick
    const cudaStream_t st = G.stream;
    cudaGraph_t gr;
    batch_ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t e = launch_zero_batch(G.dReps, R, G.launches[BS_COUNT], deterministic, st);
    if (e == cudaSuccess) e = launch_deposit_batch(G.dReps, R, G.launches[BS_DEPOSIT], order, nd, deterministic, st);
    for (int s : {BS_XFWD, BS_YFWD, BS_KSPACE, BS_YINV, BS_XINV})
        if (e == cudaSuccess) e = launch_fft_batch(s, G.dReps, R, G.launches[s], deterministic, G.txz, st);
    for (int s : {BS_GATHER, BS_INTEGRATE})
        if (e == cudaSuccess) e = launch_particles_batch(s, G.dReps, R, G.launches[s], order, nfg, extra, st);
    if (e == cudaSuccess) e = launch_batch_tick(G.dReps, R, st);
    const cudaError_t ec = cudaStreamEndCapture(st, &gr);
    batch_ck(e, "step capture");
    batch_ck(ec, "end capture");
    e = cudaGraphInstantiate(&G.gStep, gr, 0);
    cudaGraphDestroy(gr);
    batch_ck(e, "graph instantiate");
    // the re-sort: every replica's sort kernels and copies on one of the forked streams,
    // branches of one graph joined at its end
    if (sortInterval > 0) {
        std::vector<cudaEvent_t> ev(1 + forks.size());
        for (cudaEvent_t &x : ev) batch_ck(cudaEventCreateWithFlags(&x, cudaEventDisableTiming), "event");
        batch_ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
        cudaError_t err = cudaEventRecord(ev[0], st);
        const int nf = std::min((int)forks.size(), R);
        for (int f = 0; f < nf && err == cudaSuccess; f++) err = cudaStreamWaitEvent(forks[f], ev[0], 0);
        for (int r = 0; r < R && err == cudaSuccess; r++) {
            Box *b = G.reps[r];
            const cudaStream_t own = b->stream;
            b->stream = forks[r % nf];
            try {
                b->sortParticles();
            } catch (...) {
                err = cudaErrorUnknown;
            }
            b->stream = own;
        }
        for (int f = 0; f < nf && err == cudaSuccess; f++) {
            err = cudaEventRecord(ev[1 + f], forks[f]);
            if (err == cudaSuccess) err = cudaStreamWaitEvent(st, ev[1 + f], 0);
        }
        const cudaError_t ec2 = cudaStreamEndCapture(st, &gr);
        for (cudaEvent_t &x : ev) cudaEventDestroy(x);
        batch_ck(err, "sort capture");
        batch_ck(ec2, "end capture");
        err = cudaGraphInstantiate(&G.gSort, gr, 0);
        cudaGraphDestroy(gr);
        batch_ck(err, "graph instantiate");
    }
}

void Batch::step(int64_t n)
{
    if (boxes.empty() || n <= 0) return;
    cudaSetDevice(device);
    if (!built) build();
    for (int64_t i = 0; i < n; i++) {
        const bool sort = sortInterval > 0 && sinceSort >= sortInterval;
        for (Group &g : groups) {
            if (sort) batch_ck(cudaGraphLaunch(g.gSort, g.stream), "sort graph");
            batch_ck(cudaGraphLaunch(g.gStep, g.stream), "step graph");
        }
        if (sort) sinceSort = 0;
        sinceSort++;
    }
    for (Group &g : groups) batch_ck(cudaStreamSynchronize(g.stream), "batch step");
    for (Box *b : boxes) {
        b->totSteps += n;
        b->sinceSort = sinceSort;
        b->checkDeviceErrors();
    }
}

}  // namespace tild
