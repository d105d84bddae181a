// tild_box.h -- host-side mirror of MATILDA.FT's PS_Box object model.
//
// Class and member names follow the reference (PS_Box.h:19-212, ps_groups.h:27-63,
// ps_potential.h:13-53, ps_integrator.h:21-39, ps_species.h); the device work is the
// fused B200 pipeline of tild_device.h instead of per-object kernels.
#pragma once
#include <cstdint>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "tild_device.h"
#include "tild_gsd.h"

namespace tild {

class Batch;

struct BoxError {
    int code;
    std::string msg;
};

[[noreturn]] void fail(int code, const std::string &msg);   // throws BoxError

struct PS_Species {          // ps_species.cu:13-38
    std::string label;
    float mass = 1.0f;
    float mobility = 1.0f;
};

struct PS_Group {            // ps_groups.h:27-63
    std::string name;
    std::string inputCommand;
    std::vector<int> siteList;
    bool forceFlag = false;
    bool isCharges = false;
};

struct PS_Potential {        // ps_potential.h:13-53 and the Gaussian/Erf2/ErfG/Charge kinds
    std::string word;        // script word: gaussian, erf2, erfG, charges
    int kind = POT_GAUSSIAN;
    std::string grpI, grpJ;
    int Iind = -1, Jind = -1;
    float Ao = 0.f, sigma = 0.f, Rp = 0.f, LB = 0.f;
    bool ramp = false;
    int wallAxis = 0, wallSign = 1;   // `wall` (ps_potentialWall.cu:11-46): normal axis, side
    float wallPos = 0.f, wallK = 0.f;
    double Ao_initial = 0.0, Ao_final = 0.0;
    double amp_eff = 0.0;    // amplitude the k-space tables currently carry
    double energy = 0.0;     // last CalcEnergy value
    std::string input_command;
    double T0() const;       // u(k=0)/amplitude of the kind
};

struct Integrator {          // ps_integrator.h:21-39, GJF and EM kinds
    std::string groupName;
    std::string name;        // GJF / EM
    float delt = 0.002f;
    int group_index = -1;
    std::string command_line;
};

class Box {
public:
    explicit Box(int device);
    ~Box();

    // ---- input (PS_Box::readInput, PS_Box_initialization.cu:32-345) ----
    void command(const std::string &line);          // one line, word by word
    void finishInitialization();                      // endBox (:352-569) = prepareHost + initDevice
    void prepareHost();                               // host checks, default groups, k-space plan
    void initDevice();                                // device arrays, uploads, first sort
    int64_t deviceBytesEstimate() const;              // device bytes initDevice will allocate (after prepareHost)
    // stream-ordered allocation (cudaMallocAsync/cudaFreeAsync on the box's stream) and no
    // device-wide synchronisation: for boxes that share a GPU with other running work
    void setSharedDevice(bool on, cudaMemPool_t pool = nullptr)
    {
        sharedDevice = on;
        memPool = pool;
    }
    void readDataConfig(const std::string &name);     // :787-997
    void setParticles(int64_t n, const float *x, const int32_t *type, const int32_t *mol, const float *q);
    void setBonds(int64_t nb, const int64_t *pairs, const int32_t *btype);
    void setAngles(int64_t na, const int64_t *triples, const int32_t *atype);
    void setOption(const std::string &key, int64_t value);
    void setStream(cudaStream_t st);
    void setBaseDir(const std::string &d) { baseDir = d; }
    bool initialized() const { return ready; }
    cudaStream_t cudaStreamHandle() const { return stream; }

    // ---- run ----
    void NVT(int64_t nSteps);                          // PS_Box.cu:210-234
    void steps(int64_t n);                             // doTimeStep x n, no I/O
    void forces(float *f_out);                         // PS_Box::forces at current x
    // computeThermoProps (+ virial) at the current positions; with lastStepStart the pair
    // terms come from the densities the last step started from (what the reference's
    // groups still hold when a later run logs its step -1 row)
    std::vector<double> thermo(bool lastStepStart = false);
    void getPositions(float *x) const;
    void readRows3(const float *dev, float *out) const;
    void setPositions(const float *x);
    void getDensity(const std::string &group, int charge, float *rho);
    void getGridForce(const std::string &group, float *gf);   // PS_Group::d_gridForce
    void getDensityNoAlloc(const std::string &group, int charge, float *rho);
    void structureFactor(const std::string &group, int charge, int nbins, double kmax, double *k_out,
                         double *sk_out, double *count_out);
    void gridWeights(int32_t *inds, float *w);
    void modifyBox(const std::string &rest);           // PS_Box.cu:848-870
    void stageTimes(std::vector<double> &out) const { out = stageSec; }
    std::string describe() const;

    // info
    int64_t nstot = 0;
    int Dim = 0;
    int Nx[3] = {0, 0, 0};
    float L[3] = {0, 0, 0}, Lh[3] = {0, 0, 0};
    double dx[3] = {0, 0, 0};
    double gvol = 0.0;
    int pmeorder = 1;
    int64_t nBondsTot = 0;
    int64_t nBondEntries = 0;   // stored partner entries (each bond twice)
    int nBondTypes = 0;
    int64_t totSteps = 0;
    std::vector<PS_Group> psGroup;
    std::vector<PS_Potential> potentials;
    std::vector<std::vector<double>> logRows;
    int nDensityFields() const { return (int)dfields.size(); }
    int nForceGroups() const { return (int)fgroups.size(); }
    int64_t deviceBytes() const { return devBytes; }
    int logColumns() const { return 2 + (nAnglesTot > 0 ? 1 : 0) + (int)potentials.size(); }
    bool echo = false;
    Batch *inBatch = nullptr;       // the batch this box belongs to (tild_batch.h), if any

private:
    friend class Batch;
    // parse helpers
    void parseWords(std::vector<std::string> &w, size_t &i);
    void addPotential(std::vector<std::string> &w, size_t &i);
    int findGroupInteger(const std::string &name) const;
    int findSpeciesInteger(const std::string &name) const;
    void createDefaultGroups();
    void writeDataConfig(const std::string &name);
    void writeData(int64_t step, const std::vector<double> &pairE, double ubond, double uangle);
    std::string resolve(const std::string &name) const;

    // device plan
    void buildPlan();
    void allocDevice();
    void freeDevice();
    void uploadParticles();
    void enqueueStep(bool energy, bool integrate, float *fout_dev);
    void enqueueEnergyOnly(bool lastStepStart = false);
    const CUtensorMap *recordMap();
    void checkDeviceErrors();
    void updateRamps(int64_t step, int64_t maxSteps);
    void captureGraphs();
    void dropGraphs();
    std::vector<double> readEnergies(bool with_bond);
    void ck(cudaError_t e, const char *what) const;
    template <typename T> T *dalloc(size_t count);

    int device = 0;
    bool ready = false;
    bool readDimension = false;
    std::string baseDir = ".";
    // reference defaults (PS_Box_initialization.cu:36-62)
    int blockSize = 512, NSEXTRA = 0, MAXBONDS = 2, MAXANGLES = 3, Nr = 100;
    double rho0 = -1.0;
    long long RANDSEED = 0;
    // the reference's host RNG (random.cu:27-106), one state per box: ran2's generator
    // state and shuffle table, gasdev2's cached spare normal
    int64_t idum = 0, idum2 = 123456789, iy = 0;
    int64_t iv[32] = {0};
    int gasIset = 0;
    double gasGset = 0.0;
    double ran2();
    double gasdev2();
    void randomUnitVec(double *v, int dim);
    void makeLinear(std::vector<std::string> &w, size_t &i);   // PS_Box_moleculeMakers.cu:15-311
    int logFreq = 100;
    std::string datFileName = "ps_data.dat", initDataFileName = "init.input.data";
    // output written during NVT (PS_Box.cu:166-205): lammpstrj frames every trajFreq
    // steps, group density frames (density-<group>.bin) every fieldFreq steps with an
    // optional geometric growth of the interval (logspace)
    int trajFreq = 0, fieldFreq = 0;
    std::string trajFileName = "traj.lammpstrj";
    bool logSpaceFields = false;
    float logScaleFields = 1.0f;
    // GSD trajectory (PS_Box_gsdUtils.cu:14-168): a full frame when the box's step count is
    // 0 (at set-up, and again at the first step of the first run), positions (and charges)
    // every gsdFreq steps and at the end of every run
    int gsdFreq = 0;
    bool logSpaceGSD = false;
    float logScaleGSD = 1.0f;
    std::string gsdName = "traj.gsd";
    GsdWriter gsd;
    void writeGsdFrame(int64_t step, const float *x_orig);
    bool doCharges = false;
    bool verbose = false;
    int nAnglesTot = 0;

    // options
    int rngCompat = 0, deterministic = 0, exact4 = 0, writeFiles = 1, stageTiming = 0;

    std::vector<PS_Species> species;
    std::vector<Integrator> integrators;
    std::vector<float> bondK, bondReq;
    std::vector<int> bondStyle;

    // host particle state
    std::vector<float> x, charges;
    std::vector<int> intSpecies, mID;
    std::vector<int> nBonds, bondedTo, bondType;   // [n], [n*MAXBONDS]
    // angles (ps_deviceAngles.cu): every angle is stored on each of its three particles
    std::vector<int> nAngles, angleGroup, angleType;   // [n], [n*MAXANGLES*3], [n*MAXANGLES]
    std::vector<float> angleK, angleTheq;               // per angle type (theta in radians)
    std::vector<int> angleStyle;                        // 0 wlc, 1 harmonic
    std::vector<uint32_t> angleList;   // (type, i1, i2, i3) per angle read or set, in input order

    // derived plan
    struct DField { int group; int charge; };
    std::vector<DField> dfields;
    std::vector<int> fgroups;                      // group indices receiving grid forces
    Geom geom{};
    KSpace ksHost{};
    ParticleParams ppHost{};
    FftLine lx{}, ly{}, lz{};
    int nblkZ = 0, nblkP = 0;

    // device state
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    bool sharedDevice = false;
    cudaMemPool_t memPool = nullptr;   // shared-device arenas come from this pool when set
    // one arena per box: dalloc carves 256-byte aligned pieces, individual allocations
    // only if the arena is exhausted
    char *arena = nullptr;
    size_t arenaSize = 0, arenaUsed = 0;
    void *rawAlloc(size_t bytes);
    void rawFree(void *p);
    bool hostPrepared = false;
    std::vector<void *> allocs;
    int64_t devBytes = 0;
    float *dX[2] = {nullptr, nullptr};
    float *dNoise = nullptr, *dQ = nullptr, *dF = nullptr;
    uint32_t *dFlags = nullptr;
    int *dBrow = nullptr;                        // CSR bond rows [N+1] (NULL without bonds)
    int *dErr = nullptr;                         // failures the kernels record (see checkDeviceErrors)
    CUtensorMap recMap;                          // TMA descriptor of dRec for the tiles' box
    int recMapTe[3] = {0, 0, 0};
    bool recMapOk = false;
    CUtensorMap pmapA, pmapB;                    // TMA descriptors of the paired record planes
    int pmapTe[3] = {0, 0, 0}, pmapGl = -1, pmapGh[3] = {0, 0, 0};
    bool pmapOk = false;
    float *dFgrid = nullptr;                     // [3N] grid force of each particle (the gather's output)
    size_t recBytes = 0;                         // bytes of dRec: planar or paired records
    uint8_t *dBtype = nullptr;
    uint8_t *dNa = nullptr, *dAtype = nullptr;   // angles (NULL when the box has none)
    int *dAng = nullptr;
    int *dPartner = nullptr, *dOrig = nullptr;
    void *dRng = nullptr;
    float2 *dDep = nullptr, *dH = nullptr, *dHg = nullptr, *dTw = nullptr;
    unsigned long long *dDepFix = nullptr;
    float4 *dRec = nullptr;
    long long *dStep = nullptr;
    KSpace *dKs = nullptr;
    float *dUk = nullptr;   // FP32 û(k) shape table, one half-spectrum field per potential
    ParticleParams *dPp = nullptr;
    double *dEpart = nullptr, *dBpart = nullptr, *dRes = nullptr;
    KSpace *hKsPinned = nullptr;
    cudaGraphExec_t gNorm = nullptr, gEnergy = nullptr;
    std::vector<double> stageSec;
    // spatial re-sort of the particle arrays
    SortScratch sortW{};
    float *dTmp = nullptr;                 // [3N] scratch for slot <-> original order
    cudaGraphExec_t gSort = nullptr;
    int sortInterval = 10;
    int sinceSort = 0;
    bool sortedTiles = false;       // sortW.start holds the tile ranges of the current order
    uint32_t sortKeys = 0;
    TileCfg tiles{};                // codes / threads / box chosen from the density
    TileCfg dtiles{};               // the deposit's tiles (its own brick count: a larger tile
                                    // zeroes and flushes fewer halo points per particle)
    int depositCodes = 0;           // option "deposit_codes": fixed deposit tile bricks (0: chosen)
    int depositThreads = 0;         // option "deposit_threads": deposit CTA size (0: one thread per particle)
    int tileCodes = 0;              // option "tile_codes": fixed particle-pass tile bricks (0: from the density)
    int gatherThreads = 0;          // option "gather_threads": tile-gather CTA size (0: about one thread per particle)
    TileCfg tileCfg() const;
    TileCfg depTileCfg() const;
    void pairedGhosts(const TileCfg &t, int *gl, int *gh) const;   // ghost layers the tiles' boxes reach
    int densityCodes() const;       // bricks per tile from the density
    std::map<int, std::pair<uint32_t *, int>> tileLists;   // bricks per tile -> the tiles meeting the grid
    void attachTileList(TileCfg &t);  // t.list: the tiles of t.codes bricks that meet the grid (built once)
    size_t recordBytes() const;     // bytes of the force records (planar or paired)
    RecLayout recLayout();          // the records' layout for the current tiles (maps built)
    TileCfg tileGeometry(int codes, bool direct) const;
    bool autotune = false;          // option "autotune": time tile sizes at endBox
    bool directGather = false;      // option "direct_gather": particle pass reads L1/L2, no box
    float tunedMs = 0.f;            // force evaluation time of the chosen tiles
    void autotuneTiles();
    void uploadFlags();
    std::vector<int> slotOrder() const;
    void sortParticles();
    void maybeSort();
    long long deviceStep() const;
    // output snapshots: device work on the box's stream, copies into host buffers, each
    // frame written to its file once its event has completed (frames stay in step order)
    struct OutFrame {
        int kind;          // 0 field frame (all groups), 1 lammpstrj frame, 2 GSD frame
        int64_t step;
        float *host;
        size_t bytes;
        cudaEvent_t ev;
    };
    std::deque<OutFrame> outFrames;
    std::vector<std::pair<size_t, float *>> hostSpare;
    unsigned long long *dGroupMask = nullptr;   // [N] group bits of each original particle id
    float *dFieldFrame = nullptr;               // [nFrameGroups * M]
    int nFrameGroups = 0;
    bool fieldFrameValid = false;               // dFieldFrame holds the last step's densities
    bool fieldFilesReady = false;               // density-<group>.bin headers written
    void initFieldFiles();
    void computeFieldFrame();
    void enqueueFrame(int kind, int64_t step);
    void flushFrames(size_t keep);
    void writeFrame(const OutFrame &f);
    float *hostBuffer(size_t bytes);
    void releaseFrames();
    // per-kernel event timing (option "stage_timing")
    enum { STAGE_DEPOSIT, STAGE_XFWD, STAGE_YFWD, STAGE_KSPACE, STAGE_YINV, STAGE_XINV, STAGE_GATHER, STAGE_INTEGRATE,
           STAGE_COUNT };
    bool timing = false;
    std::vector<std::pair<int, cudaEvent_t>> marks;
    void mark(int stage);
};

}  // namespace tild
