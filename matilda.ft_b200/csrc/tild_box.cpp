// tild_box.cpp -- PS box host logic: script grammar, data files, plan building and the
// per-step launch sequence of the B200 TILD pipeline.
//
// Reference behaviour restated here (MATILDA.FT source tree):
//   PS_Box::readInput           PS_Box_initialization.cu:32-345 (word-by-word grammar)
//   PS_Box::finishInitialization PS_Box_initialization.cu:352-569
//   PS_Box::createDefaultGroups PS_Box_initialization.cu:573-587
//   PS_Box::readDataConfig      PS_Box_initialization.cu:787-997
//   PSPotentialFactory          ps_potential.cu:294-333, kinds' ctors (gaussian/erf2/erfG/charges)
//   IntegratorFactory / ctor    ps_integrator.cu:18-69
//   PS_Box::NVT, doTimeStep     PS_Box.cu:73-234; writeData PS_Box.cu:339-370
//   PS_Box::writeDataConfig     PS_Box.cu:629-748; modifyBox PS_Box.cu:848-870
#include "tild_box.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <numeric>
#include <sstream>

#include "tild_b200.h"

namespace tild {

void init_fft_attributes();
void init_deposit_attributes();
void init_particle_attributes();

[[noreturn]] void fail(int code, const std::string &msg) { throw BoxError{code, msg}; }

namespace {

std::vector<std::string> split(const std::string &line)
{
    std::vector<std::string> w;
    std::istringstream iss(line);
    std::string s;
    while (iss >> s) w.push_back(s);
    return w;
}

const std::string &need(const std::vector<std::string> &w, size_t &i, const char *what)
{
    if (i >= w.size()) fail(TILD_ERR_PARSE, std::string("missing value for ") + what);
    return w[i++];
}

double dnum(const std::vector<std::string> &w, size_t &i, const char *what)
{
    const std::string &s = need(w, i, what);
    char *end = nullptr;
    double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0') fail(TILD_ERR_PARSE, std::string("bad number '") + s + "' for " + what);
    return v;
}

float fnum(const std::vector<std::string> &w, size_t &i, const char *what)
{
    const std::string &s = need(w, i, what);
    char *end = nullptr;
    float v = std::strtof(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0') fail(TILD_ERR_PARSE, std::string("bad number '") + s + "' for " + what);
    return v;
}

long long inum(const std::vector<std::string> &w, size_t &i, const char *what)
{
    const std::string &s = need(w, i, what);
    char *end = nullptr;
    long long v = std::strtoll(s.c_str(), &end, 10);
    if (end == s.c_str() || *end != '\0') fail(TILD_ERR_PARSE, std::string("bad integer '") + s + "' for " + what);
    return v;
}

}  // namespace

double PS_Potential::T0() const
{
    const double PI4 = 12.566370614359172953850573533118;
    const double v = PI4 * (double)Rp * Rp * Rp / 3.0;
    if (kind == POT_ERF2) return v * v;
    if (kind == POT_ERFG) return v;
    return 1.0;
}

// =====================================================================================
Box::Box(int dev) : device(dev)
{
    RANDSEED = (long long)time(nullptr);   // idum = RANDSEED = time(0) (:45)
    idum = RANDSEED;
}

Box::~Box()
{
    releaseFrames();
    dropGraphs();
    freeDevice();
    if (hKsPinned) {
        if (sharedDevice) delete hKsPinned;
        else cudaFreeHost(hKsPinned);
    }
    if (ownStream && stream) cudaStreamDestroy(stream);
}

void Box::ck(cudaError_t e, const char *what) const
{
    if (e != cudaSuccess) fail(TILD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void *Box::rawAlloc(size_t bytes)
{
    void *p = nullptr;
    if (sharedDevice) {   // stream-ordered; usable by the synchronous uploads once the stream has reached it
        if (memPool) ck(cudaMallocFromPoolAsync(&p, bytes, memPool, stream), "cudaMallocFromPoolAsync");
        else ck(cudaMallocAsync(&p, bytes, stream), "cudaMallocAsync");
        ck(cudaStreamSynchronize(stream), "cudaMallocAsync");
    } else {
        ck(cudaMalloc(&p, bytes), "cudaMalloc");
    }
    return p;
}

void Box::rawFree(void *p)
{
    if (sharedDevice) cudaFreeAsync(p, stream);
    else cudaFree(p);
}

template <typename T>
T *Box::dalloc(size_t count)
{
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    const size_t padded = (bytes + 255) & ~(size_t)255;
    void *p;
    if (arena && arenaUsed + padded <= arenaSize) {
        p = arena + arenaUsed;
        arenaUsed += padded;
    } else {
        p = rawAlloc(bytes);
        allocs.push_back(p);
    }
    devBytes += (int64_t)bytes;
    return reinterpret_cast<T *>(p);
}

void Box::freeDevice()
{
    cudaSetDevice(device);
    for (void *p : allocs) rawFree(p);
    allocs.clear();
    if (arena) rawFree(arena);
    arena = nullptr;
    arenaSize = arenaUsed = 0;
    devBytes = 0;
}

std::string Box::resolve(const std::string &name) const
{
    if (name.empty() || name[0] == '/' || baseDir.empty() || baseDir == ".") return name;
    return baseDir + "/" + name;
}

void Box::setStream(cudaStream_t st)
{
    if (ownStream && stream) cudaStreamDestroy(stream);
    ownStream = false;
    stream = st;
    dropGraphs();
}

void Box::setOption(const std::string &key, int64_t v)
{
    if (key == "write_files") { writeFiles = (int)v; return; }
    if (key == "echo") { echo = v != 0; return; }
    if (key == "stage_timing") { stageTiming = (int)v; return; }
    if (ready && key != "sort_interval") fail(TILD_ERR_STATE, "option '" + key + "' must be set before endBox");
    if (key == "rng") rngCompat = (int)v;
    else if (key == "deterministic") deterministic = (int)v;
    else if (key == "bspline4_exact") exact4 = (int)v;
    else if (key == "autotune") autotune = v != 0;
    else if (key == "direct_gather") directGather = v != 0;
    else if (key == "deposit_codes") {
        if (v != 0 && (v < 8 || v > 64 || (v & (v - 1)))) fail(TILD_ERR_ARG, "deposit_codes must be 0 or a power of two in [8, 64]");
        depositCodes = (int)v;
    }
    else if (key == "tile_codes") {
        if (v != 0 && (v < 1 || v > 64 || (v & (v - 1)))) fail(TILD_ERR_ARG, "tile_codes must be 0 or a power of two in [1, 64]");
        tileCodes = (int)v;
    }
    else if (key == "deposit_threads") {
        if (v != 0 && (v < 64 || v > 512 || v % 32)) fail(TILD_ERR_ARG, "deposit_threads must be 0 or a multiple of 32 in [64, 512]");
        depositThreads = (int)v;
    }
    else if (key == "gather_threads") {
        if (v != 0 && (v < 64 || v > 448 || v % 32)) fail(TILD_ERR_ARG, "gather_threads must be 0 or a multiple of 32 in [64, 448]");
        gatherThreads = (int)v;
    }
    else if (key == "sort_interval") {
        if (v < 0) fail(TILD_ERR_ARG, "sort_interval must be >= 0");
        sortInterval = (int)v;
    }
    else fail(TILD_ERR_ARG, "unknown option '" + key + "'");
}

// ---------------------------------------------------------------------------------------
// Script grammar
// ---------------------------------------------------------------------------------------
void Box::command(const std::string &line)
{
    if (ready) fail(TILD_ERR_STATE, "box is already initialised (endBox was seen)");
    if (line.empty() || line[0] == '#') return;   // PS_Box_initialization.cu:71-72
    std::vector<std::string> w = split(line);
    size_t i = 0;
    while (i < w.size()) parseWords(w, i);
}

void Box::parseWords(std::vector<std::string> &w, size_t &i)
{
    const std::string fw = w[i++];
    if (fw == "endBox") {
        i = w.size();
        finishInitialization();
        return;
    }
    if (fw == "angle") {   // PS_Box_initialization.cu:83-106
        const int at = (int)inum(w, i, "angle type");
        if (at < 1 || at > kMaxAngleTypes) fail(TILD_ERR_UNSUPPORTED, "angle type out of range");
        if (at > (int)angleK.size()) {
            angleK.resize(at, 0.f);
            angleTheq.resize(at, 0.f);
            angleStyle.resize(at, 0);
        }
        const std::string style = need(w, i, "angle style");
        angleK[at - 1] = (float)dnum(w, i, "angle k");
        if (style == "wlc") {
            angleStyle[at - 1] = 0;
        } else if (style == "harmonic") {
            angleStyle[at - 1] = 1;
            angleTheq[at - 1] = (float)(dnum(w, i, "angle theta") * (3.14159265358979323846 / 180.0));
        } else {
            fail(TILD_ERR_PARSE, "Angle style not supported!");
        }
    } else if (fw == "MAXANGLES") {
        if (nstot > 0) fail(TILD_ERR_PARSE, "MAXANGLES must be set before defining any molecules");
        MAXANGLES = (int)inum(w, i, "MAXANGLES");
        if (MAXANGLES < 1 || MAXANGLES > 255) fail(TILD_ERR_PARSE, "MAXANGLES out of range");
    } else if (fw == "blocksize" || fw == "blockSize") {
        blockSize = (int)inum(w, i, "blockSize");
    } else if (fw == "bond") {
        const long long bt = inum(w, i, "bond type");
        if (bt < 1 || bt > kMaxBondTypes) fail(TILD_ERR_PARSE, "bond type out of range (1.." + std::to_string(kMaxBondTypes) + ")");
        if ((size_t)bt > bondK.size()) {
            bondK.resize(bt, 0.f);
            bondReq.resize(bt, 0.f);
            bondStyle.resize(bt, 0);
        }
        const std::string style = need(w, i, "bond style");
        bondK[bt - 1] = fnum(w, i, "bond k");
        bondReq[bt - 1] = fnum(w, i, "bond r_eq");
        if (style == "harmonic") bondStyle[bt - 1] = 0;
        else if (style == "fene" || style == "FENE") bondStyle[bt - 1] = 1;
        else fail(TILD_ERR_PARSE, "Bond type not supported!");
        nBondTypes = (int)bondK.size();
    } else if (fw == "boxLengths") {
        if (!readDimension) fail(TILD_ERR_PARSE, "boxLengths read before Dim was specified");
        for (int j = 0; j < Dim; j++) L[j] = fnum(w, i, "boxLengths");
    } else if (fw == "compute") {
        fail(TILD_ERR_UNSUPPORTED, "compute is outside the TILD step (avg_sk is never initialised in the reference)");
    } else if (fw == "datFileName" || fw == "dat_file_name") {
        datFileName = need(w, i, "datFileName");
    } else if (fw == "Dim") {
        Dim = (int)inum(w, i, "Dim");
        if (Dim != 2 && Dim != 3) fail(TILD_ERR_PARSE, "Dim must be 2 or 3");
        readDimension = true;
    } else if (fw == "doCharges") {
        if (!doCharges) {
            doCharges = true;
            if (nstot > 0) charges.assign(nstot, 0.f);
        }
    } else if (fw == "fieldFreq" || fw == "field_freq") {   // PS_Box_initialization.cu:171-183
        fieldFreq = (int)inum(w, i, fw.c_str());
        if (i < w.size()) {
            const std::string t = need(w, i, "logspace");
            if (t != "logspace" && t != "log_space" && t != "logSpace")
                fail(TILD_ERR_PARSE, "invalid option to " + fw);
            logSpaceFields = true;
            logScaleFields = fnum(w, i, "log scale");
        }
    } else if (fw == "gsdFreq" || fw == "gsd_freq") {   // PS_Box_initialization.cu:200-211
        gsdFreq = (int)inum(w, i, fw.c_str());
        if (i < w.size()) {
            const std::string t = need(w, i, "logspace");
            if (t != "logspace" && t != "log_space" && t != "logSpace")
                fail(TILD_ERR_PARSE, "invalid option to " + fw);
            logSpaceGSD = true;
            logScaleGSD = fnum(w, i, "log scale");
        }
    } else if (fw == "grid") {
        if (!readDimension) fail(TILD_ERR_PARSE, "Dim must be defined before grid!");
        for (int j = 0; j < Dim; j++) Nx[j] = (int)inum(w, i, "grid");
    } else if (fw == "group") {
        PS_Group g;
        g.name = need(w, i, "group name");
        const std::string s1 = need(w, i, "group style");
        if (s1 != "types") fail(TILD_ERR_UNSUPPORTED, "group style '" + s1 + "' (only 'types')");
        std::vector<int> tids;
        while (i < w.size()) tids.push_back(findSpeciesInteger(w[i++]));
        for (int64_t p = 0; p < nstot; p++)
            if (std::find(tids.begin(), tids.end(), intSpecies[p]) != tids.end()) g.siteList.push_back((int)p);
        g.inputCommand = "group " + g.name;
        psGroup.push_back(g);
    } else if (fw == "gsdName" || fw == "gsd_name") {   // PS_Box_initialization.cu:213-215
        gsdName = need(w, i, fw.c_str());
    } else if (fw == "trajFileName") {   // PS_Box_initialization.cu:310-312
        trajFileName = need(w, i, fw.c_str());
    } else if (fw == "integrator") {
        Integrator in;
        in.groupName = need(w, i, "integrator group");
        in.name = need(w, i, "integrator name");
        if (i < w.size()) {
            const std::string kw = need(w, i, "integrator option");
            if (kw == "delt") in.delt = fnum(w, i, "delt");
            else fail(TILD_ERR_PARSE, "Invalid keyword in Integrator command");
        }
        if (in.name == "VV") fail(TILD_ERR_UNSUPPORTED, "integrator VV is outside the TILD step (GJF, EM)");
        if (in.name != "GJF" && in.name != "EM") fail(TILD_ERR_PARSE, in.name + " is not a valid Integrator");
        integrators.push_back(in);
    } else if (fw == "initDataFileName") {
        initDataFileName = need(w, i, "initDataFileName");
    } else if (fw == "logFreq" || fw == "logfreq") {
        logFreq = (int)inum(w, i, "logFreq");
        if (logFreq <= 0) fail(TILD_ERR_PARSE, "logFreq must be positive");
    } else if (fw == "MAXBONDS") {
        if (nstot > 0) fail(TILD_ERR_PARSE, "MAXBONDS must be set before defining any molecules");
        MAXBONDS = (int)inum(w, i, "MAXBONDS");
        if (MAXBONDS < 1 || MAXBONDS > 255) fail(TILD_ERR_PARSE, "MAXBONDS out of range");
    } else if (fw == "molecule") {   // :239-251
        const std::string kind = need(w, i, "molecule type");
        if (kind == "linear") makeLinear(w, i);
        else if (kind == "grafted" || kind == "sclc")
            fail(TILD_ERR_UNSUPPORTED, "molecule " + kind + " is outside the TILD step; use readData");
        else fail(TILD_ERR_PARSE, "PS_Box_init:readInput: invalid molecule type read");
    } else if (fw == "Nr") {
        Nr = (int)inum(w, i, "Nr");
    } else if (fw == "NSEXTRA" || fw == "nsextra") {
        NSEXTRA = (int)inum(w, i, "NSEXTRA");
    } else if (fw == "Nx") {
        Nx[0] = (int)inum(w, i, "Nx");
    } else if (fw == "Ny") {
        Nx[1] = (int)inum(w, i, "Ny");
    } else if (fw == "Nz") {
        if (Dim != 3) fail(TILD_ERR_PARSE, "Nz supplied in a non-3D simulation!");
        Nx[2] = (int)inum(w, i, "Nz");
    } else if (fw == "pmeorder") {
        pmeorder = (int)inum(w, i, "pmeorder");
        if (pmeorder < 0 || pmeorder > 4) fail(TILD_ERR_PARSE, "pmeorder must be 0..4");
    } else if (fw == "potential") {
        addPotential(w, i);
    } else if (fw == "neighbor_list") {
        fail(TILD_ERR_UNSUPPORTED, "neighbor_list is only used by DPD, outside the TILD step");
    } else if (fw == "randSeed" || fw == "RAND_SEED" || fw == "RANDSEED") {
        RANDSEED = inum(w, i, "randSeed");   // seeds both the host and the device generators (:291-293)
        idum = RANDSEED;
    } else if (fw == "readData") {
        readDataConfig(need(w, i, "readData file"));
    } else if (fw == "rho0") {
        rho0 = dnum(w, i, "rho0");
    } else if (fw == "species") {
        if (i >= w.size()) fail(TILD_ERR_PARSE, "Missing label for species");
        PS_Species s;
        s.label = w[i++];
        while (i < w.size()) {   // ps_species.cu:28-37 consumes the rest of the line
            const std::string word = w[i++];
            if (word == "mass" || word == "Mass") s.mass = fnum(w, i, "mass");
            else if (word == "mobility" || word == "Mobility" || word == "Diffusivity" || word == "diffusivity")
                s.mobility = fnum(w, i, "mobility");
        }
        if ((int)species.size() >= kMaxTypes) fail(TILD_ERR_UNSUPPORTED, "too many species");
        species.push_back(s);
    } else if (fw == "trajFreq" || fw == "traj_freq") {   // PS_Box_initialization.cu:314-316
        trajFreq = (int)inum(w, i, "trajFreq");
    } else if (fw == "verbose") {
        verbose = inum(w, i, "verbose") != 0;
    } else {
        fail(TILD_ERR_PARSE, "Invalid keyword " + fw + " in PS_Box::readInput()");
    }
}

void Box::addPotential(std::vector<std::string> &w, size_t &i)
{
    PS_Potential p;
    p.word = need(w, i, "potential kind");
    auto ramp_check = [&](PS_Potential &q) {   // ps_potential.cu:253-283
        if (i >= w.size()) return;
        const std::string conv = w[i++];
        if (conv != "ramp") fail(TILD_ERR_PARSE, "Invalid keyword: " + conv);
        if (i >= w.size()) fail(TILD_ERR_PARSE, "no final prefactor specified");
        q.ramp = true;
        q.Ao_final = fnum(w, i, "ramp final prefactor");
        q.Ao_initial = q.Ao;
    };
    if (p.word == "gaussian") {                  // ps_potentialGaussian.cu:14-26
        p.kind = POT_GAUSSIAN;
        p.grpI = need(w, i, "grpI");
        p.grpJ = need(w, i, "grpJ");
        p.Ao = fnum(w, i, "amplitude");
        p.sigma = fnum(w, i, "sigma");
        ramp_check(p);
    } else if (p.word == "erf2" || p.word == "erfG") {   // ps_potentialErf2.cu:85-96
        p.kind = p.word == "erf2" ? POT_ERF2 : POT_ERFG;
        p.grpI = need(w, i, "grpI");
        p.grpJ = need(w, i, "grpJ");
        p.Ao = fnum(w, i, "amplitude");
        p.Rp = fnum(w, i, "Rp");
        p.sigma = fnum(w, i, "sigma");
        ramp_check(p);
    } else if (p.word == "charges") {            // ps_potentialCharges.cu:217-226
        p.kind = POT_CHARGES;
        p.grpI = p.grpJ = "charges";
        p.LB = fnum(w, i, "Bjerrum length");
        p.sigma = fnum(w, i, "sigma");
    } else if (p.word == "wall") {                // ps_potentialWall.cu:11-46
        p.kind = POT_WALL;
        p.grpI = p.grpJ = need(w, i, "wall group");
        const std::string axis = need(w, i, "wall axis");
        if (axis == "x" || axis == "X") p.wallAxis = 0;
        else if (axis == "y" || axis == "Y") p.wallAxis = 1;
        else if (axis == "z" || axis == "Z") p.wallAxis = 2;
        else fail(TILD_ERR_PARSE, "ps_potentialWall.cu: axis must be x, y, or z (got '" + axis + "')");
        if (p.wallAxis >= Dim)
            fail(TILD_ERR_PARSE, "ps_potentialWall.cu: requested wall normal '" + axis + "' but box is only " +
                                     std::to_string(Dim) + "-dimensional");
        p.wallPos = fnum(w, i, "wall position");
        p.wallSign = (int)inum(w, i, "wall side");
        if (p.wallSign != 1 && p.wallSign != -1)
            fail(TILD_ERR_PARSE, "ps_potentialWall.cu: dirSign must be +1 or -1 (got " + std::to_string(p.wallSign) + ")");
        p.wallK = fnum(w, i, "wall k");
        if (i < w.size()) {   // ramp_check_input(iss, -1)
            if (w[i] == "ramp") fail(TILD_ERR_PARSE, "ramping applied on an unsupported potential!");
            fail(TILD_ERR_PARSE, "Invalid keyword: " + w[i]);
        }
        int nw = 0;
        for (auto &q : potentials) nw += q.kind == POT_WALL;
        if (nw >= kMaxWalls) fail(TILD_ERR_UNSUPPORTED, "more than " + std::to_string(kMaxWalls) + " walls");
    } else if (p.word == "bias" || p.word == "bias_lc" || p.word == "Langevin" || p.word == "langevin" ||
               p.word == "dpd" || p.word == "maiersaupe") {
        fail(TILD_ERR_UNSUPPORTED, "potential " + p.word + " is outside the TILD step");
    } else {
        fail(TILD_ERR_PARSE, "ps_potential.cu: " + p.word + " is not a supported potential");
    }
    if ((int)potentials.size() >= kMaxPots) fail(TILD_ERR_UNSUPPORTED, "too many potentials");
    p.amp_eff = p.Ao;
    potentials.push_back(p);
}

int Box::findSpeciesInteger(const std::string &name) const
{
    for (size_t k = 0; k < species.size(); k++)
        if (species[k].label == name) return (int)k;
    fail(TILD_ERR_PARSE, "Species label: " + name + " not found!");
}

int Box::findGroupInteger(const std::string &name) const
{
    for (size_t k = 0; k < psGroup.size(); k++)
        if (psGroup[k].name == name) return (int)k;
    fail(TILD_ERR_PARSE, "PS_Box.cu: Group label not found: " + name);
}

// ---------------------------------------------------------------------------------------
// Particles and the LAMMPS-style data file
// ---------------------------------------------------------------------------------------
void Box::readDataConfig(const std::string &name)
{
    if (nstot != 0) fail(TILD_ERR_PARSE, "Must read data file before making additional molecules");
    if (!readDimension) fail(TILD_ERR_PARSE, "Dim must be defined before readData");
    std::ifstream in(resolve(name));
    if (!in) fail(TILD_ERR_IO, "Failed to open " + name);
    std::vector<std::string> lines;
    std::string ln;
    while (std::getline(in, ln)) lines.push_back(ln);
    int64_t natoms = -1, nbonds = 0, nangles = 0;
    int ntypes = 0;
    size_t k = 1;   // first line is the title (PS_Box_initialization.cu:805)
    auto has = [](const std::string &s, const char *kw) { return s.find(kw) != std::string::npos; };
    float Lread[3] = {0, 0, 1.0f};
    for (; k < lines.size(); k++) {
        const std::string &s = lines[k];
        std::istringstream iss(s);
        if (has(s, "xlo xhi") || has(s, "ylo yhi") || has(s, "zlo zhi")) {
            float lo, hi;
            iss >> lo >> hi;
            const int d = has(s, "xlo") ? 0 : has(s, "ylo") ? 1 : 2;
            Lread[d] = (float)(hi - lo);
        } else if (has(s, "atom types")) iss >> ntypes;
        else if (has(s, "bond types")) { int t; iss >> t; }
        else if (has(s, "angle types")) { int t; iss >> t; }
        else if (has(s, "atoms")) iss >> natoms;
        else if (has(s, "bonds")) iss >> nbonds;
        else if (has(s, "angles")) iss >> nangles;
        else if (has(s, "Masses") || has(s, "Atoms")) break;
    }
    if (natoms <= 0) fail(TILD_ERR_PARSE, "data file " + name + ": no atom count");
    L[0] = Lread[0];
    L[1] = Lread[1];
    L[2] = Dim > 2 ? Lread[2] : 1.0f;
    auto seek = [&](const char *kw) -> bool {
        for (; k < lines.size(); k++) {
            std::string t = lines[k];
            t.erase(0, t.find_first_not_of(" \t"));
            if (t.rfind(kw, 0) == 0) { k++; return true; }
        }
        return false;
    };
    auto next_data = [&]() -> const std::string & {
        while (k < lines.size() && lines[k].find_first_not_of(" \t\r") == std::string::npos) k++;
        if (k >= lines.size()) fail(TILD_ERR_PARSE, "Premature end of " + name);
        return lines[k++];
    };
    const size_t kSave = k;
    if (seek("Masses")) {
        for (int t = 0; t < ntypes; t++) {
            std::istringstream iss(next_data());
            int di;
            float m;
            iss >> di >> m;
            if (di < 1 || di > (int)species.size())
                fail(TILD_ERR_PARSE, "data file type " + std::to_string(di) + " has no declared species (declare species before readData)");
            species[di - 1].mass = m;   // :850-853
        }
    } else {
        k = kSave;
    }
    if (!seek("Atoms")) fail(TILD_ERR_PARSE, "data file " + name + ": no Atoms section");
    nstot = natoms;
    x.assign(nstot * Dim, 0.f);
    intSpecies.assign(nstot, 0);
    mID.assign(nstot, 0);
    if (doCharges) charges.assign(nstot, 0.f);
    for (int64_t a = 0; a < nstot; a++) {
        std::istringstream iss(next_data());
        long long ind, di, ltp;
        if (!(iss >> ind >> di >> ltp)) fail(TILD_ERR_PARSE, "bad atom line in " + name);
        ind -= 1;
        if (ind < 0 || ind >= nstot) fail(TILD_ERR_PARSE, "atom id out of range in " + name);
        if (ltp < 1 || ltp > (long long)species.size())
            fail(TILD_ERR_PARSE, "atom type " + std::to_string(ltp) + " has no declared species");
        mID[ind] = (int)(di - 1);
        intSpecies[ind] = (int)(ltp - 1);
        if (doCharges) iss >> charges[ind];
        for (int j = 0; j < Dim; j++)
            if (!(iss >> x[ind * Dim + j])) fail(TILD_ERR_PARSE, "bad coordinates in " + name);
    }
    nBonds.assign(nstot, 0);
    bondedTo.assign(nstot * MAXBONDS, 0);
    bondType.assign(nstot * MAXBONDS, 0);
    nAngles.assign(nstot, 0);
    angleGroup.assign(nstot * MAXANGLES * 3, 0);
    angleType.assign(nstot * MAXANGLES, 0);
    nAnglesTot = 0;
    angleList.clear();
    if (nbonds > 0) {
        if (!seek("Bonds")) fail(TILD_ERR_PARSE, "data file " + name + ": no Bonds section");
        std::vector<int64_t> pairs(2 * nbonds);
        std::vector<int32_t> bt(nbonds);
        for (int64_t b = 0; b < nbonds; b++) {
            std::istringstream iss(next_data());
            long long id, t, i1, i2;
            if (!(iss >> id >> t >> i1 >> i2)) fail(TILD_ERR_PARSE, "bad bond line in " + name);
            pairs[2 * b] = i1 - 1;
            pairs[2 * b + 1] = i2 - 1;
            bt[b] = (int32_t)(t - 1);
        }
        setBonds(nbonds, pairs.data(), bt.data());
    }
    if (nangles > 0) {   // :933-993
        if (!seek("Angles")) fail(TILD_ERR_PARSE, "data file " + name + ": no Angles section");
        std::vector<int64_t> tri(3 * nangles);
        std::vector<int32_t> at(nangles);
        for (int64_t a = 0; a < nangles; a++) {
            std::istringstream iss(next_data());
            long long id, t, i1, i2, i3;
            if (!(iss >> id >> t >> i1 >> i2 >> i3)) fail(TILD_ERR_PARSE, "bad angle line in " + name);
            tri[3 * a] = i1 - 1;
            tri[3 * a + 1] = i2 - 1;
            tri[3 * a + 2] = i3 - 1;
            at[a] = (int32_t)(t - 1);
        }
        setAngles(nangles, tri.data(), at.data());
    }
}

void Box::setParticles(int64_t n, const float *xin, const int32_t *type, const int32_t *mol, const float *q)
{
    if (ready) fail(TILD_ERR_STATE, "particles must be set before endBox");
    if (nstot != 0) fail(TILD_ERR_PARSE, "particles were already defined");
    if (!readDimension) fail(TILD_ERR_PARSE, "Dim must be defined before particles");
    if (n <= 0 || !xin || !type) fail(TILD_ERR_ARG, "particles need n > 0, x and type");
    if (doCharges && !q) fail(TILD_ERR_ARG, "doCharges is set: charges are required");
    nstot = n;
    x.assign(xin, xin + n * Dim);
    intSpecies.assign(type, type + n);
    for (int64_t p = 0; p < n; p++)
        if (intSpecies[p] < 0 || intSpecies[p] >= (int)species.size())
            fail(TILD_ERR_ARG, "particle type has no declared species");
    mID.assign(n, 0);
    if (mol) mID.assign(mol, mol + n);
    if (doCharges) charges.assign(q, q + n);
    nBonds.assign(nstot, 0);
    bondedTo.assign(nstot * MAXBONDS, 0);
    bondType.assign(nstot * MAXBONDS, 0);
    nAngles.assign(nstot, 0);
    angleGroup.assign(nstot * MAXANGLES * 3, 0);
    angleType.assign(nstot * MAXANGLES, 0);
    nAnglesTot = 0;
    angleList.clear();
}

// ---- host random numbers (random.cu) -------------------------------------------------
// Uniform deviate in (0, 1): L'Ecuyer's (1988) combination of two multiplicative LCGs
// (m1 = 2147483563, a1 = 40014; m2 = 2147483399, a2 = 40692; products by Schrage's
// decomposition) passed through a Bays-Durham shuffle of 32 entries, results capped at
// 1 - 1.2e-7.  A seed <= 0 fills the table first; a positive seed (what randSeed and the
// time-based default give) starts from the empty table with the second generator at
// 123456789, as the reference's static state does.
double Box::ran2()
{
    constexpr int64_t M1 = 2147483563, M2 = 2147483399, A1 = 40014, A2 = 40692;
    constexpr int64_t Q1 = 53668, Q2 = 52774, R1 = 12211, R2 = 3791;   // m = a q + r
    constexpr int NT = 32;
    constexpr int64_t NDIV = 1 + (M1 - 1) / NT;
    constexpr double AM = 1.0 / M1, RNMX = 1.0 - 1.2e-7;
    auto lcg1 = [&](int64_t &v) {
        const int64_t k = v / Q1;
        v = A1 * (v - k * Q1) - k * R1;
        if (v < 0) v += M1;
    };
    if (idum <= 0) {
        idum = (-idum < 1) ? 1 : -idum;
        idum2 = idum;
        for (int j = NT + 7; j >= 0; j--) {
            lcg1(idum);
            if (j < NT) iv[j] = idum;
        }
        iy = iv[0];
    }
    lcg1(idum);
    const int64_t k = idum2 / Q2;
    idum2 = A2 * (idum2 - k * Q2) - k * R2;
    if (idum2 < 0) idum2 += M2;
    const int j = (int)(iy / NDIV);
    iy = iv[j] - idum2;
    iv[j] = idum;
    if (iy < 1) iy += M1 - 1;
    const double t = AM * (double)iy;
    return t > RNMX ? RNMX : t;
}

// Normal deviate by the polar Box-Muller method, two per accepted pair (the second kept
// for the next call).
double Box::gasdev2()
{
    if (gasIset) {
        gasIset = 0;
        return gasGset;
    }
    double v1, v2, rsq;
    do {
        v1 = 2.0 * ran2() - 1.0;
        v2 = 2.0 * ran2() - 1.0;
        rsq = v1 * v1 + v2 * v2;
    } while (rsq >= 1.0 || rsq == 0.0);
    const double fac = std::sqrt(-2.0 * std::log(rsq) / rsq);
    gasGset = v1 * fac;
    gasIset = 1;
    return v2 * fac;
}

// Isotropic unit vector: normalised vector of normal deviates.
void Box::randomUnitVec(double *v, int dim)
{
    double xi[3], m2 = 0.0;
    for (int k = 0; k < dim; k++) {
        xi[k] = gasdev2();
        m2 += xi[k] * xi[k];
    }
    const double m = std::sqrt(m2);
    for (int k = 0; k < dim; k++) v[k] = xi[k] / m;
}

// molecule linear {phi F | nmolecs n} nblocks (N_b species_b)... [charge q_b...]
// [bondType t_b...] [angleType t_b...] [xrange lo hi] [yrange lo hi] [zrange lo hi]
// (PS_Box_moleculeMakers.cu:15-311): chains whose first bead is uniform in the range and
// whose next beads sit a unit step from the previous one (a fresh random direction per
// step, or per chain when the chain carries angles), wrapped into the box; bonds along
// the chain with the block's bond type on each side, angles on interior beads of blocks
// with an angle type.
void Box::makeLinear(std::vector<std::string> &w, size_t &i)
{
    if (rho0 < 0.0) fail(TILD_ERR_PARSE, "rho0 must be defined before molecules created!");
    if (!readDimension) fail(TILD_ERR_PARSE, "Dim must be defined before molecules");
    double phi = -1.0;
    int64_t nmolecs = -1;
    const std::string s1 = need(w, i, "molecule linear phi|nmolecs");
    if (s1 == "phi") phi = dnum(w, i, "phi");
    else if (s1 == "nmolecs") nmolecs = inum(w, i, "nmolecs");
    else fail(TILD_ERR_PARSE, "invalid keyword after molecule linear. must be 'phi' or 'nmolecs'");
    const int nblk = (int)inum(w, i, "number of blocks");
    if (nblk < 1) fail(TILD_ERR_PARSE, "a linear molecule needs at least one block");
    std::vector<int> nper(nblk), spec(nblk), bt(nblk, 1), at(nblk, 0);
    std::vector<float> bq(nblk, 0.f);
    int ntot = 0;
    for (int b = 0; b < nblk; b++) {
        nper[b] = (int)inum(w, i, "block length");
        spec[b] = findSpeciesInteger(need(w, i, "block species"));
        ntot += nper[b];
    }
    bool molQ = false, angles = false;
    float rmin[3] = {0.f, 0.f, 0.f}, rmax[3] = {L[0], L[1], L[2]};
    while (i < w.size()) {
        const std::string o = w[i++];
        if (o == "drude") {
            fail(TILD_ERR_UNSUPPORTED, "drude oscillators not implemented!");
        } else if (o == "charge") {
            if (!doCharges) {   // enableCharges (PS_Box_initialization.cu:1000-1010)
                doCharges = 1;
                charges.assign(nstot, 0.f);
            }
            molQ = true;
            for (int b = 0; b < nblk; b++) bq[b] = (float)dnum(w, i, "block charge");
        } else if (o == "bondType" || o == "bondtype") {
            for (int b = 0; b < nblk; b++) bt[b] = (int)inum(w, i, "block bond type");
        } else if (o == "angleType" || o == "angletype") {
            for (int b = 0; b < nblk; b++) at[b] = (int)inum(w, i, "block angle type");
            angles = true;
        } else if (o == "xrange" || o == "yrange" || o == "zrange") {
            const int d = o[0] - 'x';
            if (d == 2 && Dim != 3) fail(TILD_ERR_PARSE, "z-range defined for a non-3D simulation!");
            rmin[d] = (float)dnum(w, i, "range low");
            rmax[d] = (float)dnum(w, i, "range high");
        } else {
            fail(TILD_ERR_PARSE, "invalid keyword " + o + " in molecule linear");
        }
    }
    double V = 1.0;   // as PS_Box_initialization.cu:143-146 accumulates it
    for (int j = 0; j < Dim; j++) V *= L[j];
    if (phi > 0.0) nmolecs = (int64_t)(int)(rho0 * V * phi / (double)(float)ntot);
    if (nmolecs < 0) fail(TILD_ERR_PARSE, "molecule linear: no molecules to make");
    const int64_t first = nstot, n = nstot + nmolecs * ntot;
    x.resize(n * Dim, 0.f);
    intSpecies.resize(n, 0);
    mID.resize(n, 0);
    if (doCharges) charges.resize(n, 0.f);
    nBonds.resize(n, 0);
    bondedTo.resize(n * MAXBONDS, 0);
    bondType.resize(n * MAXBONDS, 0);
    nAngles.resize(n, 0);
    angleGroup.resize(n * MAXANGLES * 3, 0);
    angleType.resize(n * MAXANGLES, 0);
    nstot = n;
    int mol = 0;   // starting molecule id: the largest so far (:140-146)
    for (int64_t p = 0; p < first; p++) mol = std::max(mol, mID[p]);
    int64_t ind = first;
    for (int64_t m = 0; m < nmolecs; m++) {
        double ru[3] = {0.0, 0.0, 0.0};
        for (int b = 0; b < nblk; b++) {
            for (int s = 0; s < nper[b]; s++) {
                intSpecies[ind] = spec[b];
                if (b == 0 && s == 0) {
                    for (int a = 0; a < Dim; a++) x[ind * Dim + a] = (float)(ran2() * (rmax[a] - rmin[a]) + rmin[a]);
                } else {
                    if ((s == 1 && b == 0) || !angles) randomUnitVec(ru, Dim);
                    for (int a = 0; a < Dim; a++) {
                        float v = (float)(x[(ind - 1) * Dim + a] + ru[a]);
                        if (v > L[a]) v -= L[a];
                        else if (v < 0.0f) v += L[a];
                        x[ind * Dim + a] = v;
                    }
                }
                if (molQ) charges[ind] = bq[b];
                nBonds[ind] = 0;
                if (b != 0 || s != 0) {
                    bondedTo[ind * MAXBONDS + nBonds[ind]] = (int)(ind - 1);
                    bondType[ind * MAXBONDS + nBonds[ind]] = bt[b] - 1;
                    nBonds[ind]++;
                }
                if (b != nblk - 1 || s != nper[b] - 1) {
                    if (nBonds[ind] >= MAXBONDS) fail(TILD_ERR_PARSE, "MAXBONDS too small for linear molecules");
                    bondedTo[ind * MAXBONDS + nBonds[ind]] = (int)(ind + 1);
                    bondType[ind * MAXBONDS + nBonds[ind]] = bt[b] - 1;
                    nBonds[ind]++;
                }
                if (at[b] != 0 && (b > 0 || s > 0) && (b < nblk - 1 || s < nper[b] - 1)) {
                    const int64_t tri[3] = {ind - 1, ind, ind + 1};
                    for (int64_t p : tri) {
                        const int k = nAngles[p];
                        if (k >= MAXANGLES)
                            fail(TILD_ERR_PARSE, "a particle has more than MAXANGLES=" + std::to_string(MAXANGLES) + " angles");
                        for (int r = 0; r < 3; r++) angleGroup[(p * MAXANGLES + k) * 3 + r] = (int)tri[r];
                        angleType[p * MAXANGLES + k] = at[b] - 1;
                        nAngles[p] = k + 1;
                    }
                    nAnglesTot++;
                }
                mID[ind] = mol;
                ind++;
            }
        }
        mol++;
    }
}

// Angles as 0-based particle triples (i1, i2 middle, i3) and 0-based types; the ends are
// ordered i1 < i3 and the angle is stored on all three particles (:947-983).
void Box::setAngles(int64_t na, const int64_t *tri, const int32_t *atype)
{
    if (ready) fail(TILD_ERR_STATE, "angles must be set before endBox");
    if (nstot == 0) fail(TILD_ERR_STATE, "angles need particles");
    if (na < 0 || (na > 0 && !tri)) fail(TILD_ERR_ARG, "bad angle arrays");
    for (int64_t a = 0; a < na; a++) {
        int64_t i1 = tri[3 * a], i2 = tri[3 * a + 1], i3 = tri[3 * a + 2];
        if (i1 < 0 || i2 < 0 || i3 < 0 || i1 >= nstot || i2 >= nstot || i3 >= nstot)
            fail(TILD_ERR_PARSE, "angle particle out of range");
        if (i3 < i1) std::swap(i1, i3);
        const int t = atype ? atype[a] : 0;
        if (t < 0 || t >= kMaxAngleTypes) fail(TILD_ERR_PARSE, "angle type out of range");
        for (int64_t p : {i1, i2, i3}) {
            const int k = nAngles[p];
            if (k >= MAXANGLES)
                fail(TILD_ERR_PARSE, "a particle has more than MAXANGLES=" + std::to_string(MAXANGLES) + " angles");
            angleGroup[(p * MAXANGLES + k) * 3 + 0] = (int)i1;
            angleGroup[(p * MAXANGLES + k) * 3 + 1] = (int)i2;
            angleGroup[(p * MAXANGLES + k) * 3 + 2] = (int)i3;
            angleType[p * MAXANGLES + k] = t;
            nAngles[p] = k + 1;
        }
        angleList.insert(angleList.end(), {(uint32_t)t, (uint32_t)i1, (uint32_t)i2, (uint32_t)i3});
    }
    nAnglesTot += (int)na;
}

void Box::setBonds(int64_t nb, const int64_t *pairs, const int32_t *btype)
{
    if (ready) fail(TILD_ERR_STATE, "bonds must be set before endBox");
    if (nstot == 0) fail(TILD_ERR_STATE, "bonds need particles");
    if (nb < 0 || (nb > 0 && !pairs)) fail(TILD_ERR_ARG, "bad bond arrays");
    for (int64_t b = 0; b < nb; b++) {   // PS_Box_initialization.cu:897-926
        int64_t i1 = pairs[2 * b], i2 = pairs[2 * b + 1];
        if (i1 < 0 || i2 < 0 || i1 >= nstot || i2 >= nstot) fail(TILD_ERR_PARSE, "bond partner out of range");
        if (i2 < i1) std::swap(i1, i2);
        const int t = btype ? btype[b] : 0;
        if (t < 0 || t >= kMaxBondTypes) fail(TILD_ERR_PARSE, "bond type out of range");
        if (nBonds[i1] >= MAXBONDS || nBonds[i2] >= MAXBONDS)
            fail(TILD_ERR_PARSE, "a particle has more than MAXBONDS=" + std::to_string(MAXBONDS) + " bonds");
        bondedTo[i1 * MAXBONDS + nBonds[i1]] = (int)i2;
        bondType[i1 * MAXBONDS + nBonds[i1]] = t;
        nBonds[i1]++;
        bondedTo[i2 * MAXBONDS + nBonds[i2]] = (int)i1;
        bondType[i2 * MAXBONDS + nBonds[i2]] = t;
        nBonds[i2]++;
    }
}

void Box::createDefaultGroups()
{
    PS_Group all;
    all.name = "all";
    all.inputCommand = "group all";
    all.siteList.resize(nstot);
    std::iota(all.siteList.begin(), all.siteList.end(), 0);
    psGroup.push_back(all);
    for (size_t t = 0; t < species.size(); t++) {
        PS_Group g;
        g.name = species[t].label;
        g.inputCommand = "group type " + std::to_string(t + 1);
        for (int64_t p = 0; p < nstot; p++)
            if (intSpecies[p] == (int)t) g.siteList.push_back((int)p);
        psGroup.push_back(g);
    }
    if (doCharges) {
        PS_Group g;
        g.name = "charges";
        g.inputCommand = "group charges";
        g.isCharges = true;
        for (int64_t p = 0; p < nstot; p++)
            if (charges[p] != 0.0f) g.siteList.push_back((int)p);
        g.forceFlag = true;   // ps_groups.cu:131
        psGroup.push_back(g);
    }
}

// ---------------------------------------------------------------------------------------
// endBox
// ---------------------------------------------------------------------------------------
void Box::finishInitialization()
{
    if (!hostPrepared) prepareHost();
    initDevice();
}

void Box::prepareHost()
{
    if (hostPrepared) return;
    if (nstot == 0) fail(TILD_ERR_PARSE, "Box created with no particles?!?");
    if (Dim != 2 && Dim != 3) fail(TILD_ERR_PARSE, "Dim must be 2 or 3");
    if (Dim == 2) {   // a 2-D box runs as one plane of unit thickness at z = 0
        Nx[2] = 1;
        L[2] = 1.0f;
    }
    for (int j = 0; j < Dim; j++)
        if (Nx[j] <= 0) fail(TILD_ERR_PARSE, "grid must be given for every dimension");
    for (int j = 0; j < Dim; j++)   // the kernels wrap stencil indices with one add or subtract
        if (Nx[j] < pmeorder + 2)
            fail(TILD_ERR_UNSUPPORTED, "grid of " + std::to_string(Nx[j]) + " points is too small for pmeorder " +
                                           std::to_string(pmeorder) + " (needs at least pmeorder + 2)");
    for (int64_t p = 0; p < nstot && nAnglesTot > 0; p++)
        for (int k = 0; k < nAngles[p]; k++)
            if (angleType[p * MAXANGLES + k] >= (int)angleK.size())
                fail(TILD_ERR_PARSE, "angle type " + std::to_string(angleType[p * MAXANGLES + k] + 1) +
                                         " has no 'angle' command");
    if (integrators.empty()) fail(TILD_ERR_PARSE, "no integrator defined");
    if (species.size() > (size_t)kMaxTypes) fail(TILD_ERR_UNSUPPORTED, "too many species");
    gvol = 1.0;
    for (int j = 0; j < Dim; j++) {
        dx[j] = (double)L[j] / (double)Nx[j];
        gvol *= dx[j];
        Lh[j] = 0.5f * L[j];
    }
    if (Dim == 2) {   // the plane's unit thickness: cell volume dx*dy*1, as the 2-D gvol
        dx[2] = 1.0;
        Lh[2] = 0.5f;
    }
    if (doCharges) {   // PS_Box_initialization.cu:398-412
        float qtot = 0.f, qneg = 0.f, qpos = 0.f;
        for (int64_t p = 0; p < nstot; p++) {
            qtot += charges[p];
            if (charges[p] < 0.f) qneg += charges[p];
            else if (charges[p] > 0.f) qpos += charges[p];
        }
        if (qtot != 0.f)
            fail(TILD_ERR_PARSE, "Box net charge is not zero! qtotal: " + std::to_string(qtot) +
                                     "total negative: " + std::to_string(qneg) + ", positive: " + std::to_string(qpos));
    }
    nBondsTot = 0;
    nBondEntries = 0;   // both directions: the length of the device's CSR bond list
    for (int64_t p = 0; p < nstot; p++) {
        nBondEntries += nBonds[p];
        for (int b = 0; b < nBonds[p]; b++)
            if (bondedTo[p * MAXBONDS + b] > p) nBondsTot++;
    }
    for (int64_t p = 0; p < nstot; p++)
        for (int b = 0; b < nBonds[p]; b++)
            if (bondType[p * MAXBONDS + b] >= nBondTypes)
                fail(TILD_ERR_PARSE, "bond type " + std::to_string(bondType[p * MAXBONDS + b] + 1) + " has no 'bond' command");
    if (writeFiles) writeDataConfig(initDataFileName);
    createDefaultGroups();
    for (auto &g : psGroup)
        if (g.siteList.empty()) fail(TILD_ERR_PARSE, "A group with size 0 found, exiting! (group '" + g.name + "')");
    for (auto &in : integrators) in.group_index = findGroupInteger(in.groupName);
    for (auto &p : potentials) {   // PS_Potential::initializePotential (ps_potential.cu:24-33)
        if (p.kind == POT_CHARGES) {
            p.Iind = p.Jind = findGroupInteger("charges");
        } else {
            p.Iind = findGroupInteger(p.grpI);
            p.Jind = findGroupInteger(p.grpJ);
            psGroup[p.Iind].forceFlag = true;
            psGroup[p.Jind].forceFlag = true;
        }
    }
    if (writeFiles) {   // GSDinit + writeGSDtraj (PS_Box_initialization.cu:521-523)
        std::vector<float> x3(3 * nstot, 0.f);
        for (int64_t p = 0; p < nstot; p++)
            for (int j = 0; j < Dim; j++) x3[3 * p + j] = x[p * Dim + j];
        writeGsdFrame(0, x3.data());
    }
    if (writeFiles) initFieldFiles();
    if (writeFiles) { std::ofstream o(resolve(datFileName)); }   // :359-364, :543-544 truncate
    buildPlan();
    hostPrepared = true;
}

void Box::initDevice()
{
    if (!hostPrepared) fail(TILD_ERR_STATE, "the box has not been prepared");
    if (ready) fail(TILD_ERR_STATE, "endBox was already processed");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) fail(TILD_ERR_CUDA, "no CUDA device is visible");
    ck(cudaSetDevice(device), "cudaSetDevice");
    if (!stream) {
        ck(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        ownStream = true;
    }
    init_fft_attributes();
    init_deposit_attributes();
    init_particle_attributes();
    allocDevice();
    uploadParticles();
    if (sortInterval > 0) {   // start from a spatially coherent order
        sortParticles();
        ck(cudaStreamSynchronize(stream), "initial sort");
    }
    if (autotune) autotuneTiles();
    ready = true;
}

// Bricks per tile from the density: about one particle per thread of a 192-thread CTA.
int Box::densityCodes() const
{
    if (tileCodes) return tileCodes;
    const double perCode = 16.0 * std::min(4, geom.nz) * (double)nstot / (double)geom.M;   // particles per brick of 4^3 cells (4x4x1 in 2-D)
    int codes = 8;
    while (codes < 64 && perCode * codes * 2.0 <= 192.0) codes *= 2;
    return codes;
}

// Bytes of the force records: planar, or paired with the ghost layers of any tiles the
// autotuner tries (half, the same and twice the density's bricks).
size_t Box::recordBytes() const
{
    const int nfg = std::max(1, (int)fgroups.size()), codes = densityCodes();
    size_t b = sizeof(float4) * (size_t)nfg * geom.M;
    for (int c : {codes / 2, codes, codes * 2}) {
        const TileCfg t = tileGeometry(c, false);
        if (!t.paired) continue;
        int gl, gh[3];
        pairedGhosts(t, &gl, gh);
        b = std::max(b, rec_layout_bytes(geom, nfg, gl, gh));
    }
    return b;
}

int64_t Box::deviceBytesEstimate() const
{
    if (!hostPrepared) fail(TILD_ERR_STATE, "the box has not been prepared");
    const int64_t N = nstot, M = geom.M, hs = geom.hstride;
    const int64_t nd = std::max<int64_t>(1, (int64_t)dfields.size()), nfg = std::max<int64_t>(1, (int64_t)fgroups.size());
    const int64_t npair = (nd + 1) / 2;
    const int64_t rng = rngCompat ? (int64_t)rng_state_bytes() : 0, q = doCharges ? 4 : 0;
    const int64_t perParticle = 12 * 4 + 4 + 4 + q + rng + 12 + 1   // state, scratch, partials
                                + 12 + 36 + q + 8 + rng + 1;        // sort keys, copies, scan totals
    const int64_t bonds = nBondEntries > 0 ? 2 * (4 * (N + 1) + 5 * nBondEntries) : 0;   // CSR + its sort copy
    const int64_t nk = (int64_t)sort_key_count(geom);
    const int64_t angles = nAnglesTot > 0 ? 2 * (1 + 13 * (int64_t)MAXANGLES) : 0;   // arrays and sort copies
    const int64_t grid = (deterministic ? 16 : 8) * npair * M + 8 * nd * hs + 24 * nfg * hs + (int64_t)recordBytes() +
                         4 * std::max<int64_t>(1, (int64_t)potentials.size()) * hs + 8 * nk;
    return N * (perParticle + angles + 12) + bonds + grid + nk + (int64_t(4) << 20);   // + grid forces, tile lists, small arrays, alignment, graphs
}

void Box::buildPlan()
{
    const int ng = (int)psGroup.size();
    dfields.clear();
    fgroups.clear();
    auto dfield = [&](int grp, int charge) {
        for (size_t k = 0; k < dfields.size(); k++)
            if (dfields[k].group == grp && dfields[k].charge == charge) return (int)k;
        dfields.push_back({grp, charge});
        return (int)dfields.size() - 1;
    };
    // k-space terms; force groups in psGroup order (PS_Box.cu:268-270)
    struct T { int grp; int pot; int df; double mult; };
    std::vector<T> raw;
    for (size_t pi = 0; pi < potentials.size(); pi++) {
        const PS_Potential &p = potentials[pi];
        if (p.kind == POT_WALL) continue;   // a per-particle force, in the particle pass
        if (p.kind == POT_CHARGES) {
            raw.push_back({p.Iind, (int)pi, dfield(p.Iind, 1), 1.0});
        } else {
            raw.push_back({p.Iind, (int)pi, dfield(p.Jind, 0), p.Iind == p.Jind ? 2.0 : 1.0});
            if (p.Iind != p.Jind) raw.push_back({p.Jind, (int)pi, dfield(p.Iind, 0), 1.0});
        }
    }
    for (int gi = 0; gi < ng; gi++)
        for (auto &t : raw)
            if (t.grp == gi && psGroup[gi].forceFlag) { fgroups.push_back(gi); break; }
    if ((int)dfields.size() > kMaxFields) fail(TILD_ERR_UNSUPPORTED, "more than 8 density fields");
    if ((int)fgroups.size() > kMaxFGroups) fail(TILD_ERR_UNSUPPORTED, "more than 4 force groups");
    if ((int)raw.size() > kMaxTerms) fail(TILD_ERR_UNSUPPORTED, "too many k-space terms");

    // geometry
    Geom &g = geom;
    g.nx = Nx[0]; g.ny = Nx[1]; g.nz = Nx[2];
    g.nxh = g.nx / 2 + 1;
    g.hp = (g.nxh + 3) & ~3;
    g.M = (long long)g.nx * g.ny * g.nz;
    if (g.M >= (1ll << 31)) fail(TILD_ERR_UNSUPPORTED, "grids of 2^31 points or more");
    g.hstride = (long long)g.nz * g.ny * g.hp;
    for (int j = 0; j < 3; j++) {
        g.dxf[j] = (float)dx[j];
        g.dlo[j] = (float)(dx[j] - (double)g.dxf[j]);
        g.inv[j] = 1.0f / g.dxf[j];
        g.L[j] = L[j];
        g.Lh[j] = Lh[j];
    }
    // FP32 grid volume of the reference weights (ps_grid_utils.cu:97-101) and the FP64 one
    // of the gathers (ps_groups.cu:186-193): forces scale by gvol_d/(gvol_f^2 M).
    const double gvf = (double)((1.0f * g.dxf[0]) * g.dxf[1] * g.dxf[2]);
    const double norm = gvol / (gvf * gvf * (double)g.M);

    KSpace &ks = ksHost;
    std::memset(&ks, 0, sizeof(ks));
    ks.npots = (int)potentials.size();
    for (size_t pi = 0; pi < potentials.size(); pi++) {
        const PS_Potential &p = potentials[pi];
        PotDev &d = ks.pots[pi];
        d.kind = p.kind;
        d.amp = p.amp_eff;
        d.sig2 = (double)(p.sigma * p.sigma);   // sig2 = sigma*sigma in float
        d.Rp = p.Rp;
        d.lB = p.LB;
        ETerm &e = ks.eterms[pi];
        e.pot = (int)pi;
        if (p.kind == POT_WALL) {   // no k-space energy: the particle reduction gives it
            e.dI = e.dJ = 0;
            e.fac = 0.0;
        } else if (p.kind == POT_CHARGES) {
            e.dI = e.dJ = dfield(p.Iind, 1);
            e.fac = 0.5 * norm;
        } else {
            e.dI = dfield(p.Iind, 0);
            e.dJ = dfield(p.Jind, 0);
            e.fac = norm;
        }
    }
    ks.neterms = (int)potentials.size();
    ks.nterms = 0;
    for (auto &t : raw) {
        int f = -1;
        for (size_t k = 0; k < fgroups.size(); k++)
            if (fgroups[k] == t.grp) f = (int)k;
        if (f < 0) continue;
        ks.terms[ks.nterms++] = KTerm{f, t.pot, t.df, t.mult * norm};
    }
    ks.nfg = (int)fgroups.size();
    ks.nd = (int)dfields.size();
    for (int j = 0; j < 3; j++) ks.twopi_over_L[j] = 2.0 * M_PI / (double)L[j];

    // particle params
    ParticleParams &pp = ppHost;
    std::memset(&pp, 0, sizeof(pp));
    pp.N = (int)nstot;
    pp.order = pmeorder;
    pp.quirk4 = exact4 ? 0 : 1;
    pp.nd = ks.nd;
    pp.npair = (ks.nd + 1) / 2;
    for (size_t k = 0; k < dfields.size(); k++)
        if (dfields[k].charge) pp.dchan_charge |= 1u << k;
    pp.nfg = ks.nfg;
    {   // int32 fixed-point tile sums (2^24 per unit): a grid point of a tile receives at
        // most (particles) x (largest stencil weight) x (largest |q|)
        const double w1[5] = {1.0, 1.0, 0.75, 2.0 / 3.0, 115.0 / 192.0};   // max 1-D weight per order
        double wmax = 1.0;
        for (int j = 0; j < Dim; j++) wmax *= w1[std::min(std::max(pmeorder, 0), 4)];
        double qmax = 1.0;
        if (doCharges)
            for (int64_t p = 0; p < nstot; p++) qmax = std::max(qmax, (double)std::fabs(charges[p]));
        pp.int_tile_max = (int)std::floor(0.9 * 2147483647.0 / (16777216.0 * wmax * qmax));
    }
    for (size_t k = 0; k < fgroups.size(); k++)
        if (psGroup[fgroups[k]].isCharges) pp.fg_qweighted |= 1u << k;
    pp.maxb = MAXBONDS;
    pp.maxa = nAnglesTot > 0 ? MAXANGLES : 0;
    for (size_t t = 0; t < angleK.size() && t < (size_t)kMaxAngleTypes; t++) {
        pp.ak[t] = angleK[t];
        pp.atheq[t] = angleTheq[t];
        pp.astyle[t] = angleStyle[t];
    }
    pp.nbtypes = nBondTypes;
    for (int t = 0; t < nBondTypes; t++) {
        pp.bk[t] = bondK[t];
        pp.breq[t] = bondReq[t];
        pp.bstyle[t] = bondStyle[t];
    }
    if (integrators.size() > 4) fail(TILD_ERR_UNSUPPORTED, "more than 4 integrators");
    for (size_t s = 0; s < integrators.size(); s++) {   // ps_integratorGJF.cu:43-95
        const Integrator &in = integrators[s];
        pp.integ_kind[s] = in.name == "GJF" ? 0 : 1;
        const float delt = in.delt, delt2 = delt * delt, root2dt = sqrtf(2.0f * delt);
        pp.em_delt[s] = delt;
        pp.em_noise[s] = sqrtf((float)(2.0 * (double)delt));   // ps_integratorEM.cu:22-26
        for (size_t t = 0; t < species.size(); t++) {
            const float m = species[t].mass, Di = species[t].mobility;
            const float b = m / (m + delt / (2.0f * Di));
            const float a = (1.0f - delt / (2.0f * Di * m)) / (1.0f + delt / (2.0f * Di * m));
            pp.coef[s][t] = TypeCoef{a, b, root2dt / sqrtf(Di), b * delt2 / m, b * delt / (2.0f * m)};
        }
    }
    pp.seed = (unsigned long long)RANDSEED;
    pp.rng_compat = rngCompat;
    pp.dim = Dim;
    pp.nwall = 0;
    for (const PS_Potential &p : potentials)
        if (p.kind == POT_WALL) {
            const int wi = pp.nwall++;
            pp.wall_axis[wi] = p.wallAxis;
            pp.wall_sign[wi] = p.wallSign;
            pp.wall_pos[wi] = p.wallPos;
            pp.wall_k[wi] = p.wallK;
        }
}

void Box::allocDevice()
{
    const Geom &g = geom;
    const int64_t N = nstot;
    arenaSize = (size_t)deviceBytesEstimate();
    arena = static_cast<char *>(rawAlloc(arenaSize));
    arenaUsed = 0;
    dX[0] = dalloc<float>(3 * N);
    dX[1] = dalloc<float>(3 * N);
    dNoise = dalloc<float>(3 * N);
    dF = dalloc<float>(3 * N);
    dFlags = dalloc<uint32_t>(N);
    dOrig = dalloc<int>(N);
    if (doCharges) dQ = dalloc<float>(N);
    const int64_t nnz = nBondEntries;   // CSR bond list, both directions
    if (nnz > 0) {
        dBrow = dalloc<int>(N + 1);
        dPartner = dalloc<int>(nnz);
        dBtype = dalloc<uint8_t>(nnz);
    }
    if (nAnglesTot > 0) {
        dNa = dalloc<uint8_t>(N);
        dAtype = dalloc<uint8_t>(N * MAXANGLES);
        dAng = dalloc<int>(3 * N * MAXANGLES);
    }
    if (rngCompat) dRng = dalloc<unsigned char>(N * rng_state_bytes());
    const int nd = std::max(1, (int)dfields.size()), nfg = std::max(1, (int)fgroups.size());
    const int npair = (nd + 1) / 2;
    if (deterministic) dDepFix = dalloc<unsigned long long>((size_t)2 * npair * g.M);
    else dDep = dalloc<float2>((size_t)npair * g.M);
    dH = dalloc<float2>((size_t)nd * g.hstride);
    dHg = dalloc<float2>((size_t)3 * nfg * g.hstride);
    dTw = dalloc<float2>((size_t)g.nx + g.ny + g.nz);
    build_fft_line(g.nx, lx, dTw);
    build_fft_line(g.ny, ly, dTw + g.nx);
    build_fft_line(g.nz, lz, dTw + g.nx + g.ny);
    for (FftLine *l : {&lx, &ly, &lz})
        if (l->ns > kMaxStages) fail(TILD_ERR_UNSUPPORTED, "grid size factors into too many stages");
    dStep = dalloc<long long>(1);
    dKs = dalloc<KSpace>(1);
    dUk = dalloc<float>((size_t)std::max<size_t>(1, potentials.size()) * g.hstride);
    dPp = dalloc<ParticleParams>(1);
    const int TXz = kspace_tile_width(g, (int)dfields.size(), (int)fgroups.size(), (int)potentials.size());
    if (TXz == 0) fail(TILD_ERR_UNSUPPORTED, "the grid's z size is too large for the fused k-space pass with this many fields");
    nblkZ = ((g.nxh + TXz - 1) / TXz) * g.ny;
    nblkP = (int)((N + 255) / 256);
    dEpart = dalloc<double>((size_t)nblkZ * (ksHost.neterms + 6));
    dBpart = dalloc<double>((size_t)nblkP * kPartialCols);
    dRes = dalloc<double>(kResSize);
    dErr = dalloc<int>(1);
    ck(cudaMemsetAsync(dErr, 0, sizeof(int), stream), "zero error flag");
    dTmp = dalloc<float>(3 * N);
    if (sharedDevice) hKsPinned = new KSpace;   // pinned host memory would synchronise the device when freed
    else ck(cudaMallocHost(&hKsPinned, sizeof(KSpace)), "cudaMallocHost");
    // sort scratch and the permuted copies
    const uint32_t nk = sort_key_count(g);
    sortKeys = nk;
    {   // tile geometry: about one particle per thread (the density decides the bricks)
        const int codes = densityCodes();
        tiles = tileGeometry(codes, directGather);
        dtiles = tileGeometry(depositCodes ? depositCodes : codes, true);
        attachTileList(tiles);
        attachTileList(dtiles);
        recBytes = recordBytes();
        dRec = reinterpret_cast<float4 *>(dalloc<unsigned char>(recBytes));
    }
    dFgrid = dalloc<float>(3 * N);
    sortW.key = dalloc<uint32_t>(N);
    sortW.rank = dalloc<int>(N);
    sortW.newpos = dalloc<int>(N);
    sortW.count = dalloc<uint32_t>(nk);
    sortW.start = dalloc<uint32_t>(nk);
    sortW.totals = dalloc<uint32_t>(nk / 1024 + 2);
    sortW.X0 = dalloc<float>(3 * N);
    sortW.X1 = dalloc<float>(3 * N);
    sortW.noise = dalloc<float>(3 * N);
    sortW.q = doCharges ? dalloc<float>(N) : nullptr;
    sortW.flags = dalloc<uint32_t>(N);
    sortW.orig = dalloc<int>(N);
    sortW.brow = nnz > 0 ? dalloc<int>(N + 1) : nullptr;
    sortW.partner = nnz > 0 ? dalloc<int>(nnz) : nullptr;
    sortW.btype = nnz > 0 ? dalloc<uint8_t>(nnz) : nullptr;
    sortW.totalsN = dalloc<uint32_t>(N / 1024 + 2);
    sortW.rng = rngCompat ? (void *)dalloc<unsigned char>(N * rng_state_bytes()) : nullptr;
    sortW.na = nAnglesTot > 0 ? dalloc<uint8_t>(N) : nullptr;
    sortW.atype = nAnglesTot > 0 ? dalloc<uint8_t>(N * MAXANGLES) : nullptr;
    sortW.ang = nAnglesTot > 0 ? dalloc<int>(3 * N * MAXANGLES) : nullptr;
}

void Box::uploadParticles()
{
    const int64_t N = nstot;
    std::vector<float> x3(3 * N);
    for (int64_t p = 0; p < N; p++)
        for (int j = 0; j < 3; j++) x3[3 * p + j] = j < Dim ? x[p * Dim + j] : 0.f;
    ck(cudaMemcpy(dX[0], x3.data(), 12 * N, cudaMemcpyHostToDevice), "upload x");
    ck(cudaMemcpy(dX[1], x3.data(), 12 * N, cudaMemcpyHostToDevice), "upload xOld");   // GJF: xOld = x
    ck(cudaMemset(dNoise, 0, 12 * N), "zero noise");
    std::vector<int> orig(N);
    std::iota(orig.begin(), orig.end(), 0);
    ck(cudaMemcpy(dOrig, orig.data(), 4 * N, cudaMemcpyHostToDevice), "upload ids");
    if (doCharges) ck(cudaMemcpy(dQ, charges.data(), 4 * N, cudaMemcpyHostToDevice), "upload q");
    if (dBrow) {   // the padded partner lists of the data file as a CSR list
        std::vector<int> row(N + 1, 0), col;
        std::vector<uint8_t> bt;
        for (int64_t p = 0; p < N; p++) {
            for (int b = 0; b < nBonds[p]; b++) {
                col.push_back(bondedTo[p * MAXBONDS + b]);
                bt.push_back((uint8_t)bondType[p * MAXBONDS + b]);
            }
            row[p + 1] = (int)col.size();
        }
        if ((int64_t)col.size() != nBondEntries) fail(TILD_ERR_STATE, "bond list changed after set-up");
        ck(cudaMemcpy(dBrow, row.data(), 4 * (N + 1), cudaMemcpyHostToDevice), "upload bond rows");
        ck(cudaMemcpy(sortW.brow + N, row.data() + N, 4, cudaMemcpyHostToDevice), "upload bond rows");
        ck(cudaMemcpy(dPartner, col.data(), 4 * col.size(), cudaMemcpyHostToDevice), "upload partners");
        ck(cudaMemcpy(dBtype, bt.data(), bt.size(), cudaMemcpyHostToDevice), "upload bond types");
    }
    if (dNa) {
        std::vector<uint8_t> na8(N), at8(N * MAXANGLES);
        for (int64_t p = 0; p < N; p++) na8[p] = (uint8_t)nAngles[p];
        for (int64_t k = 0; k < N * MAXANGLES; k++) at8[k] = (uint8_t)angleType[k];
        ck(cudaMemcpy(dNa, na8.data(), N, cudaMemcpyHostToDevice), "upload angle counts");
        ck(cudaMemcpy(dAtype, at8.data(), N * MAXANGLES, cudaMemcpyHostToDevice), "upload angle types");
        ck(cudaMemcpy(dAng, angleGroup.data(), 12 * N * MAXANGLES, cudaMemcpyHostToDevice), "upload angles");
    }
    long long zero = 0;
    ck(cudaMemcpy(dStep, &zero, sizeof(zero), cudaMemcpyHostToDevice), "upload step");
    ck(cudaMemset(dRes, 0, sizeof(double) * kResSize), "zero results");
    uploadFlags();
    if (rngCompat) {   // d_initDeviceRNG (device_utils.cu:465-472), seed = RANDSEED (unsigned int)
        ck(launch_rng_init(dRng, dOrig, (int)N, (unsigned long long)(unsigned int)RANDSEED, stream), "rng init");
        ck(cudaStreamSynchronize(stream), "rng init sync");
    }
    ck(sharedDevice ? cudaStreamSynchronize(stream) : cudaDeviceSynchronize(), "upload");
}

// Per-particle membership flags (density fields, force groups, integrator slot, type) and
// the plan constants; flags are built in original particle order and stored in the
// current slot order.
void Box::uploadFlags()
{
    const int64_t N = nstot;
    std::vector<uint32_t> fl(N, 0u);
    std::vector<std::vector<char>> member(psGroup.size(), std::vector<char>(N, 0));
    for (size_t gi = 0; gi < psGroup.size(); gi++)
        for (int s : psGroup[gi].siteList) member[gi][s] = 1;
    for (size_t k = 0; k < dfields.size(); k++)
        for (int64_t p = 0; p < N; p++)
            if (member[dfields[k].group][p]) fl[p] |= 1u << k;
    for (size_t k = 0; k < fgroups.size(); k++)
        for (int64_t p = 0; p < N; p++)
            if (member[fgroups[k]][p]) fl[p] |= 1u << (8 + k);
    int wi = 0;
    for (const PS_Potential &p : potentials)
        if (p.kind == POT_WALL) {
            for (int s : psGroup[p.Iind].siteList) fl[s] |= 1u << (24 + wi);
            wi++;
        }
    std::vector<int> slot(N, kNoIntegrator);
    for (size_t s = 0; s < integrators.size(); s++)
        for (int p : psGroup[integrators[s].group_index].siteList) {
            if (slot[p] != kNoIntegrator) fail(TILD_ERR_UNSUPPORTED, "a particle belongs to two integrator groups");
            slot[p] = (int)s;
        }
    for (int64_t p = 0; p < N; p++) fl[p] |= ((uint32_t)slot[p] << 16) | ((uint32_t)intSpecies[p] << 20);
    const std::vector<int> orig = slotOrder();
    std::vector<uint32_t> fs(N);
    for (int64_t s = 0; s < N; s++) fs[s] = fl[orig[s]];
    ck(cudaMemcpy(dFlags, fs.data(), 4 * N, cudaMemcpyHostToDevice), "upload flags");
    ck(cudaMemcpy(dKs, &ksHost, sizeof(KSpace), cudaMemcpyHostToDevice), "upload k-space plan");
    if (ksHost.npots > 0) {
        ck(launch_uk_table(geom, dKs, dUk, stream), "u(k) table");
        ck(cudaStreamSynchronize(stream), "u(k) table");
    }
    ck(cudaMemcpy(dPp, &ppHost, sizeof(ParticleParams), cudaMemcpyHostToDevice), "upload particle params");
}

// orig[s]: original particle id stored in slot s.
std::vector<int> Box::slotOrder() const
{
    std::vector<int> orig(nstot);
    ck(cudaMemcpy(orig.data(), dOrig, 4 * nstot, cudaMemcpyDeviceToHost), "read ids");
    return orig;
}

// Spatial re-sort of every per-particle array (tild_sort.cu), then copy back in place so
// the captured step graphs keep their pointers.
void Box::sortParticles()
{
    const int64_t N = nstot;
    PermIn in{dX[0], dX[1], dNoise, dQ, dFlags, dOrig, dBrow, dPartner, dBtype, dRng, dStep, dNa, dAtype, dAng};
    ck(launch_sort(geom, (int)N, dNa ? MAXANGLES : 0, sortW, in, stream), "sort");
    auto cp = [&](void *dst, const void *src, size_t bytes) {
        ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream), "sort copy");
    };
    cp(dX[0], sortW.X0, 12 * N);
    cp(dX[1], sortW.X1, 12 * N);
    cp(dNoise, sortW.noise, 12 * N);
    cp(dFlags, sortW.flags, 4 * N);
    cp(dOrig, sortW.orig, 4 * N);
    if (dQ) cp(dQ, sortW.q, 4 * N);
    if (dBrow) {   // brow[N] (the entry count) never changes
        const int64_t nnz = nBondEntries;
        cp(dBrow, sortW.brow, 4 * N);
        cp(dPartner, sortW.partner, 4 * nnz);
        cp(dBtype, sortW.btype, nnz);
    }
    if (dRng) cp(dRng, sortW.rng, N * rng_state_bytes());
    if (dNa) {
        cp(dNa, sortW.na, N);
        cp(dAtype, sortW.atype, N * MAXANGLES);
        cp(dAng, sortW.ang, 12 * N * MAXANGLES);
    }
    sinceSort = 0;
    sortedTiles = true;
}

void Box::maybeSort()
{
    if (sortInterval > 0 && sinceSort >= sortInterval) {
        if (gSort) ck(cudaGraphLaunch(gSort, stream), "sort graph");
        else sortParticles();
        sinceSort = 0;
    }
}

// ---------------------------------------------------------------------------------------
// Step pipeline
// ---------------------------------------------------------------------------------------
void Box::mark(int stage)
{
    if (!timing) return;
    cudaEvent_t ev;
    ck(cudaEventCreate(&ev), "event");
    ck(cudaEventRecord(ev, stream), "event record");
    marks.push_back({stage, ev});
}

void Box::enqueueStep(bool energy, bool integrate, float *fout_dev)
{
    const Geom &g = geom;
    cudaStream_t st = stream;
    const int nd = (int)dfields.size(), nfg = (int)fgroups.size();
    const int npair = (nd + 1) / 2;
    mark(-1);
    if (nd > 0) {
        if (deterministic)
            ck(launch_zero(dDepFix, sizeof(unsigned long long) * 2 * npair * g.M, st), "zero");
        else
            ck(launch_zero(dDep, sizeof(float2) * npair * g.M, st), "zero");
        ck(launch_deposit(g, ppHost, dX[0], dX[1], dStep, dFlags, dQ, dDep, dDepFix, deterministic, depTileCfg(), st), "deposit");
        mark(STAGE_DEPOSIT);
        ck(launch_xfwd(g, lx, npair, nd, dDep, deterministic ? dDepFix : nullptr, dH, st), "fft x forward");
        mark(STAGE_XFWD);
        ck(launch_ypass(g, ly, nd, 0, dH, st), "fft y forward");
        mark(STAGE_YFWD);
        ck(launch_kspace_z(g, lz, ksHost, dKs, dH, dUk, dHg, dEpart, energy ? 1 : 0, nfg > 0 ? 1 : 0, nullptr, st), "kspace");
        if (energy && ksHost.neterms > 0) ck(launch_reduce_partials(dEpart, nblkZ, ksHost.neterms + 6, dRes, st), "reduce");
        mark(STAGE_KSPACE);
        if (nfg > 0) {
            ck(launch_ypass(g, ly, 3 * nfg, 1, dHg, st), "fft y inverse");
            mark(STAGE_YINV);
            ck(launch_xinv(g, lx, nfg, dHg, dRec, recLayout(), st), "fft x inverse");
            mark(STAGE_XINV);
        }
    }
    const RecLayout rl = recLayout();
    ck(launch_gather(g, ppHost, dPp, dX[0], dX[1], dFlags, dQ, dRec, rl, dStep, dFgrid, tileCfg(), recordMap(),
                     rl.paired ? &pmapA : nullptr, rl.paired ? &pmapB : nullptr, dErr, st),
       "gather");
    mark(STAGE_GATHER);
    ck(launch_integrate(g, ppHost, dPp, dX[0], dX[1], dNoise, dFlags, dQ, dBrow, dPartner, dBtype,
                        AngleArrays{dNa, dAtype, dAng}, dFgrid, rl, dOrig, dRng, dStep, fout_dev, integrate ? 1 : 0, st),
       "integrate");
    mark(STAGE_INTEGRATE);
    if (integrate) ck(launch_tick(dStep, st), "tick");
    if (energy) {
        ck(launch_bond_energy(g, ppHost, dPp, dX[0], dX[1], dStep, dBrow, dPartner, dBtype, AngleArrays{dNa, dAtype, dAng},
                              dFlags, dBpart, nullptr, st), "bond energy");
        ck(launch_reduce_partials(dBpart, nblkP, kPartialCols, dRes + kResBond, st), "reduce bonds");
    }
}

// lastStepStart: deposit from the other position buffer, which after a step holds the
// positions that step started from (GJF keeps x_{t-1} there, EM leaves x_t there).
void Box::enqueueEnergyOnly(bool lastStepStart)
{
    const Geom &g = geom;
    cudaStream_t st = stream;
    const int nd = (int)dfields.size();
    const int npair = (nd + 1) / 2;
    if (nd > 0 && ksHost.neterms > 0) {
        if (deterministic)
            ck(launch_zero(dDepFix, sizeof(unsigned long long) * 2 * npair * g.M, st), "zero");
        else
            ck(launch_zero(dDep, sizeof(float2) * npair * g.M, st), "zero");
        float *xa = lastStepStart ? dX[1] : dX[0], *xb = lastStepStart ? dX[0] : dX[1];
        ck(launch_deposit(g, ppHost, xa, xb, dStep, dFlags, dQ, dDep, dDepFix, deterministic, depTileCfg(), st), "deposit");
        ck(launch_xfwd(g, lx, npair, nd, dDep, deterministic ? dDepFix : nullptr, dH, st), "fft x forward");
        ck(launch_ypass(g, ly, nd, 0, dH, st), "fft y forward");
        ck(launch_kspace_z(g, lz, ksHost, dKs, dH, dUk, dHg, dEpart, 1, 0, nullptr, st), "kspace energy");
        ck(launch_reduce_partials(dEpart, nblkZ, ksHost.neterms + 6, dRes, st), "reduce");
    }
    ck(launch_bond_energy(g, ppHost, dPp, dX[0], dX[1], dStep, dBrow, dPartner, dBtype, AngleArrays{dNa, dAtype, dAng},
                              dFlags, dBpart, nullptr, st), "bond energy");
    ck(launch_reduce_partials(dBpart, nblkP, kPartialCols, dRes + kResBond, st), "reduce bonds");
}

std::vector<double> Box::readEnergies(bool)
{
    std::vector<double> r(kResSize, 0.0);
    ck(cudaStreamSynchronize(stream), "sync");
    ck(cudaMemcpy(r.data(), dRes, sizeof(double) * r.size(), cudaMemcpyDeviceToHost), "read energies");
    checkDeviceErrors();
    if (r[kResNonFinite] > 0.0)   // the run has blown up: stop instead of logging NaN
        fail(TILD_ERR_DEVICE, std::to_string((long long)r[kResNonFinite]) +
                                  " particle(s) with a non-finite position at step " + std::to_string(deviceStep()));
    int wi = 0;   // Wall::CalcEnergy (ps_potentialWall.cu:58-70) in the wall's potential slot
    for (size_t k = 0; k < potentials.size(); k++)
        if (potentials[k].kind == POT_WALL) r[k] = r[kResWall + wi++];
    return r;
}

void Box::dropGraphs()
{
    if (gNorm) cudaGraphExecDestroy(gNorm);
    if (gEnergy) cudaGraphExecDestroy(gEnergy);
    if (gSort) cudaGraphExecDestroy(gSort);
    gNorm = gEnergy = gSort = nullptr;
}

void Box::captureGraphs()
{
    if (gNorm && gEnergy) return;
    for (int e = 0; e < 2; e++) {
        cudaGraph_t gr;
        ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        try {
            enqueueStep(e == 1, true, nullptr);
        } catch (...) {
            cudaStreamEndCapture(stream, &gr);
            throw;
        }
        ck(cudaStreamEndCapture(stream, &gr), "end capture");
        cudaGraphExec_t ex;
        ck(cudaGraphInstantiate(&ex, gr, 0), "graph instantiate");
        cudaGraphDestroy(gr);
        (e ? gEnergy : gNorm) = ex;
    }
    if (sortInterval > 0 && !gSort) {
        cudaGraph_t gr;
        ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        try {
            sortParticles();
        } catch (...) {
            cudaStreamEndCapture(stream, &gr);
            throw;
        }
        ck(cudaStreamEndCapture(stream, &gr), "end capture");
        ck(cudaGraphInstantiate(&gSort, gr, 0), "graph instantiate");
        cudaGraphDestroy(gr);
    }
}

void Box::updateRamps(int64_t step, int64_t maxSteps)
{
    bool any = false;
    for (size_t pi = 0; pi < potentials.size(); pi++) {   // ps_potential.cu:227-248
        PS_Potential &p = potentials[pi];
        if (!p.ramp) continue;
        any = true;
        const double Ao_current = p.Ao_initial + (p.Ao_final - p.Ao_initial) / double(maxSteps) * double(step + 1);
        p.amp_eff = Ao_current / p.T0();
        ksHost.pots[pi].amp = p.amp_eff;
    }
    if (!any) return;
    *hKsPinned = ksHost;
    ck(cudaMemcpyAsync(dKs, hKsPinned, sizeof(KSpace), cudaMemcpyHostToDevice, stream), "ramp upload");
    ck(cudaStreamSynchronize(stream), "ramp sync");
}

void Box::steps(int64_t n)
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    ck(cudaSetDevice(device), "cudaSetDevice");
    if (stageTiming) {   // instrumented launches: an event after every kernel
        timing = true;
        marks.clear();
        for (int64_t i = 0; i < n; i++) {
            maybeSort();
            enqueueStep(false, true, nullptr);
            totSteps++;
            sinceSort++;
        }
        timing = false;
        ck(cudaStreamSynchronize(stream), "sync");
        stageSec.assign(STAGE_COUNT, 0.0);
        std::vector<int> cnt(STAGE_COUNT, 0);
        for (size_t k = 1; k < marks.size(); k++) {
            const int s = marks[k].first;
            if (s < 0) continue;
            float ms = 0.f;
            ck(cudaEventElapsedTime(&ms, marks[k - 1].second, marks[k].second), "elapsed");
            stageSec[s] += ms * 1e-3;
            cnt[s]++;
        }
        for (int s = 0; s < STAGE_COUNT; s++)
            if (cnt[s]) stageSec[s] /= cnt[s];
        for (auto &m : marks) cudaEventDestroy(m.second);
        marks.clear();
        return;
    }
    captureGraphs();
    for (int64_t i = 0; i < n; i++) {
        maybeSort();
        ck(cudaGraphLaunch(gNorm, stream), "graph launch");
        totSteps++;
        sinceSort++;
    }
    ck(cudaGetLastError(), "step");
}

void Box::NVT(int64_t nSteps)
{
    if (!ready) fail(TILD_ERR_STATE, "run nvt before endBox");
    ck(cudaSetDevice(device), "cudaSetDevice");
    {   // writeData(-1) (PS_Box.cu:215): computeThermoProps reads the groups' densities,
        // which after earlier steps are those the last step started from
        std::vector<double> t = thermo(totSteps > 0);
        std::vector<double> pe(t.begin() + 2, t.begin() + 2 + potentials.size());
        writeData(-1, pe, t[1], t.back());
    }
    bool anyRamp = false;
    for (auto &p : potentials) anyRamp |= p.ramp;
    if (!anyRamp) captureGraphs();
    const int npot = (int)potentials.size();
    std::vector<double> ampUsed(npot);
    std::vector<double> lastPair(npot, 0.0);
    double lastBond = 0.0, lastAngle = 0.0;
    const bool files = writeFiles != 0;
    if (files && !fieldFilesReady) initFieldFiles();   // write_files switched on after endBox
    for (int64_t i = 0; i < nSteps; i++) {
        const bool energy = (i % logFreq == 0) || (i == nSteps - 1);
        const bool fieldDue = files && fieldFreq > 0 && i % fieldFreq == 0;
        for (int k = 0; k < npot; k++) ampUsed[k] = potentials[k].amp_eff;
        maybeSort();
        // the group densities of step i come from the positions it starts from (PS_Box.cu:108-114);
        // the last step's stay in the buffer for the final frame
        if (files && (fieldDue || i == nSteps - 1)) computeFieldFrame();
        if (fieldDue) enqueueFrame(0, i);
        if (anyRamp) enqueueStep(energy, true, nullptr);
        else ck(cudaGraphLaunch(energy ? gEnergy : gNorm, stream), "graph launch");
        totSteps++;
        sinceSort++;
        updateRamps(i, nSteps);
        if (energy) {
            std::vector<double> r = readEnergies(true);
            for (int k = 0; k < npot; k++)   // CalcEnergy runs after update_prefactor (PS_Box.cu:159-172)
                lastPair[k] = r[k] * (ampUsed[k] != 0.0 ? potentials[k].amp_eff / ampUsed[k] : 1.0);
            lastBond = 0.5 * r[kResBond];
            lastAngle = r[kResAngle] / 3.0;   // each angle summed on its three particles
            if (i % logFreq == 0) writeData(i, lastPair, lastBond, lastAngle);
        }
        // positions after the step (PS_Box.cu:180-194); the GSD frame carries the step count
        // the box had before this step
        const bool gsdDue = files && gsdFreq > 0 && i % gsdFreq == 0;
        if (gsdDue) enqueueFrame(2, totSteps - 1);
        if (gsdDue && i > 1 && logSpaceGSD) gsdFreq = (int)((float)gsdFreq * logScaleGSD);
        if (files && trajFreq > 0 && i % trajFreq == 0) enqueueFrame(1, i);
        if (fieldDue && i > 1 && logSpaceFields)   // PS_Box.cu:197-203
            fieldFreq = (int)((float)fieldFreq * logScaleFields);
    }
    ck(cudaStreamSynchronize(stream), "run");
    if (nSteps > 0) writeData(nSteps, lastPair, lastBond, lastAngle);   // PS_Box.cu:227
    if (files) {   // writeFields (PS_Box.cu:228): the densities the last step started from
        if (!fieldFrameValid) computeFieldFrame();
        enqueueFrame(0, nSteps);
        enqueueFrame(2, totSteps);                // writeGSDtraj (PS_Box.cu:229)
        flushFrames(0);
        writeDataConfig("final.input.data");      // PS_Box.cu:230
    }
}

// ---- output frames ------------------------------------------------------------------

// Box::initBinaryDataFile (Box.cu:552-570) for every group's density file
// (PS_Box_initialization.cu:527-533): int Dim, int Nx[Dim], float L[Dim], native byte order.
void Box::initFieldFiles()
{
    if ((int)psGroup.size() > kMaxFrameGroups)
        fail(TILD_ERR_UNSUPPORTED, "density files support at most " + std::to_string(kMaxFrameGroups) + " groups");
    nFrameGroups = (int)psGroup.size();
    fieldFilesReady = true;
    for (const PS_Group &g : psGroup) {
        std::ofstream o(resolve("density-" + g.name + ".bin"), std::ios::binary);
        if (!o.is_open()) fail(TILD_ERR_IO, "Failed to initialize output binary file!");
        o.write(reinterpret_cast<const char *>(&Dim), sizeof(int));
        o.write(reinterpret_cast<const char *>(Nx), Dim * sizeof(int));
        o.write(reinterpret_cast<const char *>(L), Dim * sizeof(float));
    }
}

// Every frame group's density at the current positions into dFieldFrame (one pass over
// the particles, each adding its weights to the fields of the groups it belongs to).
void Box::computeFieldFrame()
{
    const int64_t M = geom.M;
    if (!dFieldFrame) {
        std::vector<unsigned long long> mask(nstot, 0ull);
        for (int g = 0; g < nFrameGroups; g++)
            for (int p : psGroup[g].siteList) mask[p] |= 1ull << g;
        dGroupMask = dalloc<unsigned long long>(nstot);
        dFieldFrame = dalloc<float>((size_t)nFrameGroups * M);
        ck(cudaMemcpyAsync(dGroupMask, mask.data(), 8 * nstot, cudaMemcpyHostToDevice, stream), "group masks");
        ck(cudaStreamSynchronize(stream), "group masks");
    }
    ck(cudaMemsetAsync(dFieldFrame, 0, 4 * (size_t)nFrameGroups * M, stream), "clear field frame");
    ck(launch_group_density_frames(geom, ppHost, dX[0], dX[1], dStep, dOrig, dGroupMask, (int)nstot, dFieldFrame,
                                   stream),
       "field frame");
    fieldFrameValid = true;
}

float *Box::hostBuffer(size_t bytes)
{
    for (size_t k = 0; k < hostSpare.size(); k++)
        if (hostSpare[k].first == bytes) {
            float *h = hostSpare[k].second;
            hostSpare.erase(hostSpare.begin() + k);
            return h;
        }
    void *h = nullptr;
    if (sharedDevice) h = ::operator new(bytes);   // cudaFreeHost would synchronise the shared device
    else ck(cudaMallocHost(&h, bytes), "cudaMallocHost");
    return static_cast<float *>(h);
}

// Queue a copy of a frame: kind 0 the field frame in dFieldFrame, kind 1 the positions
// in original order.  The copy runs on the box's stream behind the queued steps; at most
// two frames wait, the oldest written once its copy has landed.
void Box::enqueueFrame(int kind, int64_t step)
{
    OutFrame f{kind, step, nullptr, 0, nullptr};
    const float *src;
    if (kind == 0) {
        f.bytes = 4 * (size_t)nFrameGroups * geom.M;
        src = dFieldFrame;
    } else {   // lammpstrj and GSD frames: positions
        f.bytes = 12 * (size_t)nstot;
        ck(launch_snapshot_positions((int)nstot, dOrig, dX[0], dX[1], dStep, dTmp, stream), "position snapshot");
        src = dTmp;
    }
    f.host = hostBuffer(f.bytes);
    ck(cudaEventCreateWithFlags(&f.ev, cudaEventDisableTiming), "event");
    outFrames.push_back(f);   // owned by the queue from here on
    ck(cudaMemcpyAsync(f.host, src, f.bytes, cudaMemcpyDeviceToHost, stream), "frame copy");
    ck(cudaEventRecord(f.ev, stream), "frame event");
    flushFrames(2);
}

void Box::flushFrames(size_t keep)
{
    while (outFrames.size() > keep) {
        OutFrame f = outFrames.front();
        ck(cudaEventSynchronize(f.ev), "frame copy");
        outFrames.pop_front();
        cudaEventDestroy(f.ev);
        hostSpare.push_back({f.bytes, f.host});
        writeFrame(f);
    }
}

void Box::writeFrame(const OutFrame &f)
{
    if (f.kind == 0) {   // PS_Group::writeDensityFieldBinary -> Box::writeBinaryData (Box.cu:573-583)
        for (int g = 0; g < nFrameGroups; g++) {
            std::ofstream o(resolve("density-" + psGroup[g].name + ".bin"), std::ios::app | std::ios::binary);
            if (!o.is_open()) fail(TILD_ERR_IO, "Failed to open output binary file!");
            o.write(reinterpret_cast<const char *>(f.host + (size_t)g * geom.M), 4 * geom.M);
        }
        return;
    }
    if (f.kind == 2) {
        writeGsdFrame(f.step, f.host);
        return;
    }
    // PS_Box::writeLammpsTraj (PS_Box.cu:750-795): one wrap into the box, the file
    // truncated by the frame of step 0
    const std::string name = resolve(trajFileName);
    FILE *o = std::fopen(name.c_str(), f.step == 0 ? "w" : "a");
    if (!o) fail(TILD_ERR_IO, "Failed to open " + name);
    std::fprintf(o, "ITEM: TIMESTEP\n%d\nITEM: NUMBER OF ATOMS\n%d\n", (int)f.step, (int)nstot);
    std::fprintf(o, "ITEM: BOX BOUNDS pp pp pp\n");
    std::fprintf(o, "%f %f\n%f %f\n%f %f\n", 0.f, L[0], 0.f, L[1], 0.f, Dim == 3 ? L[2] : 1.f);
    std::fprintf(o, "ITEM: ATOMS id type mol x y z\n");
    std::vector<char> buf;
    buf.reserve(1 << 20);
    char line[160];
    for (int64_t p = 0; p < nstot; p++) {
        int n = std::snprintf(line, sizeof line, "%d %d %d  ", (int)p + 1, intSpecies[p] + 1, mID[p] + 1);
        for (int j = 0; j < Dim; j++) {
            float v = f.host[3 * p + j];
            if (v > L[j]) v -= L[j];
            else if (v < 0.0f) v += L[j];
            n += std::snprintf(line + n, sizeof line - n, "%f ", v);
        }
        for (int j = Dim; j < 3; j++) n += std::snprintf(line + n, sizeof line - n, "%f", 0.f);
        line[n++] = '\n';
        buf.insert(buf.end(), line, line + n);
        if (buf.size() > (1u << 20)) {
            std::fwrite(buf.data(), 1, buf.size(), o);
            buf.clear();
        }
    }
    std::fwrite(buf.data(), 1, buf.size(), o);
    std::fclose(o);
}

// PS_Box::writeGSDtraj (PS_Box_gsdUtils.cu:14-168) with the lists of GSDinit (:586-608).
// At step 0 the file is created again with the topology chunks; later frames hold the step,
// the positions shifted by -L/2 (not wrapped) and the charges.  Bonds are listed from their
// lower-index particle in particle order (GSDinit); angles in the order they were read, ends
// swapped so i1 < i3, as readDataConfig records them (:931-990) -- angles made by a molecule
// builder are never recorded there and stay zero, as in the reference.  Types are named
// type0..type<ntypes> in 10-byte rows.  Two reference defects are not reproduced: its
// bond and angle totals count data-file bonds and angles twice (the header's count plus the
// finishInit count, PS_Box_initialization.cu:430-445, 809-810), padding the lists with
// zero rows, and it fills only the low 32 bits of the 64-bit step chunk.
void Box::writeGsdFrame(int64_t step, const float *x_orig)
{
    const uint64_t N = (uint64_t)nstot;
    const uint64_t st = (uint64_t)step;
    if (step == 0 || !gsd.isOpen()) {
        gsd.create(resolve(gsdName), "gpu-tild", "hoomd", GsdWriter::version(1, 4));
        gsd.chunk("configuration/step", GSD_U64, 1, 1, &st);
        const uint8_t dims = 3;
        gsd.chunk("configuration/dimensions", GSD_U8, 1, 1, &dims);
        float box[6] = {0, 0, 0, 0, 0, 0};
        for (int j = 0; j < Dim; j++) box[j] = L[j];
        if (Dim == 2) box[2] = 5.0f;
        gsd.chunk("configuration/box", GSD_F32, 6, 1, box);
        const uint32_t n32 = (uint32_t)N;
        gsd.chunk("particles/N", GSD_U32, 1, 1, &n32);
        std::vector<float> mass(N);
        std::vector<uint32_t> typeid_(N), molid(N);
        for (uint64_t p = 0; p < N; p++) {
            mass[p] = species[intSpecies[p]].mass;
            typeid_[p] = (uint32_t)(intSpecies[p] + 1);
            molid[p] = (uint32_t)(mID[p] + 1);
        }
        gsd.chunk("particles/mass", GSD_F32, N, 1, mass.data());
        gsd.chunk("particles/typeid", GSD_U32, N, 1, typeid_.data());
        gsd.chunk("log/particles/moleculeid", GSD_U32, N, 1, molid.data());
        const size_t nt = species.size() + 1;
        std::vector<char> tn(nt * 10, 0);
        for (size_t t = 0; t < nt; t++) {
            const std::string nm = "type" + std::to_string(t);
            std::memcpy(tn.data() + t * 10, nm.c_str(), std::min<size_t>(nm.size(), 9));
        }
        gsd.chunk("particles/types", GSD_I8, nt, 10, tn.data());
        std::vector<uint32_t> btype, bgroup;
        for (int64_t p = 0; p < nstot; p++)
            for (int b = 0; b < nBonds[p]; b++)
                if (bondedTo[p * MAXBONDS + b] > p) {
                    bgroup.push_back((uint32_t)p);
                    bgroup.push_back((uint32_t)bondedTo[p * MAXBONDS + b]);
                    btype.push_back((uint32_t)bondType[p * MAXBONDS + b]);
                }
        const uint32_t nb = (uint32_t)btype.size(), na = (uint32_t)nAnglesTot;
        gsd.chunk("bonds/N", GSD_U32, 1, 1, &nb);
        gsd.chunk("bonds/typeid", GSD_U32, nb, 1, btype.data());
        gsd.chunk("bonds/group", GSD_U32, nb, 2, bgroup.data());
        std::vector<uint32_t> atype(na, 0u), agroup((size_t)na * 3, 0u);
        for (size_t a = 0; a < angleList.size() / 4 && a < na; a++) {
            atype[a] = angleList[4 * a];
            for (int r = 0; r < 3; r++) agroup[3 * a + r] = angleList[4 * a + 1 + r];
        }
        gsd.chunk("angles/N", GSD_U32, 1, 1, &na);
        gsd.chunk("angles/typeid", GSD_U32, na, 1, atype.data());
        gsd.chunk("angles/group", GSD_U32, na, 3, agroup.data());
    } else {
        gsd.chunk("configuration/step", GSD_U64, 1, 1, &st);
    }
    std::vector<float> pos(3 * N, 0.f);
    for (uint64_t p = 0; p < N; p++)
        for (int j = 0; j < Dim; j++) pos[3 * p + j] = x_orig[3 * p + j] - Lh[j];
    gsd.chunk("particles/position", GSD_F32, N, 3, pos.data());
    if (doCharges) gsd.chunk("particles/charge", GSD_F32, N, 1, charges.data());
    gsd.endFrame();
}

// Drop queued frames without writing them (error paths, destruction) and free the host buffers.
void Box::releaseFrames()
{
    if (!outFrames.empty() && stream) cudaStreamSynchronize(stream);
    for (OutFrame &f : outFrames) {
        cudaEventDestroy(f.ev);
        hostSpare.push_back({f.bytes, f.host});
    }
    outFrames.clear();
    for (auto &h : hostSpare) {
        if (sharedDevice) ::operator delete(h.second);
        else cudaFreeHost(h.second);
    }
    hostSpare.clear();
}

void Box::writeData(int64_t step, const std::vector<double> &pairE, double ubond, double uangle)
{
    double upe = ubond + uangle;
    for (size_t k = 0; k < pairE.size() && k < potentials.size(); k++) {
        potentials[k].energy = pairE[k];
        upe += pairE[k];
    }
    std::vector<double> row;
    row.push_back((double)step);
    row.push_back(ubond);
    if (nAnglesTot > 0) row.push_back(uangle);
    for (size_t k = 0; k < potentials.size(); k++) row.push_back(potentials[k].energy);
    logRows.push_back(row);
    std::ostringstream ln, echoLn;   // PS_Box.cu:339-370 (default stream formatting)
    ln << step;
    echoLn << "step: " << step << " Upe: " << upe;
    if (nBondsTot > 0) {
        ln << " " << ubond;
        echoLn << " Ubond: " << ubond;
    }
    if (nAnglesTot > 0) {   // PS_Box.cu:356-359
        ln << " " << uangle;
        echoLn << " Uangle: " << uangle;
    }
    for (size_t k = 0; k < potentials.size(); k++) {
        ln << " " << potentials[k].energy;
        echoLn << " pot[" << k << "]: " << potentials[k].energy;
    }
    if (writeFiles) {
        std::ofstream o(resolve(datFileName), std::ios_base::app);
        o << ln.str() << std::endl;
    }
    if (echo) std::cout << echoLn.str() << std::endl;
}

std::vector<double> Box::thermo(bool lastStepStart)
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    ck(cudaSetDevice(device), "cudaSetDevice");
    enqueueEnergyOnly(lastStepStart);
    std::vector<double> r = readEnergies(true);
    std::vector<double> out;
    const size_t np = potentials.size();
    const double uangle = r[kResAngle] / 3.0;   // PS_Box.cu:296-305
    double ubond = 0.5 * r[kResBond], upe = ubond + uangle, upair = 0.0, uwall = 0.0;
    for (size_t k = 0; k < np; k++) (potentials[k].kind == POT_WALL ? uwall : upair) += r[k];
    upe += upair + uwall;
    out.push_back(upe);
    out.push_back(ubond);
    for (size_t k = 0; k < np; k++) out.push_back(r[k]);
    double wb[6], wp[6];
    for (int c = 0; c < 6; c++) {
        // bonded: sum over bonds of dr_a f_b, plus over angles of r_ij,a f_i,b + r_kj,a f_k,b
        wb[c] = 0.5 * r[kResBond + 1 + c] + r[kResAngle + 1 + c] / 3.0;
        wp[c] = r[np + c] + (c < Dim ? upair : 0.0);          // pairs: -dU/d(strain_ab)
        out.push_back(wb[c]);
    }
    // pair virial, then the pressure tensor (N kT delta_ab + W_pair + W_bond) / V, kT = 1
    for (int c = 0; c < 6; c++) out.push_back(wp[c]);
    const double V = (double)L[0] * L[1] * L[2];
    for (int c = 0; c < 6; c++) out.push_back(((c < Dim ? (double)nstot : 0.0) + wp[c] + wb[c]) / V);
    out.push_back(uangle);
    return out;
}

void Box::forces(float *f_out)
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    ck(cudaSetDevice(device), "cudaSetDevice");
    enqueueStep(false, false, dF);
    ck(launch_unpermute_rows((int)nstot, 3, dOrig, dF, dTmp, stream), "unpermute forces");
    readRows3(dTmp, f_out);
    checkDeviceErrors();
}

// dev[3n] (original order) -> host out[n*Dim], the reference's layout of x and f
void Box::readRows3(const float *dev, float *out) const
{
    if (Dim == 3) {
        ck(cudaMemcpyAsync(out, dev, 12 * nstot, cudaMemcpyDeviceToHost, stream), "read rows");
        ck(cudaStreamSynchronize(stream), "read rows");
        return;
    }
    std::vector<float> h(3 * nstot);
    ck(cudaMemcpyAsync(h.data(), dev, 12 * nstot, cudaMemcpyDeviceToHost, stream), "read rows");
    ck(cudaStreamSynchronize(stream), "read rows");
    for (int64_t p = 0; p < nstot; p++)
        for (int j = 0; j < Dim; j++) out[p * Dim + j] = h[3 * p + j];
}

// Tile of `codes` consecutive brick codes: threads for about one particle each (mean plus
// two standard deviations), the deposit's box estimate, and the particle pass's fixed box
// (the tile's bricks widened by the stencil and one cell of drift per side; particles that
// drift further are gathered from global memory).  direct: the particle pass stages no
// box and reads every particle's stencil through L1/L2.
TileCfg Box::tileGeometry(int codes, bool direct) const
{
    const Geom &g = geom;
    const double perCode = 16.0 * std::min(4, g.nz) * (double)nstot / (double)g.M;
    const double e = perCode * codes;
    int thr = (int)std::ceil((e + 2.0 * std::sqrt(e) + 8.0) / 32.0) * 32;
    thr = std::max(64, std::min(512, thr));
    int bits = 0;
    while ((1 << bits) < codes) bits++;
    const int cx = 4 << ((bits + 2) / 3), cy = 4 << ((bits + 1) / 3), cz = 4 << (bits / 3);
    const int slack = pmeorder + 1 + 3;   // stencil width + drift between sorts
    long long box = (long long)(((cx + slack) | 1) * (cy + slack) | 1) * (cz + slack);
    box = std::min<long long>(box, 3072);
    const int margin = 1, ev = (pmeorder % 2 == 0) ? 1 : 0;
    auto edge = [&](int cells, int n) { return std::min(cells, n) - 1 + ev + 2 * margin + pmeorder + 1; };
    const int ex = edge(cx, g.nx), ey = edge(cy, g.ny), ez = edge(cz, g.nz);
    TileCfg t{};
    t.nkeys = (int)sortKeys;
    t.codes = codes;
    t.threads = thr;
    t.box = (int)box;
    t.pbox = (((ex | 1) * ey) | 1) * ez;
    t.direct = direct ? 1 : 0;
    t.margin = margin;
    const int nfg = (int)fgroups.size();
    if (g.nz > 1 && !direct && nfg >= 1 && nfg <= 2) {
        // paired records: an x edge of 2 (mod 4), even for plane B's rows and such that the
        // 8-lane gather's quarter warps start at eight distinct bank groups
        t.te[0] = (ex + 1) & ~1;
        if (t.te[0] % 4 == 0) t.te[0] += 2;
        t.te[1] = ey;
        t.te[2] = ez;
        t.paired = paired_box_fits(t.te, nfg) ? 1 : 0;
        if (t.paired) t.pbox = t.te[0] * t.te[1] * t.te[2];
    }
    if (g.nz > 1 && !direct && !t.paired) {   // planar TMA box: odd x and y edges keep the dense pitches odd
        t.te[0] = ex | 1;
        t.te[1] = ey | 1;
        t.te[2] = ez;
        t.pbox = std::max(t.pbox, t.te[0] * t.te[1] * t.te[2]);
    }
    return t;
}

// The tiles of t.codes bricks whose first cell lies inside the grid, for launches over
// those alone: the Morton code space of the sort is a power-of-two cube of bricks, so the
// tiles past the grid's edge (more than half of them on a 192^3 grid) hold no particle.
void Box::attachTileList(TileCfg &t)
{
    auto it = tileLists.find(t.codes);
    if (it == tileLists.end()) {
        auto compact3 = [](uint32_t v) {
            v &= 0x09249249u;
            v = (v | (v >> 2)) & 0x030C30C3u;
            v = (v | (v >> 4)) & 0x0300F00Fu;
            v = (v | (v >> 8)) & 0x030000FFu;
            v = (v | (v >> 16)) & 0x000003FFu;
            return (int)v;
        };
        std::vector<uint32_t> h;
        const uint32_t ntile = (sortKeys + (uint32_t)t.codes - 1) / (uint32_t)t.codes;
        for (uint32_t k = 0; k < ntile; k++) {
            const uint32_t k0 = k * (uint32_t)t.codes;
            if (4 * compact3(k0) < geom.nx && 4 * compact3(k0 >> 1) < geom.ny && 4 * compact3(k0 >> 2) < geom.nz)
                h.push_back(k);
        }
        uint32_t *d = dalloc<uint32_t>(std::max<size_t>(1, h.size()));
        ck(cudaMemcpy(d, h.data(), sizeof(uint32_t) * h.size(), cudaMemcpyHostToDevice), "tile list");
        it = tileLists.emplace(t.codes, std::make_pair(d, (int)h.size())).first;
    }
    t.list = it->second.first;
    t.nlist = it->second.second;
}

// Ghost layers of the paired records for the tiles t: a tile's box starts gl = P/2 + margin
// points below its first cell and spans te[] points, so the last tile along an axis reaches
// gh[] points past the grid.
void Box::pairedGhosts(const TileCfg &t, int *gl, int *gh) const
{
    *gl = pmeorder / 2 + t.margin;
    int bits = 0;
    while ((1 << bits) < t.codes) bits++;
    const int cb[3] = {4 << ((bits + 2) / 3), 4 << ((bits + 1) / 3), 4 << (bits / 3)};
    const int n[3] = {geom.nx, geom.ny, geom.nz};
    for (int j = 0; j < 3; j++) {
        const int c0max = cb[j] * ((n[j] - 1) / cb[j]);
        gh[j] = std::max(0, c0max - *gl + t.te[j] - n[j]);
    }
}

// The records' layout for the current tiles: paired (with their TMA maps) when the tiles
// use the tile gather, else planar.  Tiles whose maps cannot be built fall back to the
// planar gather with cp.async staging.
RecLayout Box::recLayout()
{
    RecLayout rl{};
    if (!tiles.paired || !sortedTiles) return rl;   // unsorted particles: windows of slots, planar gather
    int gl, gh[3];
    pairedGhosts(tiles, &gl, gh);
    if (rec_layout_bytes(geom, (int)fgroups.size(), gl, gh) <= recBytes) {
        rl = make_rec_layout(geom, (int)fgroups.size(), gl, gh, dRec);
        if (!pmapOk || std::memcmp(pmapTe, tiles.te, sizeof(pmapTe)) != 0 || pmapGl != rl.gl ||
            std::memcmp(pmapGh, rl.gh, sizeof(pmapGh)) != 0) {
            pmapOk = build_paired_maps(&pmapA, &pmapB, rl, tiles.te);
            std::memcpy(pmapTe, tiles.te, sizeof(pmapTe));
            std::memcpy(pmapGh, rl.gh, sizeof(pmapGh));
            pmapGl = rl.gl;
        }
        if (pmapOk) return rl;
    }
    tiles.paired = 0;
    tiles.te[0] = tiles.te[1] = tiles.te[2] = 0;
    return RecLayout{};
}

// Tile autotuner (option "autotune"): times the force evaluation (deposit, transforms,
// force pass without integration) with tiles of half, the same and twice the bricks of
// the density rule, each with the particle pass's staged box and with direct gathers,
// and keeps the fastest; then the deposit's own tiles from the particle pass's up to
// eight times its bricks.  Positions, the step counter, the noise and the RNG state are
// not touched.
void Box::autotuneTiles()
{
    if (!sortedTiles) return;
    // the best of two timings of five force evaluations, after one to warm up
    auto timeForces = [&](cudaEvent_t a, cudaEvent_t b) {
        enqueueStep(false, false, dF);
        float best = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            ck(cudaEventRecord(a, stream), "event");
            for (int r = 0; r < 5; r++) enqueueStep(false, false, dF);
            ck(cudaEventRecord(b, stream), "event");
            ck(cudaEventSynchronize(b), "autotune");
            float ms = 0.f;
            ck(cudaEventElapsedTime(&ms, a, b), "event");
            best = std::min(best, ms / 5.f);
        }
        return best;
    };
    // particle tiles of half, the same and twice the bricks, staged and direct; staged ones
    // also with 64 more threads (the cubic tile gather spreads a tile's particles over all
    // its warps: shorter chains of gathers per warp, fewer CTAs per SM)
    std::vector<TileCfg> cands;
    for (int c : {tiles.codes / 2, tiles.codes, tiles.codes * 2})
        if (c >= 1 && c <= 64)
            for (bool direct : {false, true}) {
                cands.push_back(tileGeometry(c, direct));
                if (!direct && pmeorder == 3 && !gatherThreads && cands.back().threads + 64 <= 448) {
                    cands.push_back(cands.back());
                    cands.back().threads += 64;
                }
            }
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    float best = 1e30f;
    TileCfg pick = tiles;
    for (TileCfg &t : cands) attachTileList(t);
    for (const TileCfg &t : cands) {
        tiles = t;
        const float ms = timeForces(e0, e1);
        if (ms < best) {
            best = ms;
            pick = t;
        }
    }
    tiles = pick;
    // the deposit's tiles: the same, twice, four and eight times the bricks (a larger tile
    // zeroes and flushes fewer halo points per particle, but its fixed-point scale drops,
    // and past four times the count bound it sums in FP32), each with one thread per
    // particle and with CTAs of 64, 128 and 256 threads (smaller CTAs, more of them per SM)
    if (!depositCodes || !depositThreads) {
        TileCfg dpick = dtiles;
        std::vector<TileCfg> dc;
        for (int c = tiles.codes; c <= std::min(64, 8 * tiles.codes); c *= 2) {
            if (depositCodes && c != depositCodes) continue;
            for (int thr : {0, 64, 128, 256}) {
                if (depositThreads && thr != depositThreads) continue;
                TileCfg t = tileGeometry(c, true);
                if (thr) t.threads = thr;
                dc.push_back(t);
            }
        }
        for (TileCfg &t : dc) {
            dtiles = t;
            attachTileList(dtiles);
            const float ms = timeForces(e0, e1);
            if (ms < best) {
                best = ms;
                dpick = dtiles;
            }
        }
        dtiles = dpick;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tunedMs = best;
}

// TMA descriptor of the force records for the current tiles' box (rebuilt when the tiles
// change); NULL where none can be built, and the particle pass stages with cp.async.
const CUtensorMap *Box::recordMap()
{
    if (tiles.te[0] <= 0 || tiles.paired || !dRec) return nullptr;
    if (!recMapOk || std::memcmp(recMapTe, tiles.te, sizeof(recMapTe)) != 0) {
        recMapOk = build_record_map(&recMap, dRec, geom, std::max(1, (int)fgroups.size()), tiles.te);
        std::memcpy(recMapTe, tiles.te, sizeof(recMapTe));
    }
    return recMapOk ? &recMap : nullptr;
}

// Device-side failures the kernels record instead of faulting (a staging wait that ran
// out): reported once as TILD_ERR_DEVICE, then cleared.
void Box::checkDeviceErrors()
{
    int e = 0;
    ck(cudaMemcpyAsync(&e, dErr, sizeof(int), cudaMemcpyDeviceToHost, stream), "read error flag");
    ck(cudaStreamSynchronize(stream), "read error flag");
    if (e) {
        ck(cudaMemsetAsync(dErr, 0, sizeof(int), stream), "clear error flag");
        fail(TILD_ERR_DEVICE, std::to_string(e) + " staging wait(s) of the particle pass ran out of time");
    }
}

TileCfg Box::tileCfg() const
{
    TileCfg t = tiles;
    if (gatherThreads) t.threads = gatherThreads;
    t.start = sortedTiles ? sortW.start : nullptr;
    return t;
}

TileCfg Box::depTileCfg() const
{
    TileCfg t = dtiles;
    if (depositThreads) t.threads = depositThreads;
    t.start = sortedTiles ? sortW.start : nullptr;
    return t;
}

long long Box::deviceStep() const
{
    long long s = 0;
    ck(cudaStreamSynchronize(stream), "sync");
    ck(cudaMemcpy(&s, dStep, sizeof(s), cudaMemcpyDeviceToHost), "read step");
    return s;
}

void Box::getPositions(float *xo) const
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    const long long s = deviceStep();
    ck(launch_unpermute_rows((int)nstot, 3, dOrig, dX[s & 1], dTmp, stream), "unpermute positions");
    readRows3(dTmp, xo);
}

void Box::setPositions(const float *xi)
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    ck(cudaStreamSynchronize(stream), "sync");
    std::vector<float> flat;
    if (Dim == 2) {   // x_in[n*2]; the device rows keep z = 0 (the plane of a 2-D box)
        flat.assign(3 * nstot, 0.f);
        for (int64_t p = 0; p < nstot; p++)
            for (int j = 0; j < 2; j++) flat[3 * p + j] = xi[2 * p + j];
        xi = flat.data();
    }
    ck(cudaMemcpyAsync(dTmp, xi, 12 * nstot, cudaMemcpyHostToDevice, stream), "set positions");
    ck(launch_permute_rows((int)nstot, 3, dOrig, dTmp, dX[0], stream), "permute positions");
    ck(cudaMemcpyAsync(dX[1], dX[0], 12 * nstot, cudaMemcpyDeviceToDevice, stream), "set positions");
    ck(cudaMemsetAsync(dNoise, 0, 12 * nstot, stream), "zero noise");
    ck(cudaStreamSynchronize(stream), "set positions");
}

void Box::getDensity(const std::string &group, int charge, float *rho)
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    const int gi = findGroupInteger(group);
    if (charge && !psGroup[gi].isCharges) fail(TILD_ERR_ARG, "only the 'charges' group has a charge density");
    const long long s = deviceStep();
    const std::vector<int> orig = slotOrder();
    std::vector<int> slotOf(nstot);
    for (int64_t k = 0; k < nstot; k++) slotOf[orig[k]] = (int)k;
    std::vector<int> sites(psGroup[gi].siteList);
    for (int &v : sites) v = slotOf[v];
    int *dSites = nullptr;
    float *dRho = nullptr;
    ck(cudaMalloc(&dSites, 4 * sites.size()), "malloc");
    ck(cudaMalloc(&dRho, 4 * geom.M), "malloc");
    cudaMemcpy(dSites, sites.data(), 4 * sites.size(), cudaMemcpyHostToDevice);
    cudaMemset(dRho, 0, 4 * geom.M);
    cudaError_t e = launch_density_single(geom, ppHost, dX[s & 1], dSites, (int)sites.size(), dQ, charge, dRho, stream);
    cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = cudaMemcpy(rho, dRho, 4 * geom.M, cudaMemcpyDeviceToHost);
    cudaFree(dSites);
    cudaFree(dRho);
    ck(e, "density");
}

// Grid force of a group from the last force evaluation (tild_box_forces or a step), in the
// reference's layout and units: gf[m*Dim + d] = -d/dx_d of the group's summed potential
// field, as PS_Group::d_gridForce holds it after CalcForces (ps_potential.cu:41-125,
// ps_groups.cu:164-179).  The records keep it scaled by the gather's gvol / gvol_f32 (the
// particle pass takes unscaled weights), which is divided out here.  A group that takes
// no grid force reads zeros, as its zeroed field would.
void Box::getGridForce(const std::string &group, float *gf)
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    const int gi = findGroupInteger(group);
    const long long M = geom.M;
    int k = -1;
    for (size_t i = 0; i < fgroups.size(); i++)
        if (fgroups[i] == gi) k = (int)i;
    if (k < 0) {
        std::fill(gf, gf + M * Dim, 0.f);
        return;
    }
    std::vector<float4> h((size_t)M);
    ck(cudaSetDevice(device), "cudaSetDevice");
    const RecLayout rl = recLayout();
    if (rl.paired) {   // group k's (x, y, z) out of the padded planes
        std::vector<float4> hA((size_t)rl.pM);
        std::vector<float2> hB(rl.nfg == 2 ? (size_t)rl.pM : 0);
        ck(cudaMemcpyAsync(hA.data(), rl.A, sizeof(float4) * rl.pM, cudaMemcpyDeviceToHost, stream), "read grid force");
        if (rl.nfg == 2)
            ck(cudaMemcpyAsync(hB.data(), rl.B, sizeof(float2) * rl.pM, cudaMemcpyDeviceToHost, stream), "read grid force");
        ck(cudaStreamSynchronize(stream), "read grid force");
        for (int z = 0; z < geom.nz; z++)
            for (int y = 0; y < geom.ny; y++)
                for (int x = 0; x < geom.nx; x++) {
                    const size_t i = ((size_t)(z + rl.gl) * rl.py + (y + rl.gl)) * rl.px + x + rl.gl;
                    const size_t m = ((size_t)z * geom.ny + y) * geom.nx + x;
                    const float4 a = hA[i];
                    if (rl.nfg == 1) h[m] = a;
                    else if (k == 0) h[m] = make_float4(a.x, a.y, hB[i].x, 0.f);
                    else h[m] = make_float4(a.z, a.w, hB[i].y, 0.f);
                }
    } else {
        ck(cudaMemcpyAsync(h.data(), dRec + (size_t)k * M, sizeof(float4) * M, cudaMemcpyDeviceToHost, stream),
           "read grid force");
        ck(cudaStreamSynchronize(stream), "read grid force");
    }
    const double gvf = (double)((1.0f * geom.dxf[0]) * geom.dxf[1] * geom.dxf[2]);
    const double scale = gvf / gvol;
    for (long long m = 0; m < M; m++) {
        gf[m * Dim] = (float)(h[m].x * scale);
        gf[m * Dim + 1] = (float)(h[m].y * scale);
        if (Dim == 3) gf[m * Dim + 2] = (float)(h[m].z * scale);
    }
}

// getDensity without any allocation: the accumulator rho[M], the slot-of-particle table
// slot_of[N] and the group's sites[ns] live in the static device scratch, in that order.
// rho must start at zero and is cleared here on every call; slot_of and sites are fully
// overwritten.  Calls on one device share the scratch and must not overlap.
void Box::getDensityNoAlloc(const std::string &group, int charge, float *rho)
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    const int gi = findGroupInteger(group);
    if (charge && !psGroup[gi].isCharges) fail(TILD_ERR_ARG, "only the 'charges' group has a charge density");
    const std::vector<int> &sites = psGroup[gi].siteList;
    const size_t need = 4 * ((size_t)geom.M + (size_t)nstot + sites.size());
    if (need > kStaticScratchBytes)
        fail(TILD_ERR_ARG, "get_density_noalloc needs " + std::to_string(need) +
                               " bytes of device scratch (4 bytes per grid point, particle and group site); "
                               "the static scratch holds " + std::to_string(kStaticScratchBytes));
    ck(cudaSetDevice(device), "cudaSetDevice");
    void *scr = nullptr;
    ck(static_scratch(device, &scr), "static scratch address");
    float *dRho = static_cast<float *>(scr);
    int *dSlotOf = reinterpret_cast<int *>(dRho + geom.M);
    int *dSites = dSlotOf + nstot;
    const long long s = deviceStep();
    ck(cudaMemsetAsync(dRho, 0, 4 * geom.M, stream), "clear density scratch");
    if (!sites.empty())
        ck(cudaMemcpyAsync(dSites, sites.data(), 4 * sites.size(), cudaMemcpyHostToDevice, stream), "copy sites");
    ck(launch_slot_map(dOrig, (int)nstot, dSlotOf, dSites, (int)sites.size(), stream), "slot map");
    ck(launch_density_single(geom, ppHost, dX[s & 1], dSites, (int)sites.size(), dQ, charge, dRho, stream),
       "density");
    ck(cudaMemcpyAsync(rho, dRho, 4 * geom.M, cudaMemcpyDeviceToHost, stream), "read density");
    ck(cudaStreamSynchronize(stream), "density");
}

// S(k) of a group's density (ps_compute_sk.cu:18-50: rho^(k) rho^(-k) with the forward
// transform divided by M) for the current positions, binned by |k| in FP64.
void Box::structureFactor(const std::string &group, int charge, int nbins, double kmax, double *k_out,
                          double *sk_out, double *count_out)
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    if (nbins < 1 || nbins > (1 << 16)) fail(TILD_ERR_ARG, "nbins must be in [1, 65536]");
    if (!(kmax > 0.0)) fail(TILD_ERR_ARG, "kmax must be > 0");
    const int gi = findGroupInteger(group);
    if (charge && !psGroup[gi].isCharges) fail(TILD_ERR_ARG, "only the 'charges' group has a charge density");
    ck(cudaSetDevice(device), "cudaSetDevice");
    const long long s = deviceStep();
    const std::vector<int> orig = slotOrder();
    std::vector<int> slotOf(nstot);
    for (int64_t k = 0; k < nstot; k++) slotOf[orig[k]] = (int)k;
    std::vector<int> sites(psGroup[gi].siteList);
    for (int &v : sites) v = slotOf[v];
    const Geom &g = geom;
    int *dSites = nullptr;
    float *dRho = nullptr;
    float2 *dPair = nullptr, *dHs = nullptr;
    double *dBins = nullptr;
    cudaError_t e = cudaMalloc(&dSites, 4 * std::max<size_t>(1, sites.size()));
    if (e == cudaSuccess) e = cudaMalloc(&dRho, 4 * g.M);
    if (e == cudaSuccess) e = cudaMalloc(&dPair, 8 * g.M);
    if (e == cudaSuccess) e = cudaMalloc(&dHs, 8 * g.hstride);
    if (e == cudaSuccess) e = cudaMalloc(&dBins, 3 * sizeof(double) * nbins);
    if (e == cudaSuccess && !sites.empty())
        e = cudaMemcpy(dSites, sites.data(), 4 * sites.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemsetAsync(dRho, 0, 4 * g.M, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dBins, 0, 3 * sizeof(double) * nbins, stream);
    if (e == cudaSuccess)
        e = launch_density_single(g, ppHost, dX[s & 1], dSites, (int)sites.size(), dQ, charge, dRho, stream);
    if (e == cudaSuccess) e = launch_to_pairs(dRho, dPair, g.M, stream);
    if (e == cudaSuccess)
        e = launch_structure_factor(g, lx, ly, lz, ksHost.twopi_over_L, dPair, dHs, nbins, kmax / nbins, dBins, stream);
    std::vector<double> b(3 * (size_t)nbins, 0.0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = cudaMemcpy(b.data(), dBins, 3 * sizeof(double) * nbins, cudaMemcpyDeviceToHost);
    cudaFree(dSites);
    cudaFree(dRho);
    cudaFree(dPair);
    cudaFree(dHs);
    cudaFree(dBins);
    ck(e, "structure factor");
    for (int i = 0; i < nbins; i++) {
        const double n = b[3 * i + 2];
        if (sk_out) sk_out[i] = n > 0.0 ? b[3 * i] / n : 0.0;
        if (k_out) k_out[i] = n > 0.0 ? b[3 * i + 1] / n : (i + 0.5) * kmax / nbins;
        if (count_out) count_out[i] = n;
    }
}

void Box::gridWeights(int32_t *inds, float *w)
{
    if (!ready) fail(TILD_ERR_STATE, "endBox has not been processed");
    const long long s = deviceStep();
    const int G = (pmeorder + 1) * (pmeorder + 1) * (Dim == 3 ? pmeorder + 1 : 1);
    int *dI = nullptr;
    float *dW = nullptr, *dO = nullptr;
    ck(cudaMalloc(&dI, 4 * nstot * G), "malloc");
    ck(cudaMalloc(&dW, 4 * nstot * G), "malloc");
    ck(cudaMalloc(&dO, 4 * nstot * G), "malloc");
    cudaError_t e = launch_grid_weights(geom, pmeorder, exact4 ? 0 : 1, dX[s & 1], (int)nstot, dI, dW, stream);
    // rows of 4-byte values from slot order back to particle order (indices moved as raw bits)
    if (e == cudaSuccess) e = launch_unpermute_rows((int)nstot, G, dOrig, reinterpret_cast<float *>(dI), dO, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(inds, dO, 4 * nstot * G, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = launch_unpermute_rows((int)nstot, G, dOrig, dW, dO, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(w, dO, 4 * nstot * G, cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    cudaFree(dI);
    cudaFree(dW);
    cudaFree(dO);
    ck(e, "grid weights");
}

void Box::modifyBox(const std::string &rest)
{
    std::vector<std::string> w = split(rest);
    if (w.size() >= 3 && w[0] == "potential" && (w[1] == "remove" || w[1] == "delete")) {
        const long long id = std::strtoll(w[2].c_str(), nullptr, 10);
        if (id > 0 && id <= (long long)potentials.size()) {
            potentials.erase(potentials.begin() + (id - 1));
            if (ready) {   // positions, GJF state, RNG state and particle order are kept
                ck(cudaStreamSynchronize(stream), "sync");
                dropGraphs();
                const int ndOld = (int)dfields.size(), nfOld = (int)fgroups.size();
                buildPlan();
                if ((int)dfields.size() > std::max(1, ndOld) || (int)fgroups.size() > std::max(1, nfOld))
                    fail(TILD_ERR_STATE, "plan grew after removing a potential");
                recMapOk = false;   // the record descriptor follows the force-group count
                uploadFlags();
                ck(cudaDeviceSynchronize(), "modify");
            }
        }
    }
}

void Box::writeDataConfig(const std::string &name)   // PS_Box.cu:629-748
{
    std::vector<float> xs(x);
    if (ready) getPositions(xs.data());   // x[n*Dim]
    std::ofstream out(resolve(name));
    if (!out) fail(TILD_ERR_IO, "cannot write " + name);
    out << "Created by MATILDA.FT\n\n";
    out << nstot << " atoms" << "\n";
    out << nBondsTot << " bonds" << "\n";
    out << nAnglesTot << " angles" << "\n";
    out << "\n";
    int mx = -342332;
    for (int64_t p = 0; p < nstot; p++) mx = std::max(mx, intSpecies[p]);
    out << mx + 1 << " atom types" << "\n";
    mx = -1;
    for (int64_t p = 0; p < nstot; p++)
        for (int b = 0; b < nBonds[p]; b++) mx = std::max(mx, bondType[p * MAXBONDS + b]);
    out << mx + 1 << " bond types" << "\n";
    mx = -1;
    for (int64_t p = 0; p < nstot && nAnglesTot > 0; p++)
        for (int a = 0; a < nAngles[p]; a++) mx = std::max(mx, angleType[p * MAXANGLES + a]);
    out << mx + 1 << " angle types" << "\n";
    out << "\n";
    out << "0.0 " << L[0] << " xlo xhi" << "\n";
    out << "0.0 " << L[1] << " ylo yhi" << "\n";
    if (Dim > 2) out << "0.0 " << L[2] << " zlo zhi" << "\n";
    else out << "0.0 1.0 zlo zhi" << "\n";
    out << "\n";
    out << "Masses\n" << "\n";
    for (size_t t = 0; t < species.size(); t++) out << t + 1 << " " << species[t].mass << "\n";
    out << "\n";
    out << "Atoms\n" << std::endl;
    for (int64_t p = 0; p < nstot; p++) {
        out << p + 1 << " " << mID[p] + 1 << " " << intSpecies[p] + 1 << "  ";
        if (doCharges) out << charges[p] << " ";
        for (int j = 0; j < Dim; j++) out << xs[p * Dim + j] << " ";
        if (Dim < 3) out << "0.0 ";
        out << "\n";
    }
    out << "\n";
    out << "Bonds\n" << "\n";
    int64_t bc = 0;
    for (int64_t p = 0; p < nstot; p++)
        for (int b = 0; b < nBonds[p]; b++)
            if (p < bondedTo[p * MAXBONDS + b]) {
                out << bc + 1 << " " << bondType[p * MAXBONDS + b] + 1 << " " << p + 1 << " " << bondedTo[p * MAXBONDS + b] + 1 << "\n";
                bc++;
            }
    if (nAnglesTot > 0) {   // PS_Box.cu:728-745: each angle once, from its first particle
        out << "\nAngles\n" << "\n";
        int64_t ac = 0;
        for (int64_t p = 0; p < nstot; p++)
            for (int a = 0; a < nAngles[p]; a++) {
                const int *gq = &angleGroup[(p * MAXANGLES + a) * 3];
                if (p == gq[0]) {
                    out << ac + 1 << " " << angleType[p * MAXANGLES + a] + 1 << " " << gq[0] + 1 << " " << gq[1] + 1
                        << " " << gq[2] + 1 << "\n";
                    ac++;
                }
            }
    }
}

std::string Box::describe() const
{
    auto q = [](const std::string &v) {
        std::string o = "\"";
        for (char c : v) {
            if (c == '"' || c == '\\') o += '\\';
            o += c;
        }
        return o + "\"";
    };
    std::ostringstream j;
    j.precision(9);
    j << "{\"ready\": " << (ready ? "true" : "false") << ", \"Dim\": " << Dim << ", \"nstot\": " << nstot
      << ", \"grid\": [" << Nx[0] << ", " << Nx[1] << ", " << Nx[2] << "], \"L\": [" << L[0] << ", " << L[1] << ", "
      << L[2] << "], \"pmeorder\": " << pmeorder << ", \"randSeed\": " << RANDSEED << ", \"logFreq\": " << logFreq
      << ", \"doCharges\": " << (doCharges ? "true" : "false") << ", \"MAXBONDS\": " << MAXBONDS
      << ", \"nBonds\": " << nBondsTot << ", \"nAngles\": " << nAnglesTot << ", \"MAXANGLES\": " << MAXANGLES
      << ", \"datFileName\": " << q(datFileName) << ", \"tiles\": {\"codes\": " << tiles.codes
      << ", \"threads\": " << (gatherThreads ? gatherThreads : tiles.threads) << ", \"gather\": \"" << (tiles.direct ? "direct" : "staged")
      << "\", \"deposit_codes\": " << dtiles.codes << ", \"deposit_threads\": " << depTileCfg().threads
      << ", \"autotuned\": " << (autotune ? "true" : "false")
      << ", \"tuned_ms\": " << tunedMs << "}, \"trajFreq\": " << trajFreq
      << ", \"trajFileName\": " << q(trajFileName) << ", \"fieldFreq\": " << fieldFreq
      << ", \"logScaleFields\": " << (logSpaceFields ? logScaleFields : 0.f) << ", \"gsdFreq\": " << gsdFreq
      << ", \"logScaleGSD\": " << (logSpaceGSD ? logScaleGSD : 0.f) << ", \"gsdName\": " << q(gsdName)
      << ", \"species\": [";
    for (size_t t = 0; t < species.size(); t++)
        j << (t ? ", " : "") << "{\"label\": " << q(species[t].label) << ", \"mass\": " << species[t].mass
          << ", \"mobility\": " << species[t].mobility << "}";
    j << "], \"bonds\": [";
    for (int t = 0; t < nBondTypes; t++)
        j << (t ? ", " : "") << "{\"style\": " << bondStyle[t] << ", \"k\": " << bondK[t] << ", \"req\": " << bondReq[t] << "}";
    j << "], \"groups\": [";
    for (size_t g = 0; g < psGroup.size(); g++)
        j << (g ? ", " : "") << "{\"name\": " << q(psGroup[g].name) << ", \"nsites\": " << psGroup[g].siteList.size()
          << ", \"force\": " << (psGroup[g].forceFlag ? "true" : "false") << "}";
    j << "], \"potentials\": [";
    for (size_t k = 0; k < potentials.size(); k++) {
        const PS_Potential &p = potentials[k];
        j << (k ? ", " : "") << "{\"kind\": " << q(p.word) << ", \"I\": " << q(p.grpI) << ", \"J\": " << q(p.grpJ)
          << ", \"A\": " << p.Ao << ", \"sigma\": " << p.sigma << ", \"Rp\": " << p.Rp << ", \"lB\": " << p.LB
          << ", \"ramp\": " << (p.ramp ? "true" : "false") << ", \"A_final\": " << p.Ao_final << "}";
    }
    j << "], \"integrators\": [";
    for (size_t k = 0; k < integrators.size(); k++)
        j << (k ? ", " : "") << "{\"group\": " << q(integrators[k].groupName) << ", \"name\": " << q(integrators[k].name)
          << ", \"delt\": " << integrators[k].delt << "}";
    j << "]}";
    return j.str();
}

}  // namespace tild
