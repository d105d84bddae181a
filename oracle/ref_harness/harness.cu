// harness.cu -- test infrastructure: drives the UNMODIFIED MATILDA.FT PS_Box (built from
// the reference sources in place, see Makefile) and dumps what the reference computes,
// so the oracle and the B200 path can be pinned against the reference's own CUDA build.
//
//   tild_ref_harness <script> <outdir> <nsteps> [time_steps] [nvt|script]
//
// With "nvt" the <nsteps> steps run through PS_Box::NVT (PS_Box.cu:210-234), which adds the
// run's closing outputs (final writeData, writeFields, writeGSDtraj, final.input.data) to
// the per-step ones doTimeStep writes at the script's frequencies.  With "script" the
// lines after endBox are executed as main.cu:96-151 executes them (`run nvt N` through
// PS_Box::NVT, `modify ...` through PS_Box::modifyBox) and <nsteps> is ignored.
//
// Runs in the current directory (readData paths are relative to it, as in main.cu).
// Dumps (raw little-endian arrays + meta.txt) into <outdir>:
//   gridInds.i32, gridW.f32        d_calcGridWeights tables after finishInitialization
//   rho_<group>.f32, rhoq_charges.f32   every group's density (PS_Box_initialization.cu:551-559)
//   f0.f32                         d_f after cudaMemset(0) + PS_Box::forces()
//   energies.f64                   Ubond, then CalcEnergy() of each potential
//   uangle.f64                     Uangle
//   x_final.f32                    d_x after <nsteps> doTimeStep calls (or the script's runs)
//   energies_final.f64             Ubond, then CalcEnergy() of each remaining potential,
//                                  after them (computeThermoProps)
// With time_steps > 0 it also times that many further doTimeStep calls with CUDA events
// and prints "ms_per_step <value>".  An <outdir> of "-" writes nothing (timing runs).
#define MAIN
#include "timing.h"
#include "random.h"
#include "Box.h"
#include "PS_Box.h"

#include <cstdio>
#include <string>
#include <vector>

std::vector<Box*> box;
Box* BoxFactory(std::istringstream&);
std::string giveQuote() { return std::string(); }

static void dump(const std::string& dir, const std::string& name, const void* dptr, size_t bytes)
{
    if (dir == "-") return;
    std::vector<char> h(bytes);
    cudaMemcpy(h.data(), dptr, bytes, cudaMemcpyDeviceToHost);
    FILE* fp = fopen((dir + "/" + name).c_str(), "wb");
    if (!fp) { fprintf(stderr, "cannot write %s\n", name.c_str()); exit(2); }
    fwrite(h.data(), 1, bytes, fp);
    fclose(fp);
}

static void dump_host(const std::string& dir, const std::string& name, const void* p, size_t bytes)
{
    if (dir == "-") return;
    FILE* fp = fopen((dir + "/" + name).c_str(), "wb");
    fwrite(p, 1, bytes, fp);
    fclose(fp);
}

int main(int argc, char** argv)
{
    if (argc < 4) { fprintf(stderr, "usage: %s script outdir nsteps [time_steps]\n", argv[0]); return 1; }
    const std::string out = argv[2];
    const int nsteps = atoi(argv[3]);
    const int tsteps = argc > 4 ? atoi(argv[4]) : 0;
    const bool nvt = argc > 5 && std::string(argv[5]) == "nvt";
    const bool script = argc > 5 && std::string(argv[5]) == "script";
    std::ifstream in(argv[1]);
    if (!in) { fprintf(stderr, "cannot open %s\n", argv[1]); return 1; }
    std::string line, word;
    while (std::getline(in, line)) {            // main.cu:96-111, first box only
        if (line.empty() || line[0] == '#') continue;
        std::istringstream iss(line);
        iss >> word;
        if (word == "box") {
            box.push_back(BoxFactory(iss));
            box.back()->readInput(in);
            break;
        }
    }
    if (box.empty()) { fprintf(stderr, "no box in script\n"); return 1; }
    PS_Box* b = dynamic_cast<PS_Box*>(box[0]);
    if (!b) { fprintf(stderr, "not a PS box\n"); return 1; }
    cudaDeviceSynchronize();
    const int N = b->nstot, D = b->returnDimension(), G = b->gridPerPartic, M = b->M;
    FILE* meta = fopen(out == "-" ? "/dev/null" : (out + "/meta.txt").c_str(), "w");
    fprintf(meta, "N %d\nDim %d\nG %d\nM %d\ngvol %.17g\nngroups %d\nnpot %d\n", N, D, G, M, b->gvol,
            (int)b->psGroup.size(), (int)b->potentials.size());
    dump(out, "gridInds.i32", b->d_gridInds, sizeof(int) * (size_t)N * G);
    dump(out, "gridW.f32", b->d_gridW, sizeof(float) * (size_t)N * G);
    for (size_t g = 0; g < b->psGroup.size(); g++) {
        const std::string nm = b->psGroup[g].returnName();
        fprintf(meta, "group %s\n", nm.c_str());
        dump(out, "rho_" + nm + ".f32", b->psGroup[g].d_rho, sizeof(float) * (size_t)M);
        if (nm == "charges") dump(out, "rhoq_charges.f32", b->psGroup[g].d_rhoq, sizeof(float) * (size_t)M);
    }
    cudaMemset(b->d_f, 0, sizeof(float) * (size_t)N * D);   // PS_Box.cu:122
    b->forces();                                            // PS_Box.cu:240-278
    cudaDeviceSynchronize();
    dump(out, "f0.f32", b->d_f, sizeof(float) * (size_t)N * D);
    b->computeThermoProps();                                // PS_Box.cu:282-317
    std::vector<double> e;
    e.push_back(b->Ubond);
    for (size_t k = 0; k < b->potentials.size(); k++) e.push_back(b->potentials[k]->energy);
    dump_host(out, "energies.f64", e.data(), e.size() * sizeof(double));
    const double ua = b->Uangle;                            // PS_Box.cu:296-305
    dump_host(out, "uangle.f64", &ua, sizeof(double));
    b->maxSteps = nsteps;
    if (script) {
        while (std::getline(in, line)) {                    // main.cu:96-151, after the box
            if (line.empty() || line[0] == '#') continue;
            std::istringstream iss(line);
            if (!(iss >> word)) continue;
            if (word == "run") {
                int n = 0;
                iss >> word >> n;
                if (word != "nvt") { fprintf(stderr, "unsupported run style %s\n", word.c_str()); return 1; }
                b->NVT(n);
            } else if (word == "modify") {
                b->modifyBox(iss);
            }
        }
    } else if (nvt) b->NVT(nsteps);
    else
        for (int i = 0; i < nsteps; i++) b->doTimeStep(i);  // PS_Box.cu:210-234 loop
    cudaDeviceSynchronize();
    dump(out, "x_final.f32", b->d_x, sizeof(float) * (size_t)N * D);
    b->computeThermoProps();
    e.clear();
    e.push_back(b->Ubond);
    for (size_t k = 0; k < b->potentials.size(); k++) e.push_back(b->potentials[k]->energy);
    dump_host(out, "energies_final.f64", e.data(), e.size() * sizeof(double));
    if (tsteps > 0) {
        b->logFreq = 1 << 30;                               // no thermo/I/O inside the timing
        b->maxSteps = nsteps + tsteps;
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        for (int i = 1; i <= tsteps; i++) b->doTimeStep(nsteps + i);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        printf("ms_per_step %.6f\n", ms / tsteps);
        fprintf(meta, "ms_per_step %.6f\n", ms / tsteps);
    }
    fprintf(meta, "cuda_error %s\n", cudaGetErrorString(cudaGetLastError()));
    fclose(meta);
    return 0;
}
