// tild_batch.h -- replicas stepped together, one launch per step stage over all of them.
// No counterpart in the reference, which runs one box per process (main.cu:63-76) and
// steps it alone (PS_Box.cu:73-207).
//
// A batch holds boxes (endBox processed) that share the kernels' compile-time settings:
// 3-D, the same spline order, one or two density fields, one or two force groups, the
// same deterministic mode, the tile gather over paired records.  Their sizes, grids,
// potentials, tiles and integrators may all differ.  Every step stage -- zeroing the
// deposit targets, the deposit, the five transform passes, the tile gather, the integrator
// pass, the step counters -- is ONE launch whose CTAs are dealt over the replicas' work by
// a prefix table of CTA counts; each replica's geometry, FFT plans, tile lists, record
// layout, TMA descriptors and arrays sit in a device table.  The ten launches of a step are
// captured once in a CUDA graph.  Every sort_interval steps each replica's spatial re-sort
// runs as a branch of one more graph.
//
// With `streams` > 1 the replicas are split into that many groups of about equal work,
// each with its own table, graphs and stream: a step is then one launch per stage per
// group, and the groups' stages overlap on the GPU (a deposit of one group beside a
// transform of another), which uses the GPU better than stages taken one at a time.
#pragma once

#include <vector>

#include "tild_box.h"

namespace tild {

class Batch {
public:
    explicit Batch(int device);
    ~Batch();
    void add(Box *box);         // a box whose endBox has been processed, on this batch's device
    void setStreams(int k);     // groups of replicas stepped on their own streams (1..8)
    void step(int64_t n);       // n steps of every replica, no logging or output files
    int size() const { return (int)boxes.size(); }

private:
    struct Group {
        std::vector<Box *> reps;                 // in table (dispatch) order
        cudaStream_t stream = nullptr;
        int txz = 0;
        BatchRep *dReps = nullptr;
        int *dPre = nullptr;                     // the stages' prefix tables, (R + 1) ints each
        BatchLaunch launches[BS_COUNT + 1];      // + the zeroing of the deposit targets
        cudaGraphExec_t gStep = nullptr, gSort = nullptr;
    };
    void build();
    void buildGroup(Group &g);
    void release();

    int device;
    int nstreams = 1;
    std::vector<Box *> boxes;
    std::vector<Group> groups;
    std::vector<cudaStream_t> forks;             // branches of the re-sort graphs
    bool built = false;
    int order = 0, nd = 0, nfg = 0, deterministic = 0, extra = 0, sortInterval = 0, sinceSort = 0;
};

}  // namespace tild
