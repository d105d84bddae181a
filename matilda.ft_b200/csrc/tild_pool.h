// tild_pool.h -- many TILD jobs on one GPU: admission against a device-memory budget and
// continuous batching of their steps.  No counterpart in the reference, which runs one
// box per process.
//
// A job is a configured box (script and particles given, endBox not yet processed) and a
// step count.  A scheduler thread admits queued jobs in arrival order while their
// estimated device memory fits the budget (and the active count stays under max_active),
// allocates them with stream-ordered allocations, and keeps two chunks of steps in flight
// on each job's own stream, so the jobs' graphs overlap on the GPU.  A finished job's
// positions and thermo are copied to the host, its device memory is freed, and the next
// queued job can enter at once.
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "tild_box.h"

namespace tild {

enum JobState { JOB_QUEUED = 0, JOB_RUNNING = 1, JOB_DONE = 2, JOB_FAILED = 3, JOB_CANCELLED = 4 };

struct Job {
    int64_t id = 0;
    std::unique_ptr<Box> box;
    int64_t nsteps = 0, issued = 0;       // issued: scheduler thread only
    std::atomic<int64_t> done{0};         // steps finished on the GPU (read by status())
    std::atomic<bool> cancel{false};      // a cancel request for a running job
    int64_t bytes = 0, N = 0, chunk = 1;
    int state = JOB_QUEUED;               // written under the pool's mutex
    double tSubmit = 0.0, tAdmit = 0.0, tDone = 0.0;   // seconds since the pool was created
    std::deque<std::pair<cudaEvent_t, int64_t>> inflight;   // chunk end events and their steps
    std::vector<cudaEvent_t> spare;
    std::vector<float> x;         // final positions, particle order
    std::vector<double> thermo;   // final thermo, tild_box_thermo layout
    std::string err;
};

class Pool {
public:
    Pool(int device, int64_t budgetBytes, int maxActive);
    ~Pool();
    int64_t submit(Box *box, int64_t nsteps);   // adopts the box only when it succeeds
    void status(int64_t id, int &state, int64_t &done, double *times3) const;
    void wait(int64_t id);
    void result(int64_t id, float *x, double *thermo, int nthermo, int *nwritten);
    void release(int64_t id);
    void cancel(int64_t id);                       // queued: dropped; running: drained, then freed
    void setBudget(int64_t bytes);                 // admissions from now on; running jobs stay
    // queued, running, done, failed, bytes in use, budget, cancelled
    void stats(std::vector<int64_t> &out) const;

private:
    void run();
    bool admit(Job *j);
    void pump(Job *j, bool &progressed);
    void harvest(Job *j);
    void failJob(Job *j, const std::string &msg);
    void finishCancel(Job *j);
    void failOversizedLocked();
    void dropEvents(Job *j);
    double now() const;
    Job *find(int64_t id) const;

    int device;
    int64_t budget;
    int maxActive;
    mutable std::mutex mu;
    std::condition_variable cvWork, cvDone;
    std::map<int64_t, std::unique_ptr<Job>> jobs;
    std::deque<Job *> queue;
    std::vector<Job *> active;   // touched by the scheduler thread only
    int64_t inUse = 0, nextId = 1;
    int nDone = 0, nFailed = 0, nCancelled = 0;
    bool stop = false;
    cudaMemPool_t memPool = nullptr;   // arenas of the jobs; keeps freed memory up to the budget
    std::chrono::steady_clock::time_point t0;
    std::thread worker;
};

}  // namespace tild
