// tild_pool.cpp -- scheduler of the job pool (tild_pool.h).
#include "tild_pool.h"

#include "tild_b200.h"

#include <algorithm>

namespace tild {

Pool::Pool(int dev, int64_t budgetBytes, int maxAct)
    : device(dev), budget(budgetBytes), maxActive(maxAct > 0 ? maxAct : 1 << 30),
      t0(std::chrono::steady_clock::now())
{
    worker = std::thread([this] { run(); });
}

Pool::~Pool()
{
    {
        std::lock_guard<std::mutex> lk(mu);
        stop = true;
        for (Job *j : queue) {   // never admitted: cancelled
            j->state = JOB_CANCELLED;
            j->err = "cancelled: the pool was destroyed";
            j->box.reset();
            nCancelled++;
        }
        queue.clear();
    }
    cvWork.notify_all();
    if (worker.joinable()) worker.join();
    if (memPool) {
        cudaSetDevice(device);
        cudaMemPoolDestroy(memPool);
    }
    cvDone.notify_all();
}

double Pool::now() const
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

Job *Pool::find(int64_t id) const
{
    auto it = jobs.find(id);
    if (it == jobs.end()) fail(TILD_ERR_ARG, "no job " + std::to_string(id) + " in this pool");
    return it->second.get();
}

int64_t Pool::submit(Box *box, int64_t nsteps)
{
    if (!box) fail(TILD_ERR_ARG, "box is NULL");
    if (nsteps < 0) fail(TILD_ERR_ARG, "nsteps must be >= 0");
    if (box->initialized()) fail(TILD_ERR_STATE, "submit a box before endBox: the pool allocates it on admission");
    box->prepareHost();   // script checks and the plan; nothing on the device yet
    const int64_t bytes = box->deviceBytesEstimate();
    auto j = std::make_unique<Job>();
    j->N = box->nstot;
    j->nsteps = nsteps;
    j->bytes = bytes;
    // chunks of about 2 ms of GPU work at ~1e9 particle-steps/s, at most 100 steps
    j->chunk = std::max<int64_t>(1, std::min<int64_t>(100, (int64_t)(2.0e6 / (double)std::max<int64_t>(1, j->N))));
    int64_t id;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (stop) fail(TILD_ERR_STATE, "the pool is shutting down");
        if (bytes > budget)
            fail(TILD_ERR_ARG, "the job needs about " + std::to_string(bytes) +
                                   " bytes of device memory; the pool's budget is " + std::to_string(budget));
        id = nextId++;
        j->id = id;
        j->box.reset(box);   // adopted: nothing below can fail
        box->setSharedDevice(true);
        j->tSubmit = now();
        queue.push_back(j.get());
        jobs[id] = std::move(j);
    }
    cvWork.notify_all();
    return id;
}

void Pool::status(int64_t id, int &state, int64_t &done, double *times3) const
{
    std::lock_guard<std::mutex> lk(mu);
    const Job *j = find(id);
    state = j->state;
    done = j->done;
    if (times3) {
        times3[0] = j->tSubmit;
        times3[1] = j->tAdmit;
        times3[2] = j->tDone;
    }
}

void Pool::wait(int64_t id)
{
    std::unique_lock<std::mutex> lk(mu);
    Job *j = find(id);
    cvDone.wait(lk, [&] { return j->state == JOB_DONE || j->state == JOB_FAILED || j->state == JOB_CANCELLED; });
    if (j->state == JOB_FAILED) fail(TILD_ERR_STATE, "job " + std::to_string(id) + " failed: " + j->err);
    if (j->state == JOB_CANCELLED) fail(TILD_ERR_STATE, "job " + std::to_string(id) + " was cancelled");
}

void Pool::cancel(int64_t id)
{
    std::unique_ptr<Box> drop;   // a queued job's box, freed after the lock (host memory only)
    {
        std::lock_guard<std::mutex> lk(mu);
        Job *j = find(id);
        if (j->state == JOB_DONE || j->state == JOB_FAILED || j->state == JOB_CANCELLED)
            fail(TILD_ERR_STATE, "job " + std::to_string(id) + " has already finished");
        auto it = std::find(queue.begin(), queue.end(), j);
        if (it != queue.end()) {   // never admitted: nothing on the device yet
            queue.erase(it);
            drop = std::move(j->box);
            j->state = JOB_CANCELLED;
            j->err = "cancelled";
            j->tDone = now();
            nCancelled++;
            cvDone.notify_all();
        } else {
            // being admitted or running: the scheduler thread drains its in-flight chunks,
            // frees its arena and reports it cancelled
            j->cancel = true;
        }
    }
    cvWork.notify_all();
}

void Pool::setBudget(int64_t bytes)
{
    if (bytes < 0) fail(TILD_ERR_ARG, "the budget must be >= 0");
    {
        std::lock_guard<std::mutex> lk(mu);
        budget = bytes;
        failOversizedLocked();
    }
    cvWork.notify_all();
}

// Queued jobs that can never fit the budget fail now instead of blocking the queue.
void Pool::failOversizedLocked()
{
    for (auto it = queue.begin(); it != queue.end();) {
        Job *j = *it;
        if (j->bytes > budget) {
            j->state = JOB_FAILED;
            j->err = "the job needs about " + std::to_string(j->bytes) + " bytes of device memory; the pool's budget is now " +
                     std::to_string(budget);
            j->tDone = now();
            j->box.reset();
            nFailed++;
            it = queue.erase(it);
        } else {
            ++it;
        }
    }
    cvDone.notify_all();
}

void Pool::result(int64_t id, float *x, double *thermo, int nthermo, int *nwritten)
{
    std::lock_guard<std::mutex> lk(mu);
    Job *j = find(id);
    if (j->state == JOB_FAILED) fail(TILD_ERR_STATE, "job " + std::to_string(id) + " failed: " + j->err);
    if (j->state != JOB_DONE) fail(TILD_ERR_STATE, "job " + std::to_string(id) + " has not finished");
    if (x) std::copy(j->x.begin(), j->x.end(), x);
    const int k = thermo ? std::min<int>(nthermo, (int)j->thermo.size()) : 0;
    for (int i = 0; i < k; i++) thermo[i] = j->thermo[i];
    if (nwritten) *nwritten = k;
}

void Pool::release(int64_t id)
{
    std::lock_guard<std::mutex> lk(mu);
    Job *j = find(id);
    if (j->state != JOB_DONE && j->state != JOB_FAILED && j->state != JOB_CANCELLED)
        fail(TILD_ERR_STATE, "job " + std::to_string(id) + " is still in the pool");
    jobs.erase(id);
}

void Pool::stats(std::vector<int64_t> &out) const
{
    std::lock_guard<std::mutex> lk(mu);
    int64_t running = 0;
    for (auto &kv : jobs) running += kv.second->state == JOB_RUNNING;
    out = {(int64_t)queue.size(), running, nDone, nFailed, inUse, budget, nCancelled};
}

// ---- scheduler thread ----

void Pool::failJob(Job *j, const std::string &msg)
{
    dropEvents(j);
    j->box.reset();
    std::lock_guard<std::mutex> lk(mu);
    inUse -= j->bytes;
    j->err = msg;
    j->state = JOB_FAILED;
    j->tDone = now();
    nFailed++;
    cvDone.notify_all();
}

// A running job whose cancel was requested: let its in-flight chunks finish (each is a
// bounded number of captured steps), then free its arena like a finished job's.
void Pool::finishCancel(Job *j)
{
    cudaStreamSynchronize(j->box->cudaStreamHandle());
    dropEvents(j);
    j->box.reset();
    std::lock_guard<std::mutex> lk(mu);
    inUse -= j->bytes;
    j->err = "cancelled";
    j->state = JOB_CANCELLED;
    j->tDone = now();
    nCancelled++;
    cvDone.notify_all();
}

void Pool::dropEvents(Job *j)
{
    for (auto &e : j->inflight) cudaEventDestroy(e.first);
    for (auto e : j->spare) cudaEventDestroy(e);
    j->inflight.clear();
    j->spare.clear();
}

bool Pool::admit(Job *j)
{
    try {
        j->box->setSharedDevice(true, memPool);
        j->box->initDevice();
        for (int k = 0; k < 2; k++) {
            cudaEvent_t e;
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
                fail(TILD_ERR_CUDA, "cudaEventCreate failed");
            j->spare.push_back(e);
        }
    } catch (const BoxError &e) {
        failJob(j, e.msg);
        return false;
    }
    std::lock_guard<std::mutex> lk(mu);
    j->state = JOB_RUNNING;
    j->tAdmit = now();
    return true;
}

void Pool::harvest(Job *j)
{
    std::vector<float> x((size_t)j->box->Dim * j->N);
    std::vector<double> th;
    try {
        j->box->getPositions(x.data());
        th = j->box->thermo();
    } catch (const BoxError &e) {
        failJob(j, e.msg);
        return;
    }
    dropEvents(j);
    j->box.reset();   // stream-ordered frees: no device-wide synchronisation
    std::lock_guard<std::mutex> lk(mu);
    j->x.swap(x);
    j->thermo.swap(th);
    inUse -= j->bytes;
    j->state = JOB_DONE;
    j->tDone = now();
    nDone++;
    cvDone.notify_all();
}

// Retire the job's finished chunks and keep two chunks in flight on its stream.
void Pool::pump(Job *j, bool &progressed)
{
    while (!j->inflight.empty()) {
        const cudaError_t q = cudaEventQuery(j->inflight.front().first);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) fail(TILD_ERR_CUDA, std::string("job step: ") + cudaGetErrorString(q));
        j->done += j->inflight.front().second;
        j->spare.push_back(j->inflight.front().first);
        j->inflight.pop_front();
        progressed = true;
    }
    while (j->inflight.size() < 2 && j->issued < j->nsteps) {
        const int64_t k = std::min(j->chunk, j->nsteps - j->issued);
        j->box->steps(k);
        cudaEvent_t e = j->spare.back();
        j->spare.pop_back();
        if (cudaEventRecord(e, j->box->cudaStreamHandle()) != cudaSuccess) fail(TILD_ERR_CUDA, "cudaEventRecord failed");
        j->inflight.push_back({e, k});
        j->issued += k;
        progressed = true;
    }
}

void Pool::run()
{
    // the jobs' arenas come from one memory pool that keeps freed memory (up to the
    // budget) for the next jobs instead of returning it to the driver; without a GPU the
    // failure surfaces when a job is admitted
    if (cudaSetDevice(device) == cudaSuccess) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        if (cudaMemPoolCreate(&memPool, &props) == cudaSuccess) {
            uint64_t keep = (uint64_t)budget;
            cudaMemPoolSetAttribute(memPool, cudaMemPoolAttrReleaseThreshold, &keep);
        } else {
            memPool = nullptr;
            cudaGetLastError();
        }
    }
    for (;;) {
        std::vector<Job *> toAdmit;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (stop && queue.empty() && active.empty()) break;
            failOversizedLocked();
            // at most two admissions per pass, so the running jobs keep getting work while
            // new ones are set up
            while (!queue.empty() && toAdmit.size() < 2 && (int)(active.size() + toAdmit.size()) < maxActive &&
                   inUse + queue.front()->bytes <= budget) {
                Job *j = queue.front();
                queue.pop_front();
                inUse += j->bytes;
                toAdmit.push_back(j);
            }
            if (active.empty() && toAdmit.empty()) {
                cvWork.wait(lk, [&] { return stop || !queue.empty(); });
                continue;
            }
        }
        for (Job *j : toAdmit)
            if (admit(j)) active.push_back(j);
        bool progressed = !toAdmit.empty();
        for (size_t i = 0; i < active.size();) {
            Job *j = active[i];
            if (j->cancel) {
                finishCancel(j);
                active.erase(active.begin() + i);
                progressed = true;
                continue;
            }
            bool finished = false;
            try {
                pump(j, progressed);
                finished = j->done == j->nsteps && j->inflight.empty();
            } catch (const BoxError &e) {
                failJob(j, e.msg);
                active.erase(active.begin() + i);
                progressed = true;
                continue;
            }
            if (finished) {
                harvest(j);
                active.erase(active.begin() + i);
                progressed = true;
                continue;
            }
            ++i;
        }
        if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

}  // namespace tild
