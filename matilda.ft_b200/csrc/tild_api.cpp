// tild_api.cpp -- extern "C" boundary of the B200 TILD library (declared in
// include/tild_b200.h).  Converts C++ exceptions into status codes; never exits.
#include <algorithm>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "tild_b200.h"
#include "tild_batch.h"
#include "tild_box.h"
#include "tild_pool.h"

struct tild_box {
    tild::Box *impl;
};

struct tild_pool {
    tild::Pool *impl;
};

struct tild_batch {
    tild::Batch *impl;
};

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &m)
{
    g_err = m;
    return code;
}

template <typename F>
int guarded(F &&f)
{
    try {
        f();
        g_err.clear();
        return TILD_OK;
    } catch (const tild::BoxError &e) {
        return fail(e.code, e.msg);
    } catch (const std::bad_alloc &) {
        return fail(TILD_ERR_ARG, "host out of memory");
    } catch (const std::exception &e) {
        return fail(TILD_ERR_ARG, e.what());
    }
}

}  // namespace

extern "C" {

const char *tild_version(void) { return "tild-b200 1.0 (sm_100a)"; }

const char *tild_last_error(void) { return g_err.c_str(); }

int tild_box_create(int device, tild_box **out)
{
    if (!out) return fail(TILD_ERR_ARG, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) ndev = 0;
    if (device < 0 || (ndev > 0 && device >= ndev))   // main.cu:63-76
        return fail(TILD_ERR_ARG, "Device " + std::to_string(device) + " not found; only detecting " +
                                      std::to_string(ndev) + " devices");
    // The device is bound at endBox, so scripts can be parsed and checked without a GPU.
    return guarded([&] { *out = new tild_box{new tild::Box(device)}; });
}

int tild_box_destroy(tild_box *box)
{
    if (!box) return TILD_OK;
    if (box->impl && box->impl->inBatch) return fail(TILD_ERR_STATE, "the box belongs to a batch: destroy the batch first");
    delete box->impl;
    delete box;
    return TILD_OK;
}

#define NEED_BOX                                                   \
    if (!box || !box->impl) return fail(TILD_ERR_ARG, "box is NULL")

int tild_box_set_stream(tild_box *box, void *cuda_stream)
{
    NEED_BOX;
    return guarded([&] { box->impl->setStream(reinterpret_cast<cudaStream_t>(cuda_stream)); });
}

int tild_box_set_base_dir(tild_box *box, const char *dir)
{
    NEED_BOX;
    if (!dir) return fail(TILD_ERR_ARG, "dir is NULL");
    return guarded([&] { box->impl->setBaseDir(dir); });
}

int tild_box_command(tild_box *box, const char *line)
{
    NEED_BOX;
    if (!line) return fail(TILD_ERR_ARG, "line is NULL");
    return guarded([&] { box->impl->command(line); });
}

int tild_box_read_input(tild_box *box, const char *text)
{
    NEED_BOX;
    if (!text) return fail(TILD_ERR_ARG, "text is NULL");
    return guarded([&] {
        std::istringstream in(text);
        std::string line;
        bool ended = false;
        while (std::getline(in, line)) {
            std::istringstream w(line);
            std::string first, second;
            w >> first >> second;
            if (first == "box") {
                if (second != "ps") throw tild::BoxError{TILD_ERR_UNSUPPORTED, "box style '" + second + "' (only ps)"};
                continue;
            }
            box->impl->command(line);
            if (box->impl->initialized()) {
                ended = true;
                break;
            }
        }
        if (!ended) throw tild::BoxError{TILD_ERR_PARSE, "input ended before endBox"};
    });
}

int tild_box_set_particles(tild_box *box, int64_t n, const float *x, const int32_t *type, const int32_t *mol,
                           const float *q)
{
    NEED_BOX;
    return guarded([&] { box->impl->setParticles(n, x, type, mol, q); });
}

int tild_box_set_bonds(tild_box *box, int64_t nbonds, const int64_t *pairs, const int32_t *btype)
{
    NEED_BOX;
    return guarded([&] { box->impl->setBonds(nbonds, pairs, btype); });
}

int tild_box_set_angles(tild_box *box, int64_t nangles, const int64_t *triples, const int32_t *atype)
{
    NEED_BOX;
    return guarded([&] { box->impl->setAngles(nangles, triples, atype); });
}

int tild_box_set_option(tild_box *box, const char *key, int64_t value)
{
    NEED_BOX;
    if (!key) return fail(TILD_ERR_ARG, "key is NULL");
    return guarded([&] { box->impl->setOption(key, value); });
}

int tild_box_get_info(const tild_box *box, tild_box_info *out)
{
    NEED_BOX;
    if (!out) return fail(TILD_ERR_ARG, "out is NULL");
    const tild::Box &b = *box->impl;
    std::memset(out, 0, sizeof(*out));
    out->nstot = b.nstot;
    out->dim = b.Dim;
    for (int j = 0; j < 3; j++) {
        out->nx[j] = b.Nx[j];
        out->L[j] = b.L[j];
    }
    out->pmeorder = b.pmeorder;
    out->n_groups = (int32_t)b.psGroup.size();
    out->n_potentials = (int32_t)b.potentials.size();
    out->n_density_fields = b.nDensityFields();
    out->n_force_groups = b.nForceGroups();
    out->n_bond_types = b.nBondTypes;
    out->n_bonds = b.nBondsTot;
    out->step = b.totSteps;
    out->device_bytes = b.deviceBytes();
    return TILD_OK;
}

int tild_box_describe(const tild_box *box, char *buf, int64_t size, int64_t *needed)
{
    NEED_BOX;
    const std::string j = box->impl->describe();
    if (needed) *needed = (int64_t)j.size() + 1;
    if (buf && size > 0) {
        const size_t n = std::min<size_t>((size_t)size - 1, j.size());
        std::memcpy(buf, j.data(), n);
        buf[n] = '\0';
    }
    return TILD_OK;
}

int tild_box_run_nvt(tild_box *box, int64_t nsteps)
{
    NEED_BOX;
    if (nsteps < 0) return fail(TILD_ERR_ARG, "nsteps < 0");
    return guarded([&] { box->impl->NVT(nsteps); });
}

int tild_box_step(tild_box *box, int64_t nsteps)
{
    NEED_BOX;
    if (nsteps < 0) return fail(TILD_ERR_ARG, "nsteps < 0");
    return guarded([&] { box->impl->steps(nsteps); });
}

int tild_box_forces(tild_box *box, float *f_out)
{
    NEED_BOX;
    if (!f_out) return fail(TILD_ERR_ARG, "f_out is NULL");
    return guarded([&] { box->impl->forces(f_out); });
}

int tild_box_thermo(tild_box *box, double *out, int nout, int *nwritten)
{
    NEED_BOX;
    if (!out && nout > 0) return fail(TILD_ERR_ARG, "out is NULL");
    return guarded([&] {
        std::vector<double> t = box->impl->thermo();
        const int n = std::min<int>(nout, (int)t.size());
        for (int k = 0; k < n; k++) out[k] = t[k];
        if (nwritten) *nwritten = n;
    });
}

int tild_box_get_positions(tild_box *box, float *x_out)
{
    NEED_BOX;
    if (!x_out) return fail(TILD_ERR_ARG, "x_out is NULL");
    return guarded([&] { box->impl->getPositions(x_out); });
}

int tild_box_set_positions(tild_box *box, const float *x_in)
{
    NEED_BOX;
    if (!x_in) return fail(TILD_ERR_ARG, "x_in is NULL");
    return guarded([&] { box->impl->setPositions(x_in); });
}

int tild_box_get_density(tild_box *box, const char *group, int charge_channel, float *rho_out)
{
    NEED_BOX;
    if (!group || !rho_out) return fail(TILD_ERR_ARG, "NULL argument");
    return guarded([&] { box->impl->getDensity(group, charge_channel, rho_out); });
}

int tild_box_modify(tild_box *box, const char *rest)
{
    NEED_BOX;
    if (!rest) return fail(TILD_ERR_ARG, "NULL argument");
    return guarded([&] { box->impl->modifyBox(rest); });
}

int tild_box_get_grid_force(tild_box *box, const char *group, float *gf_out)
{
    NEED_BOX;
    if (!group || !gf_out) return fail(TILD_ERR_ARG, "NULL argument");
    return guarded([&] { box->impl->getGridForce(group, gf_out); });
}

int tild_box_get_density_noalloc(tild_box *box, const char *group, int charge_channel, float *rho_out)
{
    NEED_BOX;
    if (!group || !rho_out) return fail(TILD_ERR_ARG, "NULL argument");
    return guarded([&] { box->impl->getDensityNoAlloc(group, charge_channel, rho_out); });
}

int tild_box_structure_factor(tild_box *box, const char *group, int charge_channel, int32_t nbins, double kmax,
                              double *k_out, double *sk_out, double *count_out)
{
    NEED_BOX;
    if (!group) return fail(TILD_ERR_ARG, "NULL argument");
    return guarded([&] { box->impl->structureFactor(group, charge_channel, nbins, kmax, k_out, sk_out, count_out); });
}

int tild_box_grid_weights(tild_box *box, int32_t *inds_out, float *w_out)
{
    NEED_BOX;
    if (!inds_out || !w_out) return fail(TILD_ERR_ARG, "NULL argument");
    return guarded([&] { box->impl->gridWeights(inds_out, w_out); });
}

int tild_box_get_log(tild_box *box, double *out, int64_t *rows, int32_t *cols)
{
    NEED_BOX;
    const auto &L = box->impl->logRows;
    int32_t c = box->impl->logColumns();   // rows logged before a `modify` can be wider
    for (const auto &r : L) c = std::max(c, (int32_t)r.size());
    if (rows) *rows = (int64_t)L.size();
    if (cols) *cols = c;
    if (out)
        for (size_t r = 0; r < L.size(); r++)
            for (int32_t k = 0; k < c; k++) out[r * c + k] = k < (int32_t)L[r].size() ? L[r][k] : 0.0;
    return TILD_OK;
}

int tild_box_stage_times(tild_box *box, double *out, int nmax, int *n)
{
    NEED_BOX;
    std::vector<double> v;
    box->impl->stageTimes(v);
    const int k = std::min<int>(nmax, (int)v.size());
    for (int i = 0; i < k; i++) out[i] = v[i];
    if (n) *n = k;
    return TILD_OK;
}

// main.cu:21-156: box blocks, run nvt, modify; other top-level words are ignored.
int tild_run_script_file(const char *path, int device)
{
    if (!path) return fail(TILD_ERR_ARG, "path is NULL");
    std::ifstream in(path);
    if (!in) return fail(TILD_ERR_IO, std::string("cannot open ") + path);
    std::string dir = path;
    const size_t sl = dir.find_last_of('/');
    dir = (sl == std::string::npos) ? "." : dir.substr(0, sl);
    tild::Box *box = nullptr;
    int rc = guarded([&] {
        std::string line;
        while (std::getline(in, line)) {
            if (line.empty() || line[0] == '#') continue;
            std::istringstream iss(line);
            std::string word;
            iss >> word;
            if (word == "box") {
                std::string style;
                iss >> style;
                if (style == "fts") throw tild::BoxError{TILD_ERR_UNSUPPORTED, "fts boxes are outside the TILD step"};
                if (style != "ps") throw tild::BoxError{TILD_ERR_PARSE, style + " is not a valid box style yet"};
                if (box) throw tild::BoxError{TILD_ERR_UNSUPPORTED, "only one box per script"};
                box = new tild::Box(device);
                box->setBaseDir(dir);
                box->echo = true;
                while (!box->initialized() && std::getline(in, line)) box->command(line);
                if (!box->initialized()) throw tild::BoxError{TILD_ERR_PARSE, "input ended before endBox"};
            } else if (word == "run") {
                std::string kind;
                iss >> kind;
                if (!box) throw tild::BoxError{TILD_ERR_STATE, "run before any box"};
                if (kind == "nvt") {
                    long long n = 0;
                    iss >> n;
                    box->NVT(n);
                } else if (kind == "vt" || kind == "findspinodal" || kind == "findSpinodal") {
                    throw tild::BoxError{TILD_ERR_PARSE, "invalid box style trying to run const 'vt' simulation"};
                } else {
                    throw tild::BoxError{TILD_ERR_PARSE, kind + " is an invalid global command!"};
                }
            } else if (word == "modify") {
                if (!box) throw tild::BoxError{TILD_ERR_STATE, "modify before any box"};
                std::string rest;
                std::getline(iss, rest);
                box->modifyBox(rest);
            }
        }
    });
    delete box;
    return rc;
}


#define NEED_POOL                                                   \
    if (!pool || !pool->impl) return fail(TILD_ERR_ARG, "pool is NULL")

int tild_pool_create(int device, int64_t mem_budget_bytes, int32_t max_active, tild_pool **out)
{
    if (!out) return fail(TILD_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (mem_budget_bytes <= 0) return fail(TILD_ERR_ARG, "mem_budget_bytes must be > 0");
    return guarded([&] { *out = new tild_pool{new tild::Pool(device, mem_budget_bytes, max_active)}; });
}

int tild_pool_destroy(tild_pool *pool)
{
    if (!pool) return TILD_OK;
    delete pool->impl;
    delete pool;
    return TILD_OK;
}

int tild_pool_submit(tild_pool *pool, tild_box *box, int64_t nsteps, int64_t *job_id)
{
    NEED_POOL;
    if (!box || !box->impl) return fail(TILD_ERR_ARG, "box is NULL or already submitted");
    if (!job_id) return fail(TILD_ERR_ARG, "job_id is NULL");
    return guarded([&] {
        *job_id = pool->impl->submit(box->impl, nsteps);   // on an error the caller keeps the box
        box->impl = nullptr;
    });
}

int tild_pool_status(tild_pool *pool, int64_t job_id, int32_t *state, int64_t *steps_done, double *times3)
{
    NEED_POOL;
    return guarded([&] {
        int st = 0;
        int64_t d = 0;
        pool->impl->status(job_id, st, d, times3);
        if (state) *state = st;
        if (steps_done) *steps_done = d;
    });
}

int tild_pool_wait(tild_pool *pool, int64_t job_id)
{
    NEED_POOL;
    return guarded([&] { pool->impl->wait(job_id); });
}

int tild_pool_result(tild_pool *pool, int64_t job_id, float *x_out, double *thermo_out, int32_t nthermo,
                     int32_t *nwritten)
{
    NEED_POOL;
    return guarded([&] {
        int n = 0;
        pool->impl->result(job_id, x_out, thermo_out, nthermo, &n);
        if (nwritten) *nwritten = n;
    });
}

int tild_pool_cancel(tild_pool *pool, int64_t job_id)
{
    NEED_POOL;
    return guarded([&] { pool->impl->cancel(job_id); });
}

int tild_pool_set_budget(tild_pool *pool, int64_t mem_budget_bytes)
{
    NEED_POOL;
    return guarded([&] { pool->impl->setBudget(mem_budget_bytes); });
}

int tild_pool_release(tild_pool *pool, int64_t job_id)
{
    NEED_POOL;
    return guarded([&] { pool->impl->release(job_id); });
}

int tild_pool_stats(tild_pool *pool, int64_t *out, int32_t nout)
{
    NEED_POOL;
    if (!out) return fail(TILD_ERR_ARG, "out is NULL");
    return guarded([&] {
        std::vector<int64_t> v;
        pool->impl->stats(v);
        for (int32_t i = 0; i < nout && i < (int32_t)v.size(); i++) out[i] = v[i];
    });
}

// ---- batch ----
int tild_batch_create(int device, tild_batch **out)
{
    if (!out) return fail(TILD_ERR_ARG, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return fail(TILD_ERR_ARG, "Device " + std::to_string(device) + " not found");
    return guarded([&] { *out = new tild_batch{new tild::Batch(device)}; });
}

int tild_batch_destroy(tild_batch *batch)
{
    if (!batch) return TILD_OK;
    delete batch->impl;
    delete batch;
    return TILD_OK;
}

int tild_batch_add(tild_batch *batch, tild_box *box)
{
    if (!batch || !batch->impl) return fail(TILD_ERR_ARG, "batch is NULL");
    if (!box || !box->impl) return fail(TILD_ERR_ARG, "box is NULL or was handed to a pool");
    return guarded([&] { batch->impl->add(box->impl); });
}

int tild_batch_size(tild_batch *batch, int32_t *n)
{
    if (!batch || !batch->impl || !n) return fail(TILD_ERR_ARG, "batch or n is NULL");
    *n = batch->impl->size();
    return TILD_OK;
}

int tild_batch_set_streams(tild_batch *batch, int32_t streams)
{
    if (!batch || !batch->impl) return fail(TILD_ERR_ARG, "batch is NULL");
    return guarded([&] { batch->impl->setStreams(streams); });
}

int tild_batch_step(tild_batch *batch, int64_t nsteps)
{
    if (!batch || !batch->impl) return fail(TILD_ERR_ARG, "batch is NULL");
    if (nsteps < 0) return fail(TILD_ERR_ARG, "nsteps must be >= 0");
    return guarded([&] { batch->impl->step(nsteps); });
}

}  // extern "C"
