// vfd_serve.cu -- request loop with continuous batching for diffusion solves.
//
// Requests (a world of fields, a number of ticks, sources) are queued by
// vfd_server_submit from any thread.  One scheduler thread owns the device:
//   * admission, FIFO: the head request is admitted while the active set has
//     a free slot and its device bytes fit the HBM budget; its fields are
//     created resident (host upload or the device generator) and stay on the
//     device for all its ticks;
//   * a round advances every active request by one tick: all their fields go
//     through one launch per axis pass per substep (vfd_batch, replayed as a
//     CUDA graph while the active set is unchanged);
//   * while a round runs, the requests finishing with it are known: new
//     arrivals are admitted into their slots and the next round's batch is
//     built on the host; after the round the finished requests are retired
//     (totals, optional download) and their memory is freed, so new arrivals
//     join while others are still on the device.
// The reference has no serving layer: it diffuses one world per tick from
// WHWorld::go (woundHealingWorld.cpp:2013-2026).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "vfd.h"

namespace {

struct Request {
    uint64_t id = 0;
    // copies of the description
    int nx = 0, ny = 0, nz = 0, nf = 0, pad_mode = 0, epi = 0, ticks = 0;
    std::vector<vfd_field_params> params;
    std::vector<const float *> init;  // empty: synthetic
    uint64_t seed = 0;
    int synth_world = 0;
    float lo = 0.f, hi = 0.f;
    std::vector<std::vector<int32_t>> src_idx;
    std::vector<std::vector<float>> src_amt;
    std::vector<float *> result;
    vfd_mass *mass = nullptr;
    // state
    vfd_world *world = nullptr;
    size_t bytes = 0;
    int ticks_done = 0;
    vfd_request_info info;
    std::string err;
};

double latency_of(const vfd_request_info &i) { return i.t_done - i.t_submit; }

}  // namespace

struct vfd_server {
    int device = 0;
    size_t budget = 0;
    int max_active = 0;
    int substeps = 1;
    std::chrono::steady_clock::time_point t0;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::map<uint64_t, std::shared_ptr<Request>> finished;
    std::vector<double> latencies;
    uint64_t next_id = 1;
    bool stop = false;
    vfd_server_stats st;

    double busy_since = -1.0;  // start of the current busy span (under mu)

    // scheduler-owned
    std::vector<std::shared_ptr<Request>> active;
    std::vector<std::pair<vfd_world *, size_t>> dead;  // retired worlds not yet destroyed
    vfd_batch *batch = nullptr;
    bool set_changed = true;
    size_t in_use = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_round[2] = {nullptr, nullptr};  // brackets each round on `stream`
    std::thread worker;
    std::string err;

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

size_t estimate_bytes(const Request &r)
{
    // fields + per-axis tables (generous) + sources
    size_t b = sizeof(float) * (size_t)r.nx * r.ny * r.nz * r.nf;
    b += (size_t)r.nf * 3 * 4096 * sizeof(float) + 3 * 4096 * 8 + 64 * 1024;
    for (const auto &v : r.src_idx) b += v.size() * 8;
    return b;
}

void finish(vfd_server *s, const std::shared_ptr<Request> &r, int status, const std::string &msg)
{
    r->info.status = status;
    r->info.t_done = s->now();
    r->err = msg;
    std::lock_guard<std::mutex> lk(s->mu);
    s->finished[r->id] = r;
    if (status == VFD_OK) {
        s->st.completed++;
        s->st.voxel_steps_done += r->info.voxel_steps;
        s->latencies.push_back(latency_of(r->info));
    } else {
        s->st.rejected++;
    }
    s->cv_done.notify_all();
}

// Creates the request's world on the device (scheduler thread).
int admit(vfd_server *s, const std::shared_ptr<Request> &r, std::string &msg)
{
    vfd_world_desc d;
    d.nx = r->nx;
    d.ny = r->ny;
    d.nz = r->nz;
    d.n_fields = r->nf;
    d.fields = r->params.data();
    d.pad_mode = r->pad_mode;
    d.epi_boundary = r->epi;
    d.fft[0] = d.fft[1] = d.fft[2] = 0;
    d.method = VFD_METHOD_SEPARABLE;
    vfd_status st = vfd_world_create(&d, s->device, &r->world);
    if (st != VFD_OK) {
        msg = vfd_last_error(nullptr);
        r->world = nullptr;
        return st;
    }
    for (int f = 0; f < r->nf && st == VFD_OK; ++f) {
        if (!r->init.empty()) {
            st = vfd_upload_field(r->world, f, r->init[f], s->stream);
        } else {
            float *p = nullptr;
            st = vfd_field_device_ptr(r->world, f, &p);
            if (st == VFD_OK)
                st = vfd_synth_field_device(r->seed, r->synth_world, f, r->lo, r->hi, p,
                                            (size_t)r->nx * r->ny * r->nz, s->stream);
        }
        if (st == VFD_OK && !r->src_idx.empty())
            st = vfd_set_sources(r->world, f, r->src_idx[f].data(), r->src_amt[f].data(),
                                 (int64_t)r->src_idx[f].size());
    }
    if (st == VFD_OK) st = vfd_world_device_bytes(r->world, &r->bytes);
    if (st != VFD_OK) {
        msg = vfd_last_error(r->world);
        vfd_world_destroy(r->world);
        r->world = nullptr;
        return st;
    }
    r->src_idx.clear();  // copied to the device
    r->src_amt.clear();
    return VFD_OK;
}

// Reads a finished request's results; its world is destroyed later (`dead`),
// after the next round has been launched, because freeing device memory
// waits for the device.
int retire(vfd_server *s, const std::shared_ptr<Request> &r, std::string &msg)
{
    int st = VFD_OK;
    if (r->mass) st = vfd_read_mass(r->world, r->mass, s->stream);
    for (int f = 0; f < r->nf && st == VFD_OK && !r->result.empty(); ++f)
        if (r->result[f]) st = vfd_download_field(r->world, f, r->result[f], s->stream);
    if (st != VFD_OK) msg = vfd_last_error(r->world);
    s->dead.push_back({r->world, r->bytes});
    r->world = nullptr;
    return st;
}

// Destroys the worlds of retired requests and returns their memory to the budget.
void bury(vfd_server *s)
{
    if (s->dead.empty()) return;
    for (auto &d : s->dead) {
        vfd_world_destroy(d.first);
        s->in_use -= d.second;
    }
    s->dead.clear();
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.hbm_in_use = s->in_use;
}

// Takes requests off the queue while slots and budget allow (FIFO; a request
// larger than the whole budget is rejected).  `occupied`: slots in use.
std::vector<std::shared_ptr<Request>> select_admissions(vfd_server *s, int occupied, size_t used)
{
    std::vector<std::shared_ptr<Request>> out;
    std::unique_lock<std::mutex> lk(s->mu);
    int slots = s->max_active - occupied;
    while (!s->pending.empty() && slots > 0) {
        auto r = s->pending.front();
        const size_t est = estimate_bytes(*r);
        if (est > s->budget) {
            s->pending.pop_front();
            s->st.queued = (int64_t)s->pending.size();
            lk.unlock();
            finish(s, r, VFD_ERR_BUDGET, "request larger than the HBM budget");
            lk.lock();
            continue;
        }
        if (used + est > s->budget) break;  // FIFO: wait for memory
        used += est;
        out.push_back(r);
        s->pending.pop_front();
        --slots;
    }
    s->st.queued = (int64_t)s->pending.size();
    return out;
}

// Creates the worlds of selected requests; returns those that are resident.
std::vector<std::shared_ptr<Request>> admit_all(vfd_server *s, const std::vector<std::shared_ptr<Request>> &sel)
{
    std::vector<std::shared_ptr<Request>> ok;
    for (auto &r : sel) {
        std::string msg;
        r->info.t_admit = s->now();
        const int st = admit(s, r, msg);
        if (st != VFD_OK) {
            finish(s, r, st, msg);
            continue;
        }
        s->in_use += r->bytes;
        ok.push_back(r);
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.admitted++;
    }
    return ok;
}

// The scheduler overlaps host work with the device: while a round runs, the
// requests that finish with it are already known, so new requests are
// admitted and the next round's batch is built before the round ends; after
// it ends the finished requests are retired and the next round starts at once.
void scheduler(vfd_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        // ---- admission while the device is idle ----------------------------
        if (s->active.empty()) bury(s);
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty() || !s->active.empty(); });
            if (s->stop) break;
        }
        {
            auto got = admit_all(s, select_admissions(s, (int)s->active.size(), s->in_use));
            if (!got.empty()) s->set_changed = true;
            s->active.insert(s->active.end(), got.begin(), got.end());
        }
        if (s->active.empty()) {
            bury(s);
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->busy_since >= 0) {
                s->st.busy_s += s->now() - s->busy_since;
                s->busy_since = -1.0;
            }
            continue;
        }
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->busy_since < 0) s->busy_since = s->now();
        }
        if (s->set_changed || !s->batch) {
            if (s->batch) vfd_batch_destroy(s->batch);
            s->batch = nullptr;
            std::vector<vfd_world *> ws;
            for (auto &r : s->active) ws.push_back(r->world);
            if (vfd_batch_create(ws.data(), (int)ws.size(), &s->batch) != VFD_OK) {
                const std::string msg = vfd_batch_last_error(nullptr);
                for (auto &r : s->active) {
                    vfd_world_destroy(r->world);
                    r->world = nullptr;
                    s->in_use -= r->bytes;
                    finish(s, r, VFD_ERR_CUDA, msg);
                }
                s->active.clear();
                continue;
            }
            s->set_changed = false;
        }

        // ---- one round: every active request advances one tick -----------
        cudaEventRecord(s->ev_round[0], s->stream);
        vfd_status st = vfd_batch_tick(s->batch, s->substeps, s->stream);
        cudaEventRecord(s->ev_round[1], s->stream);

        // while it runs: admit into the slots of requests finishing now and
        // build the next round's batch
        std::vector<std::shared_ptr<Request>> survivors, joining;
        vfd_batch *next = nullptr;
        bool next_changed = false;
        if (st == VFD_OK) {
            for (auto &r : s->active)
                if (r->ticks_done + 1 < r->ticks) survivors.push_back(r);
            joining = admit_all(s, select_admissions(s, (int)survivors.size(), s->in_use));
            next_changed = survivors.size() != s->active.size() || !joining.empty();
            if (next_changed && survivors.size() + joining.size() > 0) {
                std::vector<vfd_world *> ws;
                for (auto &r : survivors) ws.push_back(r->world);
                for (auto &r : joining) ws.push_back(r->world);
                if (vfd_batch_create(ws.data(), (int)ws.size(), &next) != VFD_OK) next = nullptr;  // rebuilt later
            }
        }
        bury(s);  // last round's retired worlds (waits for the device)
        if (st == VFD_OK && cudaStreamSynchronize(s->stream) != cudaSuccess) st = VFD_ERR_CUDA;
        float round_ms = 0.0f;
        if (st == VFD_OK) cudaEventElapsedTime(&round_ms, s->ev_round[0], s->ev_round[1]);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->st.rounds++;
            s->st.device_s += 1e-3 * round_ms;
        }
        if (st != VFD_OK) {
            const std::string msg = vfd_batch_last_error(s->batch);
            for (auto &r : s->active) {
                vfd_world_destroy(r->world);
                r->world = nullptr;
                s->in_use -= r->bytes;
                finish(s, r, st, msg);
            }
            if (next) vfd_batch_destroy(next);
            vfd_batch_destroy(s->batch);
            s->batch = nullptr;
            s->active = joining;  // admitted during the failed round: not part of it
            s->set_changed = true;
        } else {
            for (auto &r : s->active) {
                r->ticks_done++;
                if (r->ticks_done >= r->ticks) {
                    std::string msg;
                    const int rs = retire(s, r, msg);
                    finish(s, r, rs, msg);
                }
            }
            if (next_changed) {
                vfd_batch_destroy(s->batch);
                s->batch = next;
                s->set_changed = next == nullptr;
                survivors.insert(survivors.end(), joining.begin(), joining.end());
                s->active.swap(survivors);
            }
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.active = (int64_t)s->active.size();
        s->st.hbm_in_use = s->in_use;
        s->st.hbm_peak = std::max(s->st.hbm_peak, s->in_use);
    }
    // shutdown: drop what is still resident
    if (s->batch) vfd_batch_destroy(s->batch);
    s->batch = nullptr;
    bury(s);
    for (auto &r : s->active) {
        vfd_world_destroy(r->world);
        r->world = nullptr;
    }
    s->active.clear();
}

}  // namespace

extern "C" {

vfd_status vfd_server_create(int device, size_t hbm_budget_bytes, int max_active, int substeps_per_tick,
                             vfd_server **out)
{
    if (!out || hbm_budget_bytes == 0 || max_active < 1 || substeps_per_tick < 1) return VFD_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return VFD_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return VFD_ERR_INVALID_ARG;
    vfd_server *s = new vfd_server();
    s->device = device;
    s->budget = hbm_budget_bytes;
    s->max_active = max_active;
    s->substeps = substeps_per_tick;
    s->t0 = std::chrono::steady_clock::now();
    memset(&s->st, 0, sizeof(s->st));
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_round[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev_round[1]);
    if (e != cudaSuccess) {
        for (auto &ev : s->ev_round)
            if (ev) cudaEventDestroy(ev);
        if (s->stream) cudaStreamDestroy(s->stream);
        cudaSetDevice(prev);
        delete s;
        return VFD_ERR_CUDA;
    }
    cudaSetDevice(prev);
    s->worker = std::thread(scheduler, s);
    *out = s;
    return VFD_OK;
}

vfd_status vfd_server_submit(vfd_server *s, const vfd_request_desc *d, uint64_t *id)
{
    if (!s || !d || !d->fields || d->n_fields < 1 || d->ticks < 1 || d->nx < 1 || d->ny < 1 || d->nz < 1)
        return VFD_ERR_INVALID_ARG;
    auto r = std::make_shared<Request>();
    r->nx = d->nx;
    r->ny = d->ny;
    r->nz = d->nz;
    r->nf = d->n_fields;
    r->pad_mode = d->pad_mode;
    r->epi = d->epi_boundary;
    r->ticks = d->ticks;
    r->params.assign(d->fields, d->fields + d->n_fields);
    if (d->init) r->init.assign(d->init, d->init + d->n_fields);
    r->seed = d->synth_seed;
    r->synth_world = d->synth_world;
    r->lo = d->synth_lo;
    r->hi = d->synth_hi;
    if (d->n_src && d->src_idx && d->src_amt) {
        r->src_idx.resize(r->nf);
        r->src_amt.resize(r->nf);
        for (int f = 0; f < r->nf; ++f) {
            const int64_t n = d->n_src[f];
            if (n < 0 || (n > 0 && (!d->src_idx[f] || !d->src_amt[f]))) return VFD_ERR_INVALID_ARG;
            r->src_idx[f].assign(d->src_idx[f], d->src_idx[f] + n);
            r->src_amt[f].assign(d->src_amt[f], d->src_amt[f] + n);
        }
    }
    if (d->result) r->result.assign(d->result, d->result + d->n_fields);
    r->mass = d->mass;
    memset(&r->info, 0, sizeof(r->info));
    r->info.voxel_steps = (double)r->nx * r->ny * r->nz * r->nf * (double)r->ticks * s->substeps;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return VFD_ERR_INVALID_ARG;
        r->id = s->next_id++;
        r->info.id = r->id;
        r->info.t_submit = s->now();
        r->info.status = -1;
        s->pending.push_back(r);
        s->st.submitted++;
        s->st.queued = (int64_t)s->pending.size();
    }
    s->cv_work.notify_one();
    if (id) *id = r->id;
    return VFD_OK;
}

vfd_status vfd_server_wait(vfd_server *s, uint64_t id, double timeout_s, vfd_request_info *info)
{
    if (!s) return VFD_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                        [&] { return s->finished.count(id) > 0; });
    if (!ok) return VFD_ERR_TIMEOUT;
    auto r = s->finished[id];
    if (info) *info = r->info;
    return (vfd_status)r->info.status;
}

vfd_status vfd_server_drain(vfd_server *s, double timeout_s)
{
    if (!s) return VFD_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
        return (int64_t)(s->st.completed + s->st.rejected) >= s->st.submitted;
    });
    return ok ? VFD_OK : VFD_ERR_TIMEOUT;
}

static double percentile(std::vector<double> v, double p)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = p * (double)(v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

vfd_status vfd_server_get_stats(vfd_server *s, vfd_server_stats *out)
{
    if (!s || !out) return VFD_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    if (s->busy_since >= 0) out->busy_s += s->now() - s->busy_since;
    out->p50_latency_s = percentile(s->latencies, 0.50);
    out->p99_latency_s = percentile(s->latencies, 0.99);
    double m = 0.0;
    for (double x : s->latencies) m += x;
    out->mean_latency_s = s->latencies.empty() ? 0.0 : m / (double)s->latencies.size();
    return VFD_OK;
}

double vfd_server_clock(const vfd_server *s) { return s ? s->now() : 0.0; }

vfd_status vfd_server_destroy(vfd_server *s)
{
    if (!s) return VFD_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    for (auto &ev : s->ev_round) cudaEventDestroy(ev);
    cudaStreamDestroy(s->stream);
    cudaSetDevice(prev);
    delete s;
    return VFD_OK;
}

}  // extern "C"
