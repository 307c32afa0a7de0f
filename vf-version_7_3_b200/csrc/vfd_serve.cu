// vfd_serve.cu -- request loop with continuous batching for diffusion solves.
//
// Requests (a world of fields, a number of ticks, sources) are queued by
// vfd_server_submit from any thread.  One scheduler thread owns the device:
//   * admission, FIFO: the head request is admitted while the active set has
//     a free slot and its device bytes fit the HBM budget; its fields are
//     created resident (host upload or the device generator) and stay on the
//     device for all its ticks.  A world retired by an earlier request of the
//     same shape and parameters is reused (fields and sources re-initialised),
//     so a steady stream of requests allocates no device memory;
//   * a round advances every active request by one tick: all their fields go
//     through one launch per axis pass per substep (vfd_batch, replayed as a
//     CUDA graph while the active set is unchanged);
//   * up to kRoundsInFlight rounds are queued on the device: the set of the
//     next round is known when a round is launched (every request's tick
//     count is), so the host admits arrivals and builds the next batch while
//     earlier rounds run.  A request is retired (totals, optional download)
//     once the round holding its last tick has completed, on a stream of its
//     own, and its slot is free for the next admission;
//   * device memory is freed only while no round is in flight (freeing waits
//     for the device): retired worlds wait in a pool for reuse and are freed
//     when the device is idle or the budget needs their bytes.
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

constexpr int kRoundsInFlight = 4;

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
    int ticks_launched = 0;
    vfd_request_info info;
    std::string err;
};

double latency_of(const vfd_request_info &i) { return i.t_done - i.t_submit; }

// One round queued on the device.
struct Round {
    cudaEvent_t start = nullptr, end = nullptr;
    std::vector<std::shared_ptr<Request>> finishing;  // requests whose last tick this round holds
    std::vector<vfd_batch *> done_batches;            // batches this round was the last to use
};

// Worlds are reused by requests of the same shape and parameters.
std::string world_key(const Request &r)
{
    std::string k(reinterpret_cast<const char *>(r.params.data()), r.params.size() * sizeof(vfd_field_params));
    const int d[6] = {r.nx, r.ny, r.nz, r.nf, r.pad_mode, r.epi};
    k.append(reinterpret_cast<const char *>(d), sizeof(d));
    return k;
}

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
    std::map<uint64_t, double> open_submit;  // submitted, not finished: submit time
    std::vector<double> latencies;
    uint64_t next_id = 1;
    bool stop = false;
    vfd_server_stats st;

    double busy_since = -1.0;  // start of the current busy span (under mu)

    // scheduler-owned
    std::vector<std::shared_ptr<Request>> active;    // requests with ticks still to launch
    std::deque<Round> inflight;
    std::vector<cudaEvent_t> ev_pool;
    std::multimap<std::string, std::pair<vfd_world *, size_t>> pool;  // retired worlds, by key
    size_t pool_bytes = 0;
    std::vector<vfd_batch *> dead_batches;           // replaced batches, destroyed while idle
    vfd_batch *batch = nullptr;
    bool set_changed = true;
    size_t in_use = 0;                               // active + retiring + pooled world bytes
    cudaStream_t stream = nullptr;                   // rounds
    cudaStream_t rstream = nullptr;                  // retirement reads
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
    s->open_submit.erase(r->id);
    if (status == VFD_OK) {
        s->st.completed++;
        s->st.voxel_steps_done += r->info.voxel_steps;
        s->latencies.push_back(latency_of(r->info));
    } else {
        s->st.rejected++;
    }
    s->cv_done.notify_all();
}

cudaEvent_t take_event(vfd_server *s)
{
    if (!s->ev_pool.empty()) {
        cudaEvent_t e = s->ev_pool.back();
        s->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Fills the request's fields and sources into its world.
int fill(vfd_server *s, const std::shared_ptr<Request> &r)
{
    vfd_status st = VFD_OK;
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
        if (st == VFD_OK) {
            const bool has = !r->src_idx.empty();
            st = vfd_set_sources(r->world, f, has ? r->src_idx[f].data() : nullptr,
                                 has ? r->src_amt[f].data() : nullptr, has ? (int64_t)r->src_idx[f].size() : 0);
        }
    }
    return st;
}

// Puts the request's world on the device: a pooled world of the same key, or
// a new one (scheduler thread).  `reused` tells which.
int admit(vfd_server *s, const std::shared_ptr<Request> &r, bool *reused, std::string &msg)
{
    *reused = false;
    auto it = s->pool.find(world_key(*r));
    if (it != s->pool.end()) {
        r->world = it->second.first;
        r->bytes = it->second.second;
        s->pool_bytes -= r->bytes;
        s->pool.erase(it);
        *reused = true;
    } else {
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
        if ((st = vfd_world_device_bytes(r->world, &r->bytes)) != VFD_OK) {
            msg = vfd_last_error(r->world);
            vfd_world_destroy(r->world);
            r->world = nullptr;
            return st;
        }
    }
    const int st = fill(s, r);
    if (st != VFD_OK) {
        msg = vfd_last_error(r->world);
        if (*reused) {
            s->in_use -= r->bytes;  // a pooled world's bytes were counted already
            *reused = false;
        }
        vfd_world_destroy(r->world);  // only reached with no round using this world
        r->world = nullptr;
        return st;
    }
    r->src_idx.clear();  // copied to the device
    r->src_amt.clear();
    return VFD_OK;
}

// Reads a finished request's results (its last round has completed); its
// world goes to the pool.
int retire(vfd_server *s, const std::shared_ptr<Request> &r, std::string &msg)
{
    int st = VFD_OK;
    if (r->mass) st = vfd_read_mass(r->world, r->mass, s->rstream);
    for (int f = 0; f < r->nf && st == VFD_OK && !r->result.empty(); ++f)
        if (r->result[f]) st = vfd_download_field(r->world, f, r->result[f], s->rstream);
    if (st != VFD_OK) msg = vfd_last_error(r->world);
    s->pool.insert({world_key(*r), {r->world, r->bytes}});
    s->pool_bytes += r->bytes;
    r->world = nullptr;
    return st;
}

// Waits for the oldest round in flight, accounts its device time and retires
// the requests it finished.
void complete_oldest(vfd_server *s)
{
    Round rd = std::move(s->inflight.front());
    s->inflight.pop_front();
    float ms = 0.0f;
    const double tw = s->now();
    const bool ok = cudaEventSynchronize(rd.end) == cudaSuccess;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.host_wait_s += s->now() - tw;
    }
    if (ok) cudaEventElapsedTime(&ms, rd.start, rd.end);
    s->ev_pool.push_back(rd.start);
    s->ev_pool.push_back(rd.end);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.rounds++;
        s->st.device_s += 1e-3 * ms;
    }
    // a batch the round was the last to use keeps its arena and stream for
    // the next batch (its work is complete: nothing on the device waits)
    for (auto *b : rd.done_batches) vfd_batch_destroy(b);
    for (auto &r : rd.finishing) {
        std::string msg;
        const int st = ok ? retire(s, r, msg) : VFD_ERR_CUDA;
        if (!ok) {
            msg = "a round failed on the device";
            s->pool.insert({world_key(*r), {r->world, r->bytes}});
            s->pool_bytes += r->bytes;
            r->world = nullptr;
        }
        finish(s, r, st, msg);
    }
}

void complete_all(vfd_server *s)
{
    while (!s->inflight.empty()) complete_oldest(s);
}

// Frees pooled worlds and replaced batches; only with no round in flight.
void free_idle(vfd_server *s)
{
    complete_all(s);
    for (auto *b : s->dead_batches) vfd_batch_destroy(b);
    s->dead_batches.clear();
    for (auto &kv : s->pool) {
        vfd_world_destroy(kv.second.first);
        s->in_use -= kv.second.second;
    }
    s->pool.clear();
    s->pool_bytes = 0;
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.hbm_in_use = s->in_use;
}

// Takes requests off the queue while slots and budget allow (FIFO; a request
// larger than the whole budget is rejected).  A request that fits only once
// pooled worlds are freed gets them freed first (the pool's bytes count
// against the budget; a pooled world of its own shape is reused instead).
std::vector<std::shared_ptr<Request>> select_admissions(vfd_server *s, int occupied)
{
    std::vector<std::shared_ptr<Request>> out;
    std::map<std::string, size_t> taken;  // pooled worlds already promised, by key
    std::unique_lock<std::mutex> lk(s->mu);
    int slots = s->max_active - occupied;
    size_t used = s->in_use;
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
        const std::string key = world_key(*r);
        bool pooled = s->pool.count(key) > taken[key];
        if (!pooled && used + est > s->budget) {
            if (s->pool_bytes == 0) break;  // FIFO: wait for memory
            lk.unlock();
            free_idle(s);  // device idle: pooled worlds are freed
            lk.lock();
            taken.clear();
            used = s->in_use;
            for (auto &q : out) used += estimate_bytes(*q);
            if (used + est > s->budget) break;
        }
        if (pooled) taken[key]++;
        else used += est;
        out.push_back(r);
        s->pending.pop_front();
        --slots;
    }
    s->st.queued = (int64_t)s->pending.size();
    return out;
}

// Creates (or reuses) the worlds of selected requests; returns those that are resident.
std::vector<std::shared_ptr<Request>> admit_all(vfd_server *s, const std::vector<std::shared_ptr<Request>> &sel)
{
    std::vector<std::shared_ptr<Request>> ok;
    if (sel.empty()) return ok;
    const double t0 = s->now();
    struct Account {
        vfd_server *s;
        double t0;
        ~Account()
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->st.host_admit_s += s->now() - t0;
        }
    } account{s, t0};
    for (auto &r : sel) {
        std::string msg;
        bool reused = false;
        r->info.t_admit = s->now();
        const int st = admit(s, r, &reused, msg);
        if (st != VFD_OK) {
            finish(s, r, st, msg);
            continue;
        }
        if (!reused) s->in_use += r->bytes;
        ok.push_back(r);
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.admitted++;
    }
    return ok;
}

void note_busy(vfd_server *s, bool busy)
{
    std::lock_guard<std::mutex> lk(s->mu);
    if (busy && s->busy_since < 0) s->busy_since = s->now();
    if (!busy && s->busy_since >= 0) {
        s->st.busy_s += s->now() - s->busy_since;
        s->busy_since = -1.0;
    }
}

void scheduler(vfd_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        // ---- rounds: keep at most kRoundsInFlight queued ----------------------
        while ((int)s->inflight.size() >= kRoundsInFlight || (s->active.empty() && !s->inflight.empty())) {
            complete_oldest(s);
            if (s->active.empty()) break;
        }
        if (s->active.empty() && s->inflight.empty()) {
            note_busy(s, false);
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->pending.empty() && !s->stop) {
                // idle: return pooled memory while waiting
                lk.unlock();
                free_idle(s);
                lk.lock();
            }
            s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty(); });
            if (s->stop) break;
        }
        {
            auto got = admit_all(s, select_admissions(s, (int)s->active.size()));
            if (!got.empty()) s->set_changed = true;
            s->active.insert(s->active.end(), got.begin(), got.end());
        }
        if (s->active.empty()) continue;
        note_busy(s, true);
        if (s->set_changed || !s->batch) {
            // the old batch may still be used by rounds in flight: destroyed
            // when the last of them completes
            if (s->batch) {
                if (!s->inflight.empty()) s->inflight.back().done_batches.push_back(s->batch);
                else vfd_batch_destroy(s->batch);
            }
            s->batch = nullptr;
            std::vector<vfd_world *> ws;
            for (auto &r : s->active) ws.push_back(r->world);
            const double tb = s->now();
            const vfd_status bs = vfd_batch_create(ws.data(), (int)ws.size(), &s->batch);
            {
                std::lock_guard<std::mutex> lk(s->mu);
                s->st.host_batch_s += s->now() - tb;
            }
            if (bs != VFD_OK) {
                const std::string msg = vfd_batch_last_error(nullptr);
                complete_all(s);
                for (auto &r : s->active) {
                    vfd_world_destroy(r->world);
                    r->world = nullptr;
                    s->in_use -= r->bytes;
                    finish(s, r, VFD_ERR_CUDA, msg);
                }
                s->active.clear();
                s->batch = nullptr;
                continue;
            }
            s->set_changed = false;
        }

        // ---- launch one round: every active request advances one tick ------
        Round rd;
        rd.start = take_event(s);
        rd.end = take_event(s);
        cudaEventRecord(rd.start, s->stream);
        const vfd_status st = vfd_batch_tick(s->batch, s->substeps, s->stream);
        cudaEventRecord(rd.end, s->stream);
        if (st != VFD_OK) {
            const std::string msg = vfd_batch_last_error(s->batch);
            s->inflight.push_back(std::move(rd));
            complete_all(s);
            for (auto &r : s->active) {
                vfd_world_destroy(r->world);
                r->world = nullptr;
                s->in_use -= r->bytes;
                finish(s, r, st, msg);
            }
            s->active.clear();
            s->dead_batches.push_back(s->batch);
            s->batch = nullptr;
            s->set_changed = true;
            continue;
        }
        std::vector<std::shared_ptr<Request>> survivors;
        for (auto &r : s->active) {
            if (++r->ticks_launched >= r->ticks) rd.finishing.push_back(r);
            else survivors.push_back(r);
        }
        if (!rd.finishing.empty()) {
            s->active.swap(survivors);
            s->set_changed = true;
        }
        s->inflight.push_back(std::move(rd));
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.active = (int64_t)s->active.size();
        s->st.hbm_in_use = s->in_use;
        s->st.hbm_peak = std::max(s->st.hbm_peak, s->in_use);
    }
    // shutdown: finish the rounds in flight, drop what is still resident
    complete_all(s);
    for (auto &r : s->active) {
        vfd_world_destroy(r->world);
        r->world = nullptr;
    }
    s->active.clear();
    if (s->batch) s->dead_batches.push_back(s->batch);
    s->batch = nullptr;
    free_idle(s);
    for (auto e : s->ev_pool) cudaEventDestroy(e);
    s->ev_pool.clear();
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
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->rstream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        if (s->stream) cudaStreamDestroy(s->stream);
        if (s->rstream) cudaStreamDestroy(s->rstream);
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
        s->open_submit[r->id] = r->info.t_submit;
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
    const double t = s->now();
    if (s->busy_since >= 0) out->busy_s += t - s->busy_since;
    out->p50_completed_s = percentile(s->latencies, 0.50);
    out->p99_completed_s = percentile(s->latencies, 0.99);
    // every arrival: the unfinished ones with the time they have waited so far
    std::vector<double> all(s->latencies);
    for (const auto &kv : s->open_submit) all.push_back(t - kv.second);
    out->censored = (int64_t)s->open_submit.size();
    out->p50_latency_s = percentile(all, 0.50);
    out->p99_latency_s = percentile(all, 0.99);
    double m = 0.0;
    for (double x : all) m += x;
    out->mean_latency_s = all.empty() ? 0.0 : m / (double)all.size();
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
    cudaStreamDestroy(s->stream);
    cudaStreamDestroy(s->rstream);
    cudaSetDevice(prev);
    delete s;
    return VFD_OK;
}

}  // extern "C"
