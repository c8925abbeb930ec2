// server.cu -- request loop with continuous batching (the serving mode).
//
// A request is a set of cells of one network, an interval and tolerances
// (host arrays, copied at submit).  A worker thread per server:
//  * admits waiting requests in arrival order while the device footprint of
//    the admitted ones stays under the HBM budget (admission by footprint);
//  * whenever one of `max_inflight` launch slots is free, merges every
//    admitted request that is not yet running -- of any network size -- into
//    ONE batch launch (mass-action groups share one persistent kernel,
//    builtin networks run beside it) on that slot's stream, followed by the
//    result copies to pinned host buffers and an event;
//  * requests that arrive while earlier batches run are launched on another
//    slot at once, so their work overlaps with the running kernels;
//  * polls the slots' events; a finished batch releases its device memory
//    (admitting more waiting requests) and completes its requests.
// Every wait is bounded: the worker sleeps on a condition variable for at
// most `poll_us`; wind_server_poll waits at most its timeout.
#include <algorithm>
#include <chrono>
#include <type_traits>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "api_internal.h"

namespace wind {

using Clock = std::chrono::steady_clock;

struct ServerRequest {
    int64_t id = 0;
    int kind = 0, N = 0, n_const = 0, n_react = 0;
    int64_t nsys = 0;
    double tnow = 0, tend = 0, atol = 0, rtol = 0;
    int32_t n_steps = 1;
    // host copies of the inputs
    std::vector<double> y0, constants, rates;
    std::vector<uint16_t> species;
    std::vector<float> linear;
    // device buffers while resident
    double *d_y = nullptr, *d_constants = nullptr, *d_rates = nullptr;
    uint16_t* d_species = nullptr;
    float* d_linear = nullptr;
    int32_t* d_status = nullptr;
    int64_t* d_nsteps = nullptr;
    // pinned results
    double* h_y = nullptr;
    int32_t* h_status = nullptr;
    int64_t* h_nsteps = nullptr;
    size_t footprint = 0;
    enum { WAITING, ADMITTED, RUNNING, DONE } state = WAITING;
    int result = WIND_OK;
    Clock::time_point t_submit, t_start, t_done;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<ServerRequest*> reqs;
    bool busy = false;
};

struct Server {
    wind_server_config cfg{};
    int device = 0;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<ServerRequest*> waiting;
    std::vector<ServerRequest*> admitted;
    std::unordered_map<int64_t, ServerRequest*> all;
    std::vector<Slot> slots;
    size_t resident = 0;
    int64_t next_id = 1;
    bool stop = false;
    int64_t launches = 0, completed = 0, systems_done = 0;
    int worker_error = WIND_OK;
};

// Device bytes a request holds while admitted: its state, network, status
// and step counters, and -- for mass action with N > 32 -- the per-block
// global scratch the CTA kernels take for what does not fit in shared
// memory (one slot per resident block: up to two blocks per SM), counted
// in full for every such request since each launch sizes it for its
// largest group.
static size_t footprint(const ServerRequest& r, const wind_server_config& cfg) {
    size_t b = r.nsys * (size_t)r.N * 8 + r.constants.size() * 8 + r.rates.size() * 8 +
               r.species.size() * 2 + r.linear.size() * 4 + r.nsys * 12 + 64 * 8;
    if (r.kind == WIND_NET_MASS_ACTION && r.N > wind::WIND_TEAM_MAX_EQ) {
        const int solver = (cfg.method == WIND_METHOD_RK2) ? WIND_SOLVER_LU_F64
                                                             : wind::resolve_solver(cfg.solver, r.kind, r.N);
        b += wind::cta_scratch_bytes_per_block(r.N, r.n_react, !r.linear.empty(), solver) *
             (size_t)wind::device_sm_count() * 2;
    }
    return b;
}

// Upload inputs and allocate outputs on `s` (stream-ordered pool).
static int upload(ServerRequest& r, cudaStream_t s) {
    auto up = [&](auto** dst, const auto& v) -> bool {
        using T = std::remove_reference_t<decltype(**dst)>;
        if (v.empty()) { *dst = nullptr; return true; }
        if (cudaMallocAsync((void**)dst, v.size() * sizeof(T), s) != cudaSuccess) return false;
        return cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s) == cudaSuccess;
    };
    if (!up(&r.d_y, r.y0) || !up(&r.d_constants, r.constants) || !up(&r.d_rates, r.rates) ||
        !up(&r.d_species, r.species) || !up(&r.d_linear, r.linear))
        return WIND_ERR_NOMEM;
    if (cudaMallocAsync((void**)&r.d_status, r.nsys * sizeof(int32_t), s) != cudaSuccess ||
        cudaMallocAsync((void**)&r.d_nsteps, r.nsys * sizeof(int64_t), s) != cudaSuccess)
        return WIND_ERR_NOMEM;
    return WIND_OK;
}

static void release_device(ServerRequest& r, cudaStream_t s) {
    for (void* p : {(void*)r.d_y, (void*)r.d_constants, (void*)r.d_rates, (void*)r.d_species,
                    (void*)r.d_linear, (void*)r.d_status, (void*)r.d_nsteps})
        if (p) cudaFreeAsync(p, s);
    r.d_y = r.d_constants = r.d_rates = nullptr;
    r.d_species = nullptr;
    r.d_linear = nullptr;
    r.d_status = nullptr;
    r.d_nsteps = nullptr;
}

static void release_host(ServerRequest& r) {
    if (r.h_y) cudaFreeHost(r.h_y);
    if (r.h_status) cudaFreeHost(r.h_status);
    if (r.h_nsteps) cudaFreeHost(r.h_nsteps);
    r.h_y = nullptr;
    r.h_status = nullptr;
    r.h_nsteps = nullptr;
}

static wind_group group_of(const ServerRequest& r) {
    wind_group g;
    std::memset(&g, 0, sizeof(g));
    g.net.kind = r.kind;
    g.net.n_eq = r.N;
    g.net.n_const = r.n_const;
    g.net.n_react = r.n_react;
    g.net.constants = r.d_constants;
    g.net.rates = r.d_rates;
    g.net.species = r.d_species;
    g.net.linear = r.d_linear;
    g.y = r.d_y;
    g.nsys = r.nsys;
    g.tnow = r.tnow;
    g.tend = r.tend;
    g.n_integration_steps = r.n_steps;
    g.atol = r.atol;
    g.rtol = r.rtol;
    g.sys_status = r.d_status;
    g.sys_nsteps = r.d_nsteps;
    return g;
}

static void worker_main(Server* S) {
    cudaSetDevice(S->device);
    wind_options o;
    wind_default_options(&o);
    o.method = S->cfg.method;
    o.solver = S->cfg.solver;
    o.controller = S->cfg.controller;
    while (true) {
        std::vector<ServerRequest*> batch;
        Slot* slot = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            // admission by device footprint, in arrival order
            while (!S->waiting.empty() &&
                   (S->resident + S->waiting.front()->footprint <= (size_t)S->cfg.hbm_budget_bytes ||
                    S->resident == 0)) {
                ServerRequest* r = S->waiting.front();
                S->waiting.pop_front();
                S->resident += r->footprint;
                r->state = ServerRequest::ADMITTED;
                S->admitted.push_back(r);
            }
            if (!S->admitted.empty()) {
                for (Slot& sl : S->slots)
                    if (!sl.busy) { slot = &sl; break; }
            }
            if (slot) {
                const size_t take = std::min<size_t>(S->admitted.size(), WIND_SERVER_MAX_GROUPS);
                batch.assign(S->admitted.begin(), S->admitted.begin() + take);
                S->admitted.erase(S->admitted.begin(), S->admitted.begin() + take);
                for (ServerRequest* r : batch) {
                    r->state = ServerRequest::RUNNING;
                    r->t_start = Clock::now();
                }
                slot->busy = true;
                slot->reqs = batch;
            } else {
                bool any_busy = false;
                for (Slot& sl : S->slots) any_busy |= sl.busy;
                if (S->stop && !any_busy && S->admitted.empty() && S->waiting.empty()) return;
                if (!any_busy)
                    S->cv_work.wait_for(lk, std::chrono::microseconds(S->cfg.poll_us));
            }
        }
        if (slot) {
            // upload, one merged launch, result copies, completion event
            int st = WIND_OK;
            std::vector<wind_group> groups;
            for (ServerRequest* r : batch) {
                if (st == WIND_OK) st = upload(*r, slot->stream);
                groups.push_back(group_of(*r));
            }
            if (st == WIND_OK) st = launch_batch(o, groups.data(), (int)groups.size(), slot->stream);
            for (ServerRequest* r : batch) {
                if (st != WIND_OK) break;
                cudaMemcpyAsync(r->h_y, r->d_y, r->nsys * (size_t)r->N * 8, cudaMemcpyDeviceToHost, slot->stream);
                cudaMemcpyAsync(r->h_status, r->d_status, r->nsys * 4, cudaMemcpyDeviceToHost, slot->stream);
                cudaMemcpyAsync(r->h_nsteps, r->d_nsteps, r->nsys * 8, cudaMemcpyDeviceToHost, slot->stream);
            }
            for (ServerRequest* r : batch) r->result = st;
            cudaEventRecord(slot->done, slot->stream);
            std::lock_guard<std::mutex> lk(S->mu);
            S->launches++;
        }
        // completion of in-flight batches
        for (Slot& sl : S->slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) continue;
            const Clock::time_point now = Clock::now();
            for (ServerRequest* r : sl.reqs) release_device(*r, sl.stream);
            std::lock_guard<std::mutex> lk(S->mu);
            for (ServerRequest* r : sl.reqs) {
                if (q != cudaSuccess && r->result == WIND_OK) r->result = WIND_ERR_CUDA;
                r->state = ServerRequest::DONE;
                r->t_done = now;
                S->resident -= r->footprint;
                S->completed++;
                S->systems_done += r->nsys;
            }
            sl.reqs.clear();
            sl.busy = false;
            S->cv_done.notify_all();
        }
        if (!slot) {
            bool any_busy = false;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                for (Slot& sl : S->slots) any_busy |= sl.busy;
            }
            if (any_busy) std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
}

}  // namespace wind

using namespace wind;

extern "C" {

void wind_server_default_config(wind_server_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->method = WIND_METHOD_SIE;
    c->solver = WIND_SOLVER_LU_F64;
    c->controller = WIND_CTRL_DEVICE;
    c->hbm_budget_bytes = (int64_t)16 << 30;
    c->max_inflight = 4;
    c->max_waiting = 1 << 16;
    c->poll_us = 200;
}

int wind_server_create(const wind_server_config* cfg, wind_server** out) {
    if (!out) return WIND_ERR_ARGUMENT;
    *out = nullptr;
    wind_server_config c;
    if (cfg) c = *cfg; else wind_server_default_config(&c);
    if (c.max_inflight < 1 || c.max_inflight > 64 || c.hbm_budget_bytes <= 0 || c.max_waiting < 1)
        return WIND_ERR_ARGUMENT;
    // the batch kernels' method, solver and controller (no fixed-step SIM)
    wind_options oc;
    wind_default_options(&oc);
    oc.method = c.method;
    oc.solver = c.solver;
    oc.controller = c.controller;
    if (check_options(oc) != WIND_OK || oc.solver == WIND_SOLVER_MIXED_TC) return WIND_ERR_ARGUMENT;
    if (c.poll_us <= 0) c.poll_us = 200;
    Server* S = new Server();
    S->cfg = c;
    if (cudaGetDevice(&S->device) != cudaSuccess) { delete S; return WIND_ERR_CUDA; }
    S->slots.resize(c.max_inflight);
    for (Slot& sl : S->slots) {
        if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess) {
            for (Slot& t : S->slots) {
                if (t.stream) cudaStreamDestroy(t.stream);
                if (t.done) cudaEventDestroy(t.done);
            }
            delete S;
            return WIND_ERR_CUDA;
        }
    }
    S->worker = std::thread(worker_main, S);
    *out = reinterpret_cast<wind_server*>(S);
    return WIND_OK;
}

int wind_server_submit(wind_server* srv, const wind_request* q, int64_t* id_out) {
    Server* S = reinterpret_cast<Server*>(srv);
    if (!S || !q || !id_out || !q->y0 || q->nsys <= 0 || q->n_integration_steps < 1) return WIND_ERR_ARGUMENT;
    const wind_status ns = check_network(&q->net, q->nsys);
    if (ns != WIND_OK) return ns;
    auto* r = new ServerRequest();
    r->kind = q->net.kind;
    r->N = q->net.n_eq;
    r->n_const = q->net.n_const;
    r->n_react = q->net.n_react;
    r->nsys = q->nsys;
    r->tnow = q->tnow;
    r->tend = q->tend;
    r->atol = q->atol;
    r->rtol = q->rtol;
    r->n_steps = q->n_integration_steps;
    r->y0.assign(q->y0, q->y0 + q->nsys * (size_t)r->N);
    if (q->net.constants) r->constants.assign(q->net.constants, q->net.constants + q->nsys * (size_t)r->n_const);
    if (q->net.rates) r->rates.assign(q->net.rates, q->net.rates + q->nsys * (size_t)r->n_react);
    if (q->net.species) {
        r->species.assign(q->net.species, q->net.species + q->nsys * (size_t)r->n_react * 4);
        for (uint16_t v : r->species)
            if (v >= r->N) { delete r; return WIND_ERR_ARGUMENT; }
    }
    if (q->net.linear) r->linear.assign(q->net.linear, q->net.linear + q->nsys * (size_t)r->N * r->N);
    r->footprint = footprint(*r, S->cfg);
    // pinned result buffers, taken in the caller's thread so the worker's
    // launch path stays free of host allocations
    if (cudaMallocHost((void**)&r->h_y, r->nsys * (size_t)r->N * sizeof(double)) != cudaSuccess ||
        cudaMallocHost((void**)&r->h_status, r->nsys * sizeof(int32_t)) != cudaSuccess ||
        cudaMallocHost((void**)&r->h_nsteps, r->nsys * sizeof(int64_t)) != cudaSuccess) {
        release_host(*r);
        delete r;
        return WIND_ERR_NOMEM;
    }
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if ((int64_t)S->waiting.size() >= S->cfg.max_waiting || S->stop) {
            release_host(*r);
            delete r;
            return WIND_ERR_BUSY;
        }
        r->id = S->next_id++;
        S->all[r->id] = r;
        S->waiting.push_back(r);
    }
    S->cv_work.notify_one();
    *id_out = r->id;
    return WIND_OK;
}

int wind_server_poll(wind_server* srv, int64_t id, double timeout_s, double* y_out, int32_t* status_out,
                     int64_t* nsteps_out, double* latency_s) {
    Server* S = reinterpret_cast<Server*>(srv);
    if (!S) return WIND_ERR_ARGUMENT;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return WIND_ERR_NOT_FOUND;
    ServerRequest* r = it->second;
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                             std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 0));
    while (r->state != ServerRequest::DONE) {
        if (timeout_s <= 0 || S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
            if (r->state != ServerRequest::DONE) return WIND_ERR_TIMEOUT;
        }
    }
    const int result = r->result;
    if (result == WIND_OK) {
        if (y_out) std::memcpy(y_out, r->h_y, r->nsys * (size_t)r->N * sizeof(double));
        if (status_out) std::memcpy(status_out, r->h_status, r->nsys * sizeof(int32_t));
        if (nsteps_out) std::memcpy(nsteps_out, r->h_nsteps, r->nsys * sizeof(int64_t));
    }
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    S->all.erase(it);
    lk.unlock();
    release_host(*r);
    delete r;
    return result;
}

int wind_server_stats(wind_server* srv, int64_t* out6) {
    Server* S = reinterpret_cast<Server*>(srv);
    if (!S || !out6) return WIND_ERR_ARGUMENT;
    std::lock_guard<std::mutex> lk(S->mu);
    out6[0] = (int64_t)S->waiting.size();
    out6[1] = (int64_t)S->admitted.size();
    int64_t running = 0;
    for (Slot& sl : S->slots) running += (int64_t)sl.reqs.size();
    out6[2] = running;
    out6[3] = S->completed;
    out6[4] = S->launches;
    out6[5] = (int64_t)S->resident;
    return WIND_OK;
}

int wind_server_destroy(wind_server* srv) {
    Server* S = reinterpret_cast<Server*>(srv);
    if (!S) return WIND_ERR_ARGUMENT;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    if (S->worker.joinable()) S->worker.join();
    for (Slot& sl : S->slots) {
        cudaStreamSynchronize(sl.stream);
        cudaStreamDestroy(sl.stream);
        cudaEventDestroy(sl.done);
    }
    for (auto& kv : S->all) {
        release_host(*kv.second);
        delete kv.second;
    }
    delete S;
    return WIND_OK;
}

}  // extern "C"
