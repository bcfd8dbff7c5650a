// server.cpp -- continuous-batching request loop over libgwb200 handles.
//
// A server owns `slots` worker threads on one device; each worker owns one gwb200_handle (its own
// CUDA stream and resident buffers) with a device-memory limit of hbm_budget / slots.  Requests
// (one G0W0 solve each: system + grid size + states) wait in a FIFO and are admitted as soon as a
// worker is free; a request whose smallest footprint (V_ph + its states' panel rows + one frequency
// of the tall matrices) exceeds a slot's budget is rejected with GWB200_OOM.  Requests in
// different slots run concurrently on different streams, so their kernels overlap on the GPU.
// Every kernel is deterministic and a request's arithmetic does not depend on its chunking, so
// a result is bit-identical whether the request ran alone or in a mix.
//
// No counterpart in the reference (it runs one molecule per process).
#include <atomic>
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

#include "internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct Job {
    int64_t ticket;
    gwb200_request req;
    std::vector<int64_t> states;  // copied at submit
    Clock::time_point submitted;
};

struct Result {
    bool done = false;
    int status = GWB200_OK;
    std::string message;
    double queue_ms = 0.0, service_ms = 0.0, device_ms = 0.0;
};

} // namespace

struct gwb200_server {
    int device = 0;
    int slots = 1;
    size_t slot_budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Job> queue;
    std::map<int64_t, Result> results;
    int64_t next_ticket = 1;
    bool stopping = false;
    std::vector<std::thread> workers;
    std::atomic<int> workers_ready{0};
    std::string start_error;
    // the workers' exact-size buffers come from this pool, which keeps up to the budget reserved so
    // that requests reuse memory instead of re-mapping it
    cudaMemPool_t pool = nullptr;
};

namespace {

// Resident V_ph and panel rows of the request's states (gwb200_load_system_states) plus one
// frequency of the tall matrices.
size_t min_footprint(const gwb200_request& r) {
    const size_t nmo = (size_t)r.nmo, nocc = (size_t)r.nocc, n = nocc * (nmo - nocc);
    const size_t m = (size_t)r.nstates * nmo;
    const size_t n64 = (n + 63) / 64 * 64, m64 = (m + 63) / 64 * 64;
    const size_t per = (r.eta != 0.0 ? 2 : 1) * (n64 + m64) * n64 * sizeof(double);
    return n * n * sizeof(double) + m * n * sizeof(double) + nmo * nocc * sizeof(double) + per;
}

void worker_main(gwb200_server* s) {
    gwb200_handle* h = nullptr;
    int rc = gwb200_create(s->device, &h);
    if (rc == GWB200_OK) rc = gwb200_set_memory_limit(h, (int64_t)s->slot_budget);
    if (rc == GWB200_OK) {
        gwb200_attach_pool(h, s->pool);
        gwb200_share_sms(h, s->slots);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (rc != GWB200_OK && s->start_error.empty()) s->start_error = gwb200_last_error();
        s->workers_ready.fetch_add(1);
    }
    s->cv_done.notify_all();
    if (rc != GWB200_OK) {
        gwb200_destroy(h);
        return;
    }
    for (;;) {
        Job job;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stopping || !s->queue.empty(); });
            if (s->queue.empty()) break;  // stopping with nothing left
            job = std::move(s->queue.front());
            s->queue.pop_front();
        }
        const auto start = Clock::now();
        Result res;
        res.queue_ms = std::chrono::duration<double, std::milli>(start - job.submitted).count();
        const gwb200_request& r = job.req;
        int st = gwb200_load_system_states(h, r.nmo, r.nocc, r.mo_energy, r.eri, r.vxc, r.fermi_energy,
                                           job.states.data(), (int64_t)job.states.size());
        gwb200_stats stats{};
        if (st == GWB200_OK)
            st = gwb200_run_g0w0(h, r.nfreq, r.npade, job.states.data(), (int64_t)job.states.size(), r.eta, r.precision,
                                 r.omega_out, r.weight_out, r.sigma_out, r.sigma_x_out, r.qp_out, &stats);
        res.status = st;
        if (st != GWB200_OK) res.message = gwb200_last_error();
        res.service_ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
        res.device_ms = stats.device_ms_total;
        res.done = true;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->results[job.ticket] = std::move(res);
        }
        s->cv_done.notify_all();
    }
    gwb200_destroy(h);
}

} // namespace

extern "C" {

int gwb200_server_create(int device, int slots, int64_t hbm_budget_bytes, gwb200_server** out) {
    if (!out || slots <= 0 || hbm_budget_bytes <= 0) return GWB200_BAD_ARGUMENT;
    auto* s = new gwb200_server();
    s->device = device;
    s->slots = slots;
    s->slot_budget = (size_t)hbm_budget_bytes / (size_t)slots;
    {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        if (cudaSetDevice(device) != cudaSuccess || cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) {
            cudaGetLastError();
            delete s;
            *out = nullptr;
            return gwb200_fail_status(GWB200_CUDA_ERROR, "server start: cannot create a device memory pool");
        }
        uint64_t keep = (uint64_t)hbm_budget_bytes;
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        // Never make one worker's stream wait for another's free to reuse a block (that would
        // serialise the slots); reuse a block across streams only once its free has completed.
        int off = 0, on = 1;
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolReuseAllowInternalDependencies, &off);
        cudaMemPoolSetAttribute(s->pool, cudaMemPoolReuseAllowOpportunistic, &on);
        // Map the whole budget now (one allocation, freed at once; the release threshold keeps it
        // in the pool): growing the pool while requests run stalled every slot for about a second
        // whenever a new peak of concurrent use was reached.  Best effort: on failure the pool
        // grows on demand as before.
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
            void* p = nullptr;
            if (cudaMallocFromPoolAsync(&p, (size_t)hbm_budget_bytes, s->pool, st) == cudaSuccess) cudaFreeAsync(p, st);
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        cudaGetLastError();
    }
    for (int i = 0; i < slots; ++i) s->workers.emplace_back(worker_main, s);
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] { return s->workers_ready.load() == slots; });
    }
    if (!s->start_error.empty()) {
        const std::string msg = s->start_error;
        gwb200_server_destroy(s);
        *out = nullptr;
        return gwb200_fail_status(GWB200_CUDA_ERROR, ("server start: " + msg).c_str());
    }
    *out = s;
    return GWB200_OK;
}

int gwb200_server_submit(gwb200_server* s, const gwb200_request* req, int64_t* ticket) {
    if (!s || !req || !ticket) return gwb200_fail_status(GWB200_BAD_ARGUMENT, "null server, request or ticket");
    if (req->nmo <= 0 || req->nocc <= 0 || req->nocc >= req->nmo || req->nfreq <= 0 || req->npade <= 0 ||
        req->nstates <= 0 || !req->states)
        return gwb200_fail_status(GWB200_BAD_SHAPE, "request: bad nmo/nocc/nfreq/npade/states");
    if (min_footprint(*req) > s->slot_budget)
        return gwb200_fail_status(GWB200_OOM, "request does not fit one slot's device-memory budget");
    Job job;
    job.req = *req;
    job.states.assign(req->states, req->states + req->nstates);
    job.submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        job.ticket = s->next_ticket++;
        *ticket = job.ticket;
        s->results[job.ticket] = Result{};
        s->queue.push_back(std::move(job));
    }
    s->cv_work.notify_one();
    return GWB200_OK;
}

int gwb200_server_wait(gwb200_server* s, int64_t ticket, int* status, double* queue_ms, double* service_ms,
                       double* device_ms) {
    if (!s) return gwb200_fail_status(GWB200_BAD_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->results.find(ticket);
    if (it == s->results.end()) return gwb200_fail_status(GWB200_BAD_ARGUMENT, "unknown ticket");
    s->cv_done.wait(lk, [&] { return s->results[ticket].done; });
    const Result r = s->results[ticket];
    s->results.erase(ticket);
    lk.unlock();
    if (status) *status = r.status;
    if (queue_ms) *queue_ms = r.queue_ms;
    if (service_ms) *service_ms = r.service_ms;
    if (device_ms) *device_ms = r.device_ms;
    if (r.status != GWB200_OK) return gwb200_fail_status(r.status, r.message.c_str());
    return GWB200_OK;
}

int gwb200_server_destroy(gwb200_server* s) {
    if (!s) return GWB200_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    for (auto& t : s->workers)
        if (t.joinable()) t.join();
    if (s->pool) {
        cudaSetDevice(s->device);
        cudaDeviceSynchronize();  // every worker's stream-ordered frees have completed
        cudaMemPoolDestroy(s->pool);
    }
    delete s;
    return GWB200_OK;
}

} // extern "C"
