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
// Merging: when a worker frees up and several compatible requests wait (eta = 0, the same
// precision, small enough not to fill the GPU alone), it takes up
// to `max_merge` of them at once (and no more than a fair share of the queue per worker), loads
// each into a handle of its own (the worker's handle leads, the others come from the worker's
// member handles), and solves them with one gwb200_run_g0w0_batch: their frequency work is
// bucketed by size and factored in shared launches.  The batch is bit-identical to each request's
// own solve, so merging does not change results.  Requests are merged only while their resident
// data plus one frequency of the largest tall matrix fits the slot's budget; the lead's cap is
// lowered by the members' resident bytes for the batch call.  A batch that fails falls back to
// solving its requests one by one.
//
// No counterpart in the reference (it runs one molecule per process).
#include <algorithm>
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
    bool sliced = false;          // system given as slices (gwb200_server_submit_slices)
    gwb200_request_slices slices{};
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
    int max_merge = 8;               // requests one worker may take at once (1: no merging)
    int64_t merged_batches = 0;      // batches of two or more requests solved
    int64_t merged_requests = 0;     // requests solved inside those batches
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

// Device bytes a request keeps on its handle through a batch: V_ph, panel rows, exchange diagonal,
// scale vectors and forms of all its frequencies.
size_t resident_bytes(const gwb200_request& r) {
    const size_t nmo = (size_t)r.nmo, nocc = (size_t)r.nocc, n = nocc * (nmo - nocc);
    const size_t m = (size_t)r.nstates * nmo;
    const size_t n64 = (n + 63) / 64 * 64, m64 = (m + 63) / 64 * 64;
    const size_t pchol = r.precision == GWB200_MIXED_REFINED ? 2 * n * n64 : 0;  // the factor of V (refined form)
    return sizeof(double) * (n * n + m * n + nmo * nocc + (size_t)r.nfreq * (n64 + m64) + 4 * nmo * (size_t)r.nfreq +
                             pchol) +
           ((size_t)1 << 16);
}

// One frequency of the request's tall matrix in the form's element size.
size_t matrix_bytes(const gwb200_request& r) {
    const size_t nmo = (size_t)r.nmo, nocc = (size_t)r.nocc, n = nocc * (nmo - nocc);
    const size_t m = (size_t)r.nstates * nmo;
    const size_t n64 = (n + 63) / 64 * 64, m64 = (m + 63) / 64 * 64;
    return (n64 + m64) * n64 * (r.precision == GWB200_MIXED ? sizeof(float) : sizeof(double));
}

// Above this many particle-hole pairs one request's launches already fill the GPU (a 64-wide block
// step of n = 1536 has 24 x 24 tiles per frequency), so merging it only makes the small requests
// of its batch wait for it.
constexpr int64_t kMergeMaxNph = 1536;

bool mergeable(const gwb200_request& r) {
    const int64_t n = r.nocc * (r.nmo - r.nocc);
    return r.eta == 0.0 && n <= kMergeMaxNph &&
           (r.precision == GWB200_FP64 || r.precision == GWB200_MIXED || r.precision == GWB200_MIXED_REFINED);
}

int make_slot_handle(gwb200_server* s, gwb200_handle** out) {
    gwb200_handle* h = nullptr;
    int rc = gwb200_create(s->device, &h);
    if (rc == GWB200_OK) rc = gwb200_set_memory_limit(h, (int64_t)s->slot_budget);
    if (rc == GWB200_OK) {
        gwb200_attach_pool(h, s->pool);
        gwb200_share_sms(h, s->slots);
    } else {
        gwb200_destroy(h);
        h = nullptr;
    }
    *out = h;
    return rc;
}

int load_job(gwb200_handle* h, const Job& job) {
    const gwb200_request& r = job.req;
    if (job.sliced)
        return gwb200_load_system_slices(h, r.nmo, r.nocc, r.mo_energy, job.slices.vph, job.slices.panel,
                                         job.slices.xdiag, job.slices.vxc_diag, r.fermi_energy, job.states.data(),
                                         (int64_t)job.states.size());
    return gwb200_load_system_states(h, r.nmo, r.nocc, r.mo_energy, r.eri, r.vxc, r.fermi_energy, job.states.data(),
                                     (int64_t)job.states.size());
}

// One request on one handle (load, whole solve).
Result solve_alone(gwb200_handle* h, const Job& job, bool loaded) {
    const auto start = Clock::now();
    Result res;
    res.queue_ms = std::chrono::duration<double, std::milli>(start - job.submitted).count();
    const gwb200_request& r = job.req;
    int st = loaded ? GWB200_OK : load_job(h, job);
    gwb200_stats stats{};
    if (st == GWB200_OK)
        st = gwb200_run_g0w0(h, r.nfreq, r.npade, job.states.data(), (int64_t)job.states.size(), r.eta, r.precision,
                             r.omega_out, r.weight_out, r.sigma_out, r.sigma_x_out, r.qp_out, &stats);
    res.status = st;
    if (st != GWB200_OK) res.message = gwb200_last_error();
    res.service_ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
    res.device_ms = stats.device_ms_total;
    res.done = true;
    return res;
}

// Several compatible requests as one gwb200_run_g0w0_batch: jobs[0] on the lead handle h, the others
// on member handles.  Falls back to one solve per request if the batch call fails.
std::vector<Result> solve_merged(gwb200_server* s, gwb200_handle* h, std::vector<gwb200_handle*>& members,
                                 const std::vector<Job>& jobs) {
    const auto start = Clock::now();
    const size_t k = jobs.size();
    std::vector<Result> res(k);
    std::vector<gwb200_handle*> hs(k, nullptr);
    std::vector<int> load_st(k, GWB200_OK);
    std::vector<std::string> load_msg(k);
    hs[0] = h;
    for (size_t i = 1; i < k; ++i) {
        while (members.size() < i) {
            gwb200_handle* m = nullptr;
            if (make_slot_handle(s, &m) != GWB200_OK) break;
            members.push_back(m);
        }
        hs[i] = i <= members.size() ? members[i - 1] : nullptr;
    }
    // load every request (a request whose load fails leaves the batch with its status)
    std::vector<size_t> live;
    size_t members_resident = 0;
    for (size_t i = 0; i < k; ++i) {
        res[i].queue_ms = std::chrono::duration<double, std::milli>(start - jobs[i].submitted).count();
        if (!hs[i]) {
            load_st[i] = GWB200_CUDA_ERROR;
            load_msg[i] = "server: cannot create a member handle";
            continue;
        }
        load_st[i] = load_job(hs[i], jobs[i]);
        if (load_st[i] != GWB200_OK) {
            load_msg[i] = gwb200_last_error();
            continue;
        }
        live.push_back(i);
        if (i > 0) members_resident += resident_bytes(jobs[i].req);
    }
    int bst = GWB200_BAD_ARGUMENT;
    gwb200_stats stats{};
    if (live.size() >= 2) {
        std::vector<gwb200_handle*> bh;
        std::vector<int64_t> nf, np, ns;
        std::vector<const int64_t*> sp;
        std::vector<double*> so, qo;
        for (size_t i : live) {
            const gwb200_request& r = jobs[i].req;
            bh.push_back(hs[i]);
            nf.push_back(r.nfreq);
            np.push_back(r.npade);
            sp.push_back(jobs[i].states.data());
            ns.push_back((int64_t)jobs[i].states.size());
            so.push_back(r.sigma_out);
            qo.push_back(r.qp_out);
        }
        // the batch's workspaces live on the lead: its cap less what the members keep resident
        const int64_t lead_cap = (int64_t)s->slot_budget - (int64_t)members_resident;
        int64_t nbuckets = 0;
        if (lead_cap > 0 && gwb200_set_memory_limit(h, lead_cap) == GWB200_OK) {
            bst = gwb200_run_g0w0_batch(bh.data(), (int64_t)bh.size(), nf.data(), np.data(), sp.data(), ns.data(),
                                        jobs[live[0]].req.precision, so.data(), qo.data(), &nbuckets, &stats);
            gwb200_set_memory_limit(h, (int64_t)s->slot_budget);
        }
    }
    if (bst == GWB200_OK) {
        for (size_t i : live) {  // grid and exchange diagonal of each request (not part of the batch outputs)
            const gwb200_request& r = jobs[i].req;
            int st = GWB200_OK;
            if (r.omega_out || r.weight_out) {
                std::vector<double> om((size_t)r.nfreq), w((size_t)r.nfreq);
                st = gwb200_grid(r.nfreq, om.data(), w.data());
                if (r.omega_out) std::memcpy(r.omega_out, om.data(), sizeof(double) * om.size());
                if (r.weight_out) std::memcpy(r.weight_out, w.data(), sizeof(double) * w.size());
            }
            if (st == GWB200_OK && r.sigma_x_out) st = gwb200_sigma_x_diag(hs[i], r.sigma_x_out);
            res[i].status = st;
            if (st != GWB200_OK) res[i].message = gwb200_last_error();
            res[i].device_ms = stats.device_ms_total;
        }
        std::lock_guard<std::mutex> lk(s->mu);
        s->merged_batches += 1;
        s->merged_requests += (int64_t)live.size();
    } else {
        for (size_t i : live) {  // one by one, on the loaded handles
            const double q = res[i].queue_ms;
            res[i] = solve_alone(hs[i], jobs[i], /*loaded=*/true);
            res[i].queue_ms = q;
        }
    }
    const double service = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
    for (size_t i = 0; i < k; ++i) {
        if (load_st[i] != GWB200_OK) {
            res[i].status = load_st[i];
            res[i].message = load_msg[i];
        }
        if (bst == GWB200_OK || load_st[i] != GWB200_OK) res[i].service_ms = service;
        res[i].done = true;
    }
    return res;
}

void worker_main(gwb200_server* s) {
    gwb200_handle* h = nullptr;
    int rc = make_slot_handle(s, &h);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (rc != GWB200_OK && s->start_error.empty()) s->start_error = gwb200_last_error();
        s->workers_ready.fetch_add(1);
    }
    s->cv_done.notify_all();
    if (rc != GWB200_OK) return;
    std::vector<gwb200_handle*> members;
    for (;;) {
        std::vector<Job> jobs;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stopping || !s->queue.empty(); });
            if (s->queue.empty()) break;  // stopping with nothing left
            jobs.push_back(std::move(s->queue.front()));
            s->queue.pop_front();
            // continuous batching: compatible requests already waiting join this one
            if (s->max_merge > 1 && mergeable(jobs[0].req)) {
                // a fair share of what waits, so that the other workers get requests too
                const int share = (int)((s->queue.size() + 1 + (size_t)s->slots - 1) / (size_t)s->slots);
                const int take = std::min(s->max_merge, std::max(2, share));
                size_t need = resident_bytes(jobs[0].req), big = matrix_bytes(jobs[0].req);
                for (auto it = s->queue.begin(); it != s->queue.end() && (int)jobs.size() < take;) {
                    const gwb200_request& r = it->req;
                    const size_t need2 = need + resident_bytes(r), big2 = std::max(big, matrix_bytes(r));
                    if (mergeable(r) && r.precision == jobs[0].req.precision &&
                        (double)(need2 + big2) <= 0.8 * (double)s->slot_budget) {
                        need = need2;
                        big = big2;
                        jobs.push_back(std::move(*it));
                        it = s->queue.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
        }
        std::vector<Result> res;
        if (jobs.size() == 1) res.push_back(solve_alone(h, jobs[0], /*loaded=*/false));
        else res = solve_merged(s, h, members, jobs);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (size_t i = 0; i < jobs.size(); ++i) s->results[jobs[i].ticket] = std::move(res[i]);
        }
        s->cv_done.notify_all();
    }
    for (gwb200_handle* m : members) gwb200_destroy(m);
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

namespace {
int submit_job(gwb200_server* s, const gwb200_request* req, const gwb200_request_slices* slices, int64_t* ticket) {
    if (!s || !req || !ticket) return gwb200_fail_status(GWB200_BAD_ARGUMENT, "null server, request or ticket");
    if (req->nmo <= 0 || req->nocc <= 0 || req->nocc >= req->nmo || req->nfreq <= 0 || req->npade <= 0 ||
        req->nstates <= 0 || !req->states)
        return gwb200_fail_status(GWB200_BAD_SHAPE, "request: bad nmo/nocc/nfreq/npade/states");
    if (min_footprint(*req) > s->slot_budget)
        return gwb200_fail_status(GWB200_OOM, "request does not fit one slot's device-memory budget");
    Job job;
    job.req = *req;
    job.states.assign(req->states, req->states + req->nstates);
    if (slices) {
        job.sliced = true;
        job.slices = *slices;
    }
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
} // namespace

int gwb200_server_submit(gwb200_server* s, const gwb200_request* req, int64_t* ticket) {
    return submit_job(s, req, nullptr, ticket);
}

int gwb200_server_submit_slices(gwb200_server* s, const gwb200_request* req, const gwb200_request_slices* slices,
                                int64_t* ticket) {
    if (!slices || !slices->vph || !slices->panel || !slices->xdiag || !slices->vxc_diag)
        return gwb200_fail_status(GWB200_BAD_ARGUMENT, "null slice array");
    return submit_job(s, req, slices, ticket);
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

int gwb200_server_set_merge(gwb200_server* s, int max_requests) {
    if (!s || max_requests < 1) return gwb200_fail_status(GWB200_BAD_ARGUMENT, "null server or max_requests < 1");
    std::lock_guard<std::mutex> lk(s->mu);
    s->max_merge = std::min(max_requests, 4096);
    return GWB200_OK;
}

int gwb200_server_counters(gwb200_server* s, int64_t* merged_batches, int64_t* merged_requests) {
    if (!s) return gwb200_fail_status(GWB200_BAD_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (merged_batches) *merged_batches = s->merged_batches;
    if (merged_requests) *merged_requests = s->merged_requests;
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
