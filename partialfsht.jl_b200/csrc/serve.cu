// Serving loop (pfsht_server_*): plans kept resident on one device, synthesis and adjoint
// requests on host buffers admitted as they arrive and run concurrently.
//
// A server owns `nslots` streams. Plans are registered against an HBM budget: a plan counts
// its own device memory and the staging buffers that requests on host arrays go through, and a
// registration that would exceed the budget is refused. Requests queue in arrival order; a
// worker thread admits a request as soon as a stream is free and its plan is idle, together with
// the requests for the same plan queued behind it (up to kMaxGroup): the group's applies run on
// one stream one after the other, since they share the plan's buffers, while their copies run on
// the plan's own copy streams, so one request's copies in and out overlap its neighbours' kernels
// (requests for different plans overlap as well: one's copies with another's kernels). Each
// admitted request is enqueued as copy in -> apply -> copy out, and a host callback on the plan's
// copy-out stream marks it done; the group's last one frees its stream and plan and wakes the
// worker, so requests that arrive while others are on the GPU start as soon as resources free up.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "plan_internal.hpp"

namespace {

struct Request;

}  // namespace

struct pfsht_server {
    int device = 0;
    int64_t budget = 0, used = 0;
    std::vector<pfsht_plan*> plans;
    std::vector<int64_t> plan_bytes;
    std::vector<char> plan_busy;
    std::vector<int> plan_left;  // requests of the plan's admitted group still running
    std::vector<cudaStream_t> slots;
    std::vector<char> slot_busy;
    std::deque<Request*> pending;
    std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    int running = 0;
    int64_t next_id = 1, completed = 0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

using namespace pf;

enum { kPending = 0, kRunning = 1, kDone = 2, kFailed = 3 };
constexpr int kMaxGroup = 8;  // same-plan requests admitted together

struct Request {
    pfsht_server* srv = nullptr;
    int64_t id = 0;
    int plan = 0, fwd = 1, slot = -1;
    const void* in = nullptr;
    void* out = nullptr;
    double t_submit = 0, t_start = 0, t_done = 0;
    int state = kPending;
    int status = 0;
    std::string err;
};

int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

// host callback at the end of a request's work: no CUDA calls here
void CUDART_CB request_done(void* arg) {
    Request* r = static_cast<Request*>(arg);
    pfsht_server* s = r->srv;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->t_done = s->now();
        r->state = kDone;
        s->running -= 1;
        s->completed += 1;
        if (--s->plan_left[r->plan] == 0) {
            s->plan_busy[r->plan] = 0;
            s->slot_busy[r->slot] = 0;
        }
    }
    s->cv_work.notify_one();
    s->cv_done.notify_all();
}

// one request of an admitted group: the apply on the group's stream, the copies on the plan's
// copy streams, and the completion after the request's copy out (on the plan's copy-out stream)
int launch(pfsht_server* s, Request* r) {
    pfsht_plan* p = s->plans[r->plan];
    cudaStream_t st = s->slots[r->slot];
    PF_TRY(plan_host_enqueue(p, r->in, r->out, r->fwd != 0, st, false));
    PF_CUDA(cudaLaunchHostFunc(p->d2h, request_done, r));
    return 0;
}

void worker_main(pfsht_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // admit in arrival order, skipping requests whose plan is busy; an admitted request
        // takes the requests queued behind it for the same plan along
        for (auto it = s->pending.begin(); it != s->pending.end();) {
            const auto fs = std::find(s->slot_busy.begin(), s->slot_busy.end(), 0);
            if (fs == s->slot_busy.end()) break;
            Request* r = *it;
            if (s->plan_busy[r->plan]) {
                ++it;
                continue;
            }
            const int slot = (int)(fs - s->slot_busy.begin());
            std::vector<Request*> group;
            for (auto jt = it; jt != s->pending.end() && (int)group.size() < kMaxGroup;) {
                if ((*jt)->plan == r->plan) {
                    group.push_back(*jt);
                    jt = s->pending.erase(jt);
                } else {
                    ++jt;
                }
            }
            s->slot_busy[slot] = 1;
            s->plan_busy[r->plan] = 1;
            s->plan_left[r->plan] = (int)group.size();
            s->running += (int)group.size();
            const double t = s->now();
            for (Request* g : group) {
                g->slot = slot;
                g->state = kRunning;
                g->t_start = t;
            }
            lk.unlock();
            size_t k = 0;
            int rc = 0;
            for (; k < group.size() && !rc; ++k) rc = launch(s, group[k]);
            std::string msg = rc ? get_error() : std::string();
            lk.lock();
            if (rc) {
                // the failed request and those after it run no callback: release them here
                for (size_t q = k - 1; q < group.size(); ++q) {
                    Request* g = group[q];
                    g->status = rc;
                    g->err = msg;
                    g->state = kFailed;
                    g->t_done = s->now();
                    s->running -= 1;
                    if (--s->plan_left[g->plan] == 0) {
                        s->plan_busy[g->plan] = 0;
                        s->slot_busy[g->slot] = 0;
                    }
                }
                s->cv_done.notify_all();
            }
            it = s->pending.begin();  // the lock was released: start over
        }
        if (s->stop && s->pending.empty() && s->running == 0) break;
        s->cv_work.wait(lk);
    }
}

int server_create(int device, int64_t budget, int nslots, pfsht_server** out) {
    if (!out) return fail(PFSHT_ERR_ARGUMENT, "out is NULL");
    if (budget <= 0) return fail(PFSHT_ERR_ARGUMENT, "the HBM budget must be positive");
    if (nslots < 1 || nslots > 64) return fail(PFSHT_ERR_ARGUMENT, "nslots must lie in 1..64");
    int dev = device;
    if (dev < 0) PF_CUDA(cudaGetDevice(&dev));
    DeviceGuard dg(dev);
    std::unique_ptr<pfsht_server> s(new pfsht_server());
    s->device = dev;
    s->budget = budget;
    s->slots.resize(nslots);
    s->slot_busy.assign(nslots, 0);
    for (int k = 0; k < nslots; ++k) PF_CUDA(cudaStreamCreateWithFlags(&s->slots[k], cudaStreamNonBlocking));
    s->worker = std::thread(worker_main, s.get());
    *out = s.release();
    return 0;
}

int server_add(pfsht_server* s, pfsht_plan* p, int32_t* id) {
    if (!s || !p || !id) return fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    if (p->device != s->device) return fail(PFSHT_ERR_ARGUMENT, "the plan lives on another device");
    DeviceGuard dg(s->device);
    std::lock_guard<std::mutex> lk(s->mu);
    for (pfsht_plan* q : s->plans)
        if (q == p) return fail(PFSHT_ERR_ARGUMENT, "the plan is registered already");
    // one coefficient array and one field per direction of the host copies
    const int64_t staging = 2 * (int64_t)sizeof(double2) *
                            ((int64_t)(p->L + 1) * (2 * p->L + 1) + p->M) * p->B;
    const int64_t bytes = p->info.device_bytes + (p->st_alm.p ? 0 : staging);
    if (s->used + bytes > s->budget)
        return fail(PFSHT_ERR_OUT_OF_MEMORY,
                    "registering this plan needs " + std::to_string(bytes) + " bytes of device memory; " +
                    std::to_string(s->budget - s->used) + " of the server's budget are left");
    PF_TRY(plan_host_staging(p));
    s->plans.push_back(p);
    s->plan_bytes.push_back(bytes);
    s->plan_busy.push_back(0);
    s->plan_left.push_back(0);
    s->used += bytes;
    *id = (int32_t)(s->plans.size() - 1);
    return 0;
}

}  // namespace

extern "C" {

pfsht_status pfsht_server_create(int32_t device, int64_t hbm_budget_bytes, int32_t nslots,
                                 pfsht_server** out) {
    if (out) *out = nullptr;
    return (pfsht_status)server_create(device, hbm_budget_bytes, nslots, out);
}

pfsht_status pfsht_server_add_plan(pfsht_server* s, pfsht_plan* plan, int32_t* plan_id) {
    return (pfsht_status)server_add(s, plan, plan_id);
}

pfsht_status pfsht_server_submit(pfsht_server* s, int32_t plan_id, int32_t forward,
                                 const void* in, void* out, int64_t* request_id) {
    if (!s || !in || !out || !request_id)
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL argument");
    std::unique_lock<std::mutex> lk(s->mu);
    if (plan_id < 0 || plan_id >= (int32_t)s->plans.size())
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "unknown plan id");
    if (s->stop) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "the server is shutting down");
    std::unique_ptr<Request> r(new Request());
    r->srv = s;
    r->id = s->next_id++;
    r->plan = plan_id;
    r->fwd = forward ? 1 : 0;
    r->in = in;
    r->out = out;
    r->t_submit = s->now();
    *request_id = r->id;
    s->pending.push_back(r.get());
    s->reqs.emplace(r->id, std::move(r));
    lk.unlock();
    s->cv_work.notify_one();
    return PFSHT_OK;
}

pfsht_status pfsht_server_wait(pfsht_server* s, int64_t request_id, double timeout_s,
                               double* latency_s) {
    if (!s) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "unknown request id");
    Request* r = it->second.get();
    const auto pred = [&] { return r->state == kDone || r->state == kFailed; };
    if (timeout_s < 0) s->cv_done.wait(lk, pred);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
        return (pfsht_status)fail(PFSHT_ERR_TIMEOUT, "the request is not done yet");
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    if (r->state == kFailed) return (pfsht_status)fail(r->status, r->err);
    return PFSHT_OK;
}

pfsht_status pfsht_server_request_times(pfsht_server* s, int64_t request_id, double* t_submit,
                                        double* t_start, double* t_done) {
    if (!s) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "unknown request id");
    const Request* r = it->second.get();
    if (t_submit) *t_submit = r->t_submit;
    if (t_start) *t_start = r->t_start;
    if (t_done) *t_done = r->t_done;
    return PFSHT_OK;
}

pfsht_status pfsht_server_release(pfsht_server* s, int64_t request_id) {
    if (!s) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "unknown request id");
    if (it->second->state != kDone && it->second->state != kFailed)
        return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "the request has not finished");
    s->reqs.erase(it);
    return PFSHT_OK;
}

pfsht_status pfsht_server_stats(pfsht_server* s, int64_t* completed, int64_t* queued,
                                int64_t* running, int64_t* bytes_resident) {
    if (!s) return (pfsht_status)fail(PFSHT_ERR_ARGUMENT, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (completed) *completed = s->completed;
    if (queued) *queued = (int64_t)s->pending.size();
    if (running) *running = s->running;
    if (bytes_resident) *bytes_resident = s->used;
    return PFSHT_OK;
}

pfsht_status pfsht_server_destroy(pfsht_server* s) {
    if (!s) return PFSHT_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_one();
    if (s->worker.joinable()) s->worker.join();
    DeviceGuard dg(s->device);
    for (cudaStream_t st : s->slots) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    delete s;
    return PFSHT_OK;
}

}  // extern "C"
