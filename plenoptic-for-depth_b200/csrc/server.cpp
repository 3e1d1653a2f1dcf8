// server.cpp -- the request loop of include/pfd_serve.h.
//
// One dispatcher thread issues every device call; the slots' contexts each
// own a stream, so requests in different slots overlap on the GPU.  A request
// is admitted in arrival order when a slot is free and its frame fits the
// budget beside the admitted ones (the queue head waits; nothing overtakes
// it, so a large frame is not starved by small ones).  Its completion is
// signalled by a host function enqueued behind its last copy; the dispatcher
// then checks the context's device error flag, frees the frame (stream
// ordered) and hands the slot to the next request.  Results wait in pinned
// buffers, drawn from a pool so that no allocation or free of pinned memory
// (which would synchronise the device) happens while requests run.
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

#include <cuda_runtime.h>

#include "../../include/pfd_serve.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Pinned {
    void* p = nullptr;
    size_t bytes = 0;
};

struct Job {
    uint64_t ticket = 0;
    std::vector<uint8_t> raw;
    int W = 0, H = 0;
    std::vector<float> centers;
    std::vector<int> keys, nb_ids, nb_counts;
    int V = 0, mi_w = 0, mi_h = 0, max_nb = 0;
    pfd_pm_params params{};
    uint64_t seed = 0;
    int run_filter = 0;
    pfd_filter_cfg fcfg{};
    float unit = 0.0f;
    size_t bytes = 0;
    enum State { Queued, Running, GpuDone, Done, Failed } state = Queued;
    int slot = -1, fid = 0;
    Pinned out;                        // plane | cost | disp | sel
    pfd_status status = PFD_OK;
    std::string error;
    Clock::time_point t_submit, t_done;
    struct pfd_server* srv = nullptr;
};

}  // namespace

struct pfd_server {
    int device = 0;
    size_t budget = 0, admitted = 0;
    std::vector<pfd_ctx*> slots;
    std::vector<uint64_t> slot_job;    // ticket running in the slot, 0 = free
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<uint64_t> queue;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    std::mutex pinned_mu;              // the pinned pool has its own lock: never held across a CUDA call
    std::vector<Pinned> pinned_free;
    uint64_t next_ticket = 1;
    bool stopping = false;
    std::thread dispatcher;
    std::string last_error;
};

namespace {

size_t result_bytes(const Job& j)
{
    const size_t px = (size_t)j.V * j.mi_w * j.mi_h;
    return px * (16 + 4 + 16 + 4);
}

// Pinned buffers: best fit from the free list, else a new allocation (only
// while the pool grows).  Called without the server lock.
Pinned pinned_get(pfd_server* s, size_t bytes)
{
    std::unique_lock<std::mutex> lk(s->pinned_mu);
    size_t best = SIZE_MAX;
    int bi = -1;
    for (size_t i = 0; i < s->pinned_free.size(); ++i)
        if (s->pinned_free[i].bytes >= bytes && s->pinned_free[i].bytes < best) { best = s->pinned_free[i].bytes; bi = (int)i; }
    if (bi >= 0) {
        Pinned p = s->pinned_free[bi];
        s->pinned_free.erase(s->pinned_free.begin() + bi);
        return p;
    }
    lk.unlock();
    Pinned p;
    if (cudaHostAlloc(&p.p, bytes, cudaHostAllocPortable) == cudaSuccess) p.bytes = bytes;
    else { cudaGetLastError(); p.p = nullptr; }
    return p;
}

void CUDART_CB on_gpu_done(void* arg)
{
    Job* j = static_cast<Job*>(arg);
    pfd_server* s = j->srv;
    std::lock_guard<std::mutex> lk(s->mu);
    j->t_done = Clock::now();
    if (j->state == Job::Running) j->state = Job::GpuDone;
    s->cv_work.notify_all();
}

// Issues a request on its slot (dispatcher thread, lock not held).
pfd_status start_job(pfd_server* s, Job& j)
{
    pfd_ctx* ctx = s->slots[j.slot];
    pfd_status st = pfd_frame_upload(ctx, &j.fid, j.raw.data(), j.W, j.H, j.W, j.centers.data(), j.keys.data(), j.V,
                                     j.mi_w, j.mi_h, j.nb_ids.data(), j.nb_counts.data(), j.max_nb, nullptr);
    if (st != PFD_OK) { j.fid = 0; return st; }
    if ((st = pfd_patchmatch(ctx, j.fid, &j.params, j.seed)) != PFD_OK) return st;
    if (j.run_filter && (st = pfd_filter(ctx, j.fid, &j.fcfg, j.unit, nullptr, nullptr)) != PFD_OK) return st;
    const size_t px = (size_t)j.V * j.mi_w * j.mi_h;
    char* o = static_cast<char*>(j.out.p);
    if ((st = pfd_download_async(ctx, j.fid, (float*)o, (float*)(o + 16 * px), (float*)(o + 20 * px),
                                 (uint32_t*)(o + 36 * px))) != PFD_OK)
        return st;
    cudaStream_t stream = static_cast<cudaStream_t>(pfd_stream(ctx));
    if (cudaLaunchHostFunc(stream, on_gpu_done, &j) != cudaSuccess) {
        cudaGetLastError();
        return PFD_ECUDA;
    }
    return PFD_OK;
}

void fail_job(pfd_server* s, Job& j, pfd_status st, const std::string& why)
{
    j.status = st;
    j.error = why;
    j.state = Job::Failed;
    j.t_done = Clock::now();
    s->last_error = why;
}

void dispatch_loop(pfd_server* s)
{
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // finished requests: error flag, frame freed, slot and budget returned
        for (size_t k = 0; k < s->slots.size(); ++k) {
            const uint64_t t = s->slot_job[k];
            if (!t) continue;
            Job& j = *s->jobs[t];
            if (j.state != Job::GpuDone) continue;
            pfd_ctx* ctx = s->slots[k];
            lk.unlock();
            const pfd_status st = pfd_sync(ctx);
            std::string why = st == PFD_OK ? "" : pfd_last_error(ctx);
            pfd_frame_free(ctx, j.fid);
            lk.lock();
            if (st == PFD_OK) j.state = Job::Done;
            else fail_job(s, j, st, why);
            s->slot_job[k] = 0;
            s->admitted -= j.bytes;
            s->cv_done.notify_all();
        }
        if (s->stopping) {
            bool busy = false;
            for (uint64_t t : s->slot_job) busy = busy || t != 0;
            if (!busy) break;
        }
        // admissions, in arrival order
        while (!s->stopping && !s->queue.empty()) {
            Job& j = *s->jobs[s->queue.front()];
            int free_slot = -1;
            for (size_t k = 0; k < s->slots.size(); ++k)
                if (!s->slot_job[k]) { free_slot = (int)k; break; }
            if (free_slot < 0) break;
            if (s->budget && s->admitted + j.bytes > s->budget) break;
            s->queue.pop_front();
            j.slot = free_slot;
            j.state = Job::Running;
            s->slot_job[free_slot] = j.ticket;
            s->admitted += j.bytes;
            lk.unlock();
            j.out = pinned_get(s, result_bytes(j));
            const pfd_status st = j.out.p ? start_job(s, j) : PFD_ENOMEM;
            std::string why = st == PFD_OK ? "" : (j.out.p ? pfd_last_error(s->slots[free_slot]) : "pinned result buffer");
            lk.lock();
            if (st != PFD_OK) {
                // nothing of it remains queued on the stream once the slot's work drains
                pfd_ctx* ctx = s->slots[free_slot];
                lk.unlock();
                pfd_sync(ctx);
                if (j.fid) pfd_frame_free(ctx, j.fid);
                lk.lock();
                fail_job(s, j, st, why);
                s->slot_job[free_slot] = 0;
                s->admitted -= j.bytes;
                s->cv_done.notify_all();
            }
        }
        s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
    }
}

}  // namespace

extern "C" {

pfd_status pfd_server_create(pfd_server** out, int device, size_t hbm_budget_bytes, int slots)
{
    if (!out || slots < 1 || slots > 16) return PFD_EINVAL;
    *out = nullptr;
    pfd_server* s = new pfd_server;
    s->budget = hbm_budget_bytes;
    for (int k = 0; k < slots; ++k) {
        pfd_ctx* c = nullptr;
        const pfd_status st = pfd_create(&c, device, 0);
        if (st != PFD_OK) {
            for (pfd_ctx* x : s->slots) pfd_destroy(x);
            delete s;
            return st;
        }
        s->slots.push_back(c);
    }
    s->slot_job.assign(slots, 0);
    s->dispatcher = std::thread(dispatch_loop, s);
    *out = s;
    return PFD_OK;
}

void pfd_server_destroy(pfd_server* s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->queue.clear();
        s->cv_work.notify_all();
    }
    s->dispatcher.join();
    for (pfd_ctx* c : s->slots) pfd_destroy(c);
    for (auto& kv : s->jobs)
        if (kv.second->out.p) cudaFreeHost(kv.second->out.p);
    for (Pinned& p : s->pinned_free) cudaFreeHost(p.p);
    delete s;
}

pfd_status pfd_server_submit(pfd_server* s, const pfd_request* r, uint64_t* ticket)
{
    if (!s || !r || !ticket) return PFD_EINVAL;
    if (!r->raw || !r->centers || !r->tilekeys || !r->nb_ids || !r->nb_counts || r->W < 1 || r->H < 1 ||
        r->raw_pitch < r->W || r->n_views < 1 || r->max_nb < 1 || r->max_nb > 32 || r->mi_w < 2 || r->mi_h < 2)
        return PFD_EINVAL;
    auto j = std::make_unique<Job>();
    j->srv = s;
    j->W = r->W;
    j->H = r->H;
    j->raw.resize((size_t)r->W * r->H);
    for (int y = 0; y < r->H; ++y) std::memcpy(&j->raw[(size_t)y * r->W], r->raw + (size_t)y * r->raw_pitch, r->W);
    j->V = r->n_views;
    j->mi_w = r->mi_w;
    j->mi_h = r->mi_h;
    j->max_nb = r->max_nb;
    j->centers.assign(r->centers, r->centers + 2 * (size_t)r->n_views);
    j->keys.assign(r->tilekeys, r->tilekeys + 2 * (size_t)r->n_views);
    j->nb_ids.assign(r->nb_ids, r->nb_ids + (size_t)r->n_views * r->max_nb);
    j->nb_counts.assign(r->nb_counts, r->nb_counts + r->n_views);
    j->params = r->params;
    j->seed = r->seed;
    j->run_filter = r->run_filter;
    j->fcfg = r->filter_cfg;
    j->unit = r->baseline_unit;
    j->bytes = pfd_frame_bytes(r->W, r->H, r->n_views, r->mi_w, r->mi_h, r->max_nb, 0);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->budget && j->bytes > s->budget) {
        s->last_error = "request needs " + std::to_string(j->bytes) + " bytes, more than the budget";
        return PFD_ENOMEM;
    }
    j->ticket = s->next_ticket++;
    j->t_submit = Clock::now();
    *ticket = j->ticket;
    s->queue.push_back(j->ticket);
    s->jobs[j->ticket] = std::move(j);
    s->cv_work.notify_all();
    return PFD_OK;
}

pfd_status pfd_server_wait(pfd_server* s, uint64_t ticket, int timeout_ms, float* plane, float* cost, float* disp,
                           uint32_t* sel, double* latency_ms)
{
    if (!s) return PFD_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return PFD_ENOFRAME;
    Job& j = *it->second;
    auto finished = [&] { return j.state == Job::Done || j.state == Job::Failed; };
    if (timeout_ms < 0) s->cv_done.wait(lk, finished);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished)) return PFD_ETIMEDOUT;
    const pfd_status st = j.status;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(j.t_done - j.t_submit).count();
    std::unique_ptr<Job> done = std::move(it->second);
    s->jobs.erase(it);
    lk.unlock();
    if (st == PFD_OK) {
        const size_t px = (size_t)done->V * done->mi_w * done->mi_h;
        const char* o = static_cast<const char*>(done->out.p);
        if (plane) std::memcpy(plane, o, 16 * px);
        if (cost) std::memcpy(cost, o + 16 * px, 4 * px);
        if (disp) std::memcpy(disp, o + 20 * px, 16 * px);
        if (sel) std::memcpy(sel, o + 36 * px, 4 * px);
    }
    if (done->out.p) {
        std::lock_guard<std::mutex> pl(s->pinned_mu);
        s->pinned_free.push_back(done->out);
    }
    return st;
}

pfd_status pfd_server_load(pfd_server* s, int* queued, int* running, size_t* bytes_admitted)
{
    if (!s) return PFD_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    int run = 0;
    for (uint64_t t : s->slot_job) run += t != 0;
    if (queued) *queued = (int)s->queue.size();
    if (running) *running = run;
    if (bytes_admitted) *bytes_admitted = s->admitted;
    return PFD_OK;
}

const char* pfd_server_last_error(pfd_server* s)
{
    if (!s) return "";
    return s->last_error.c_str();
}

}  // extern "C"
