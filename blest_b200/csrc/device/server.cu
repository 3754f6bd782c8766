// Query server with continuous batching (no counterpart in the reference,
// whose driver runs one BFS per call, Benchmark.cuh:247-269).
//
// Requests (BFS from a source, or CC) on resident graphs are queued; a
// scheduler thread forms jobs whenever an executor lane is free:
//  - pending BFS requests on the same graph are coalesced, up to
//    max_batch, into one multi-source BFS (a lone request uses the
//    single-source kernel, which has lower latency); under the adaptive
//    policy a batch runs only when the graph's measured lane time of a
//    multi-source job of its width is below that of its requests one by
//    one, else the front request runs alone and the rest stay pending for
//    the next free lanes;
//  - pending CC requests on the same graph share one CC run;
//  - a job is admitted only if its device scratch fits the memory budget
//    (the batch is shrunk, or the job waits for running jobs to finish;
//    a single request that can never fit is refused with
//    BLEST_ERR_ADMISSION).
// Each lane has its own CUDA stream and per-graph workspaces whose
// cooperative grids are capped to a share of the SMs, so jobs on different
// lanes run side by side on the device. Results land in the caller's
// buffer, host memory or (for a consumer on the GPU) device memory: a
// batch writes the device-bound results straight into their buffers (one
// output row per source) and stages only the host-bound ones. Each request
// records submit / start / done times; an optional completion queue hands
// finished tickets to the client in completion order.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <string>
#include <vector>

#include "../host/errors.hpp"
#include "blest.h"
#include "runtime.hpp"

namespace blest {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    uint32_t graph = 0;
    int kind = BLEST_QUERY_BFS;
    uint32_t source = 0;
    uint32_t* out = nullptr;
    int out_mem = BLEST_MEM_HOST;  // where `out` lives
    int status = BLEST_OK;
    uint32_t batch = 0;
    double submit = 0, start = 0, done_t = 0;
    bool done = false;
    std::string error;
};

struct GraphEntry {
    blest_graph* g = nullptr;  // null for virtual (dry-run) graphs
    uint32_t n = 0;
    // running estimates (lane seconds) of a single-source BFS job and of a
    // multi-source job per width class (32 / 64 / 128 sources), for the
    // adaptive batch policy; 0 = not measured yet
    double single_s = 0, mbfs_s[3] = {0, 0, 0};
    uint64_t nnz = 0;
    uint64_t ws_bytes = 0;     // one workspace
};

struct Job {
    uint32_t graph = 0;
    int kind = BLEST_QUERY_BFS;
    std::vector<Request*> reqs;
    uint64_t bytes = 0;
};

struct Lane {
    int idx = 0;
    cudaStream_t stream = nullptr;
    std::vector<blest_workspace*> ws;  // per graph, created on first use
    std::unique_ptr<Job> job;
    bool busy = false;
    std::thread th;
    std::condition_variable cv;
};

}  // namespace
}  // namespace blest

struct blest_server {
    blest_server_params p{};
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<blest::Request*> pending;
    std::unordered_map<uint64_t, std::unique_ptr<blest::Request>> requests;
    std::vector<blest::GraphEntry> graphs;
    std::vector<std::unique_ptr<blest::Lane>> lanes;
    uint64_t budget = 0, reserved = 0, peak = 0, resident = 0;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread scheduler;
    blest::Clock::time_point t0;
    int device = 0;
    uint32_t lane_grid = 0;
    std::deque<uint64_t> done_q;  // finished tickets (completion_queue servers)
    // stats
    uint64_t submitted = 0, completed = 0, rejected = 0, jobs = 0, batched = 0, unbatched = 0;
    uint64_t kind_jobs[3] = {0, 0, 0}, kind_requests[3] = {0, 0, 0};  // single BFS, multi-source BFS, CC
    double busy_s = 0, kind_busy[3] = {0, 0, 0};
    std::vector<double> latencies;
};

namespace blest {
namespace {

double now(const blest_server* s) { return std::chrono::duration<double>(Clock::now() - s->t0).count(); }

// Job kinds for the per-kind statistics.
int job_kind(const Job& job) {
    return job.kind == BLEST_QUERY_CC ? 2 : (job.reqs.size() > 1 ? 1 : 0);
}

// Width class of a multi-source batch of k sources (group width 32/64/128).
int width_class(size_t k) { return k <= 32 ? 0 : (k <= 64 ? 1 : 2); }

void update_estimate(double& est, double t) { est = est > 0 ? 0.75 * est + 0.25 * t : t; }

// Device bytes a job needs beyond already-resident workspaces: the MBFS
// state and a staging row per host-bound result (device-bound results are
// written straight into their buffers).
uint64_t job_bytes(const GraphEntry& ge, int kind, const std::vector<Request*>& reqs, uint32_t k) {
    if (kind == BLEST_QUERY_CC || k <= 1) return 0;
    const uint64_t words = k <= 32 ? 1 : (k <= 64 ? 2 : 4);
    uint64_t host = 0;
    for (uint32_t i = 0; i < k && i < reqs.size(); ++i) host += reqs[i]->out_mem == BLEST_MEM_HOST;
    return 4ull * mbfs_state_words(ge.n, (uint32_t)words) + 4ull * host * ge.n;
}

void finish(blest_server* s, Job& job, int status, const std::string& err, double start) {
    std::lock_guard<std::mutex> lk(s->mu);
    const double t = now(s);  // under the lock: done times follow the completion queue's order
    for (Request* r : job.reqs) {
        r->status = status;
        r->error = err;
        r->start = start;
        r->done_t = t;
        r->batch = (uint32_t)job.reqs.size();
        r->done = true;
        ++s->completed;
        s->latencies.push_back(t - r->submit);
        if (s->p.completion_queue) s->done_q.push_back(r->id);
    }
    const int kk = job_kind(job);
    if (status == BLEST_OK && kk < 2) {
        GraphEntry& ge = s->graphs[job.graph];
        update_estimate(kk == 0 ? ge.single_s : ge.mbfs_s[width_class(job.reqs.size())], t - start);
    }
    ++s->kind_jobs[kk];
    s->kind_requests[kk] += job.reqs.size();
    s->kind_busy[kk] += t - start;
    s->reserved -= job.bytes;
    s->busy_s += t - start;
}

int run_job(blest_server* s, Lane& lane, Job& job) {
    // copies taken under the lock: blest_server_add_graph may grow the graph
    // and workspace tables while this job runs
    GraphEntry ge;
    blest_workspace* ws = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        ge = s->graphs[job.graph];
        ws = lane.ws[job.graph];
    }
    if (s->p.dry_run) {
        for (Request* r : job.reqs)
            if (r->out) r->out[0] = (uint32_t)job.reqs.size();  // marks the batch in dry runs
        // stands in for the device time of a job, so that requests arriving
        // meanwhile queue up behind it as they would behind a real run: 1 ms
        // for a single request or a CC run, 20 ms for a multi-source batch
        const bool batch = job.kind == BLEST_QUERY_BFS && job.reqs.size() > 1;
        std::this_thread::sleep_for(std::chrono::microseconds(batch ? 20000 : 1000));
        return BLEST_OK;
    }
    cudaSetDevice(s->device);
    if (!ws) {
        const int rc = blest_workspace_create(ge.g, &ws);
        if (rc != BLEST_OK) return rc;
        blest_workspace_set_grid(ws, s->lane_grid);
        std::lock_guard<std::mutex> lk(s->mu);
        lane.ws[job.graph] = ws;
    }
    if (job.kind == BLEST_QUERY_CC) {
        const Request& r0 = *job.reqs[0];
        int rc = blest_cc_ws(ws, r0.out, r0.out_mem, lane.stream, nullptr);
        if (rc != BLEST_OK) return rc;
        for (size_t i = 1; i < job.reqs.size() && rc == BLEST_OK; ++i)
            if (cudaMemcpyAsync(job.reqs[i]->out, r0.out, 4ull * ge.n, cudaMemcpyDefault, lane.stream) != cudaSuccess)
                rc = BLEST_ERR_CUDA;
        if (cudaStreamSynchronize(lane.stream) != cudaSuccess && rc == BLEST_OK) rc = BLEST_ERR_CUDA;
        return rc;
    }
    if (job.reqs.size() == 1)
        return blest_bfs_ws(ws, job.reqs[0]->source, job.reqs[0]->out, nullptr, job.reqs[0]->out_mem, nullptr,
                            lane.stream, 0, nullptr);
    // one output row per source: a device-bound result's own buffer, or a
    // staging row for a host-bound one (copied out after the run)
    const uint32_t k = (uint32_t)job.reqs.size();
    std::vector<uint32_t> src(k);
    std::vector<uint32_t*> rows(k);
    uint32_t host = 0;
    for (uint32_t i = 0; i < k; ++i) {
        src[i] = job.reqs[i]->source;
        host += job.reqs[i]->out_mem == BLEST_MEM_HOST;
    }
    blest_mbfs_params mp{};
    mp.group_width = k <= 32 ? 32 : (k <= 64 ? 64 : 128);
    uint32_t* staging = nullptr;
    if (host && cudaMallocAsync((void**)&staging, 4ull * host * ge.n, lane.stream) != cudaSuccess) {
        cudaGetLastError();
        return BLEST_ERR_OOM;
    }
    for (uint32_t i = 0, h = 0; i < k; ++i)
        rows[i] = job.reqs[i]->out_mem == BLEST_MEM_HOST ? staging + (size_t)(h++) * ge.n : job.reqs[i]->out;
    int rc = blest_mbfs_rows_ws(ws, src.data(), k, rows.data(), &mp, lane.stream, nullptr);
    for (uint32_t i = 0; i < k && rc == BLEST_OK; ++i)
        if (job.reqs[i]->out_mem == BLEST_MEM_HOST &&
            cudaMemcpyAsync(job.reqs[i]->out, rows[i], 4ull * ge.n, cudaMemcpyDeviceToHost, lane.stream) !=
                cudaSuccess)
            rc = BLEST_ERR_CUDA;
    if (staging) cudaFreeAsync(staging, lane.stream);
    if (cudaStreamSynchronize(lane.stream) != cudaSuccess && rc == BLEST_OK) rc = BLEST_ERR_CUDA;
    return rc;
}

void lane_main(blest_server* s, Lane* lane) {
    for (;;) {
        std::unique_ptr<Job> job;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            lane->cv.wait(lk, [&] { return s->stop || lane->job; });
            if (!lane->job) return;
            job = std::move(lane->job);
        }
        const double start = now(s);
        const int rc = run_job(s, *lane, *job);
        finish(s, *job, rc, rc == BLEST_OK ? std::string() : std::string(blest_last_error()), start);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            lane->busy = false;
        }
        s->cv_sched.notify_all();
        s->cv_done.notify_all();
    }
}

// Pick the next job for a free lane (called with the lock held). Returns
// false when the front request must wait for memory.
bool form_job(blest_server* s, Job& job) {
    Request* front = s->pending.front();
    const GraphEntry& ge = s->graphs[front->graph];
    job.graph = front->graph;
    job.kind = front->kind;
    std::vector<Request*> take;
    for (Request* r : s->pending) {
        if (r->graph != front->graph || r->kind != front->kind) continue;
        if (r->kind == BLEST_QUERY_BFS && take.size() >= s->p.max_batch) break;
        take.push_back(r);
    }
    // shrink the batch until it fits the memory that is free now
    uint32_t k = (uint32_t)take.size();
    if (job.kind == BLEST_QUERY_BFS) {
        while (k > 1 && s->reserved + job_bytes(ge, job.kind, take, k) > s->budget) k = k > 32 ? (k + 1) / 2 : k - 1;
    }
    // adaptive policy: run the front request alone when the batch would cost
    // more lane time than its requests one by one (after the shrink, so the
    // estimate is for the batch that would run)
    if (job.kind == BLEST_QUERY_BFS && k > 1 && s->p.batch_policy == BLEST_BATCH_ADAPTIVE) {
        const double m = ge.mbfs_s[width_class(k)];
        if (ge.single_s > 0 && m > 0 && k * ge.single_s < m) {
            k = 1;
            ++s->unbatched;
        }
    }
    const uint64_t need = job_bytes(ge, job.kind, take, job.kind == BLEST_QUERY_BFS ? k : 1);
    if (s->reserved + need > s->budget) return false;
    take.resize(job.kind == BLEST_QUERY_BFS ? k : take.size());
    job.reqs = take;
    job.bytes = need;
    for (Request* r : take) s->pending.erase(std::find(s->pending.begin(), s->pending.end(), r));
    return true;
}

void scheduler_main(blest_server* s) {
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        Lane* freeLane = nullptr;
        s->cv_sched.wait(lk, [&] {
            if (s->stop) return true;
            if (s->pending.empty()) return false;
            for (auto& l : s->lanes)
                if (!l->busy) return true;
            return false;
        });
        if (s->stop) return;
        for (auto& l : s->lanes)
            if (!l->busy) {
                freeLane = l.get();
                break;
            }
        auto job = std::make_unique<Job>();
        if (!form_job(s, *job)) {
            // waits for running jobs to release memory; if nothing runs, the
            // front request can never fit: refuse it
            bool anyBusy = false;
            for (auto& l : s->lanes) anyBusy |= l->busy;
            if (!anyBusy) {
                Request* r = s->pending.front();
                s->pending.pop_front();
                r->status = BLEST_ERR_ADMISSION;
                r->done = true;
                r->done_t = now(s);
                ++s->rejected;
                if (s->p.completion_queue) s->done_q.push_back(r->id);
                s->cv_done.notify_all();
                continue;
            }
            s->cv_sched.wait(lk);
            continue;
        }
        s->reserved += job->bytes;
        s->peak = std::max(s->peak, s->reserved);
        ++s->jobs;
        if (job->reqs.size() > 1) s->batched += job->reqs.size();
        freeLane->busy = true;
        freeLane->job = std::move(job);
        freeLane->cv.notify_one();
    }
}

}  // namespace
}  // namespace blest

using blest::guarded;

extern "C" {

int blest_server_create(const blest_server_params* p, blest_server** out) {
    blest_server* s = nullptr;
    const int rc = guarded([&] {
        blest::require(out, "null argument");
        blest::require(!p || p->batch_policy == BLEST_BATCH_ADAPTIVE || p->batch_policy == BLEST_BATCH_ALWAYS,
                       "bad batch_policy");
        s = new blest_server;
        if (p) s->p = *p;
        if (!s->p.lanes) s->p.lanes = 4;
        if (!s->p.max_batch || s->p.max_batch > 128) s->p.max_batch = 128;
        if (!s->p.queue_capacity) s->p.queue_capacity = 1u << 20;
        s->t0 = blest::Clock::now();
        if (!s->p.dry_run) {
            BLEST_CUDA(cudaGetDevice(&s->device));
            size_t freeB = 0, totalB = 0;
            BLEST_CUDA(cudaMemGetInfo(&freeB, &totalB));
            s->budget = s->p.memory_budget ? s->p.memory_budget : freeB / 2;
            const int sms = blest::device_sm_count(s->device);
            s->lane_grid = std::max<uint32_t>(1, (uint32_t)(2 * sms) / s->p.lanes);
        } else {
            s->budget = s->p.memory_budget ? s->p.memory_budget : (1ull << 40);
        }
        for (uint32_t i = 0; i < s->p.lanes; ++i) {
            auto lane = std::make_unique<blest::Lane>();
            lane->idx = (int)i;
            if (!s->p.dry_run) BLEST_CUDA(cudaStreamCreateWithFlags(&lane->stream, cudaStreamNonBlocking));
            s->lanes.push_back(std::move(lane));
        }
        for (auto& l : s->lanes) l->th = std::thread(blest::lane_main, s, l.get());
        s->scheduler = std::thread(blest::scheduler_main, s);
        *out = s;
    });
    if (rc != BLEST_OK && s) blest_server_destroy(s);
    return rc;
}

static int add_graph(blest_server* s, blest_graph* g, uint32_t n, uint64_t nnz, uint32_t* id) {
    return guarded([&] {
        blest::require(s && id, "null argument");
        std::lock_guard<std::mutex> lk(s->mu);
        blest::GraphEntry ge;
        ge.g = g;
        ge.n = n;
        ge.nnz = nnz;
        s->graphs.push_back(ge);
        for (auto& l : s->lanes) {
            blest_workspace* ws = nullptr;
            if (g) {
                // one workspace per lane, created now so no request pays for
                // device allocation; its cooperative grids get the lane's share
                const int rc = blest_workspace_create(g, &ws);
                if (rc != BLEST_OK) throw blest::Error(rc, blest_last_error());
                blest_workspace_set_grid(ws, s->lane_grid);
                blest::mbfs_reserve(ws->w, n, 4);
            }
            l->ws.push_back(ws);
        }
        *id = (uint32_t)(s->graphs.size() - 1);
    });
}

int blest_server_add_graph(blest_server* s, blest_graph* g, uint32_t* graph_id) {
    if (!s || !g || s->p.dry_run) {
        blest::set_last_error(!s || !g ? "null argument" : "dry-run server takes virtual graphs only");
        return BLEST_ERR_INVALID_ARG;
    }
    return add_graph(s, g, g->d.n, g->d.nnz, graph_id);
}

int blest_server_add_virtual_graph(blest_server* s, uint32_t n, uint64_t nnz, uint32_t* graph_id) {
    if (!s || !s->p.dry_run) {
        blest::set_last_error("virtual graphs need a dry-run server");
        return BLEST_ERR_INVALID_ARG;
    }
    return add_graph(s, nullptr, n, nnz, graph_id);
}

int blest_server_submit(blest_server* s, uint32_t graph_id, int kind, uint32_t source, uint32_t* out_host,
                        uint64_t* ticket) {
    return blest_server_submit_ex(s, graph_id, kind, source, out_host, BLEST_MEM_HOST, ticket);
}

int blest_server_submit_ex(blest_server* s, uint32_t graph_id, int kind, uint32_t source, uint32_t* out, int out_mem,
                           uint64_t* ticket) {
    return guarded([&] {
        blest::require(s && ticket && out, "null argument");
        blest::require(kind == BLEST_QUERY_BFS || kind == BLEST_QUERY_CC, "bad query kind");
        blest::require(out_mem == BLEST_MEM_HOST || out_mem == BLEST_MEM_DEVICE, "bad out_mem");
        blest::require(!(s->p.dry_run && out_mem == BLEST_MEM_DEVICE), "dry-run servers take host buffers only");
        if (out_mem == BLEST_MEM_DEVICE) {
            // refused here rather than failing the whole batch it would join
            cudaPointerAttributes at{};
            BLEST_CUDA(cudaPointerGetAttributes(&at, out));
            if (!((at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) && at.device == s->device))
                throw blest::Error(BLEST_ERR_INVALID_ARG, "out is not device memory of the server's device");
        }
        std::lock_guard<std::mutex> lk(s->mu);
        blest::require(graph_id < s->graphs.size(), "unknown graph id");
        if (kind == BLEST_QUERY_BFS && source >= s->graphs[graph_id].n)
            throw blest::Error(BLEST_ERR_INVALID_ARG, "source vertex out of range");
        if (s->pending.size() >= s->p.queue_capacity) throw blest::Error(BLEST_ERR_BUSY, "request queue is full");
        auto r = std::make_unique<blest::Request>();
        r->id = s->next_id++;
        r->graph = graph_id;
        r->kind = kind;
        r->source = source;
        r->out = out;
        r->out_mem = out_mem;
        r->submit = blest::now(s);
        s->pending.push_back(r.get());
        *ticket = r->id;
        s->requests[r->id] = std::move(r);
        ++s->submitted;
        s->cv_sched.notify_one();
    });
}

static void fill_result(const blest::Request& r, blest_query_result* out) {
    if (!out) return;
    out->status = r.status;
    out->kind = r.kind;
    out->graph_id = r.graph;
    out->source = r.source;
    out->batch_size = r.batch;
    out->submit_s = r.submit;
    out->start_s = r.start;
    out->done_s = r.done_t;
}

int blest_server_poll(blest_server* s, uint64_t ticket, int* done, blest_query_result* result) {
    return guarded([&] {
        blest::require(s && done, "null argument");
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->requests.find(ticket);
        blest::require(it != s->requests.end(), "unknown ticket");
        *done = it->second->done ? 1 : 0;
        if (*done) fill_result(*it->second, result);
    });
}

int blest_server_wait(blest_server* s, uint64_t ticket, double timeout_s, blest_query_result* result) {
    return guarded([&] {
        blest::require(s, "null argument");
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->requests.find(ticket);
        blest::require(it != s->requests.end(), "unknown ticket");
        blest::Request* r = it->second.get();
        const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->done; });
        if (!ok) throw blest::Error(BLEST_ERR_BUSY, "timed out waiting for the request");
        fill_result(*r, result);
        if (r->status != BLEST_OK)
            throw blest::Error(r->status, "request failed: " + (r->error.empty() ? std::string("refused") : r->error));
    });
}

int blest_server_drain(blest_server* s, double timeout_s) {
    return guarded([&] {
        blest::require(s, "null argument");
        std::unique_lock<std::mutex> lk(s->mu);
        const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
            return s->completed + s->rejected == s->submitted;
        });
        if (!ok) throw blest::Error(BLEST_ERR_BUSY, "timed out draining the server");
    });
}

int blest_server_next_done(blest_server* s, double timeout_s, uint64_t* ticket, blest_query_result* result) {
    return guarded([&] {
        blest::require(s && ticket, "null argument");
        blest::require(s->p.completion_queue, "server was created without a completion queue");
        *ticket = 0;
        std::unique_lock<std::mutex> lk(s->mu);
        const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                            [&] { return !s->done_q.empty(); });
        if (!ok) throw blest::Error(BLEST_ERR_BUSY, "no request finished within the timeout");
        *ticket = s->done_q.front();
        s->done_q.pop_front();
        auto it = s->requests.find(*ticket);
        if (it != s->requests.end())
            fill_result(*it->second, result);
        else if (result)  // released before it was taken from the queue
            std::memset(result, 0, sizeof(*result));
    });
}

int blest_server_release(blest_server* s, uint64_t ticket) {
    return guarded([&] {
        blest::require(s, "null argument");
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->requests.find(ticket);
        blest::require(it != s->requests.end(), "unknown ticket");
        blest::require(it->second->done, "request has not finished");
        s->requests.erase(it);
    });
}

int blest_server_stats_get(blest_server* s, blest_server_stats* out) {
    return guarded([&] {
        blest::require(s && out, "null argument");
        std::lock_guard<std::mutex> lk(s->mu);
        std::memset(out, 0, sizeof(*out));
        out->submitted = s->submitted;
        out->completed = s->completed;
        out->rejected = s->rejected;
        out->jobs = s->jobs;
        out->batched_requests = s->batched;
        out->busy_s = s->busy_s;
        out->peak_reserved_bytes = s->peak;
        out->memory_budget = s->budget;
        out->jobs_bfs = s->kind_jobs[0];
        out->jobs_mbfs = s->kind_jobs[1];
        out->jobs_cc = s->kind_jobs[2];
        out->requests_mbfs = s->kind_requests[1];
        out->requests_cc = s->kind_requests[2];
        out->busy_bfs_s = s->kind_busy[0];
        out->busy_mbfs_s = s->kind_busy[1];
        out->busy_cc_s = s->kind_busy[2];
        out->unbatched_requests = s->unbatched;
        std::vector<double> l = s->latencies;
        if (!l.empty()) {
            std::sort(l.begin(), l.end());
            auto pct = [&](double q) { return l[std::min(l.size() - 1, (size_t)(q * (l.size() - 1) + 0.5))]; };
            out->p50_latency_s = pct(0.50);
            out->p99_latency_s = pct(0.99);
            double sum = 0;
            for (double x : l) sum += x;
            out->mean_latency_s = sum / l.size();
        }
    });
}

int blest_server_destroy(blest_server* s) {
    if (!s) return BLEST_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_sched.notify_all();
    for (auto& l : s->lanes) l->cv.notify_all();
    if (s->scheduler.joinable()) s->scheduler.join();
    for (auto& l : s->lanes) {
        if (l->th.joinable()) l->th.join();
        for (blest_workspace* ws : l->ws)
            if (ws) blest_workspace_destroy(ws);
        if (l->stream) cudaStreamDestroy(l->stream);
    }
    delete s;
    return BLEST_OK;
}

}  // extern "C"
