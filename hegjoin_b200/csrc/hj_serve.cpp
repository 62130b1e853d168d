// hj_serve.cpp -- continuous-batching self-join service.
//
// Beyond the reference (which joins one dataset per process): requests of
// uneven (n, d, eps) arrive at any time; a request is admitted as soon as a
// worker slot is free and its device-memory reservation fits the HBM budget,
// and each worker runs its request's whole pipeline (copy-in, index, workload
// order, join) on its own CUDA stream, so the kernels of concurrent requests
// overlap on the device (the persistent refine kernels take only as many SMs
// as the request has work items).  Results stay resident in HBM until the
// client collects them; their bytes count against the budget until then.
//
// Timestamps (seconds on the steady clock) are kept per request: submit,
// admit, finish; latency = finish - submit.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "hegjoin_b200.h"
#include "hj_workspace.h"

namespace hj {
void result_set_stream(hj_result* r, cudaStream_t s);   // hj_join.cu
}

namespace {
constexpr size_t kWorkspaceBytes = 256ull << 20;   // per worker
}

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Req {
    uint64_t ticket = 0;
    const void* h_db = nullptr;
    uint32_t n = 0, d = 0, k = 0;
    int dtype = HJ_F32;
    double eps = 0;
    uint64_t fixed = 0;         // bytes held while running: dataset, index, operand forms
    uint64_t allowance = 0;     // bytes held while running: the join's result buffers and results
    uint64_t result_bytes = 0;  // bytes held after completion, until collected
    int state = 0;              // 0 queued, 1 running, 2 done
    hj_status status = HJ_OK;
    char err[256] = {0};
    hj_result* result = nullptr;
    hj_join_stats stats{};
    uint32_t regrants = 0;      // times the join asked for a larger allowance
    double t_submit = 0, t_admit = 0, t_done = 0;
};

}  // namespace

struct hj_server {
    hj_server_opts opts{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req*> queue;
    std::map<uint64_t, Req*> reqs;
    uint64_t next_ticket = 1;
    uint64_t in_use = 0;        // bytes reserved by running requests and held by uncollected results
    uint64_t peak_in_use = 0;
    uint32_t running = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    int device = 0;
};

namespace {

// Device bytes a request holds while it runs, apart from its join's result
// buffers and results: the dataset copy, the index (points in cell order,
// perm, cell tables and hash, workload order, work items, the sort's
// temporaries beyond the worker's workspace) and the tensor-core operand forms.
uint64_t fixed_bytes(const Req& r) {
    const uint64_t s = r.dtype == HJ_F64 ? 8 : 4;
    const uint64_t kpad = ((r.d + 4 + 31) / 32) * 32;
    uint64_t b = 2ull * r.n * r.d * s;          // dataset + points in cell order
    b += 128ull * r.n;                          // perm, cell tables and hash, workload, sort temporaries
    if (r.dtype == HJ_F32 && r.d >= 16) b += 4ull * r.n * kpad + 16ull * r.n;   // TC operands
    return b + (16ull << 20);
}
// The first allowance for the join's result buffers and kept results: ~64
// neighbours per point.  The join is capped at its allowance
// (hj_join_opts.device_bytes_cap); a join that needs more is refused before it
// allocates, and the request waits for the larger allowance it asked for.
uint64_t first_allowance(const Req& r) { return 64ull * r.n * 28ull + (16ull << 20); }

void worker_main(hj_server* S) {
    cudaSetDevice(S->device);
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    // the worker's device workspace: the temporaries of its requests' index builds and
    // joins come from it, so a small request makes no allocator calls for them
    hj::Workspace ws;
    ws.stream = st;
    if (cudaMallocAsync((void**)&ws.base, kWorkspaceBytes, st) == cudaSuccess) {
        ws.cap = kWorkspaceBytes;
        hj::set_current_workspace(&ws);
    } else {
        cudaGetLastError();   // no workspace: every temporary comes from the pool
        std::lock_guard<std::mutex> lk(S->mu);
        S->in_use -= kWorkspaceBytes;
    }
    for (;;) {
        Req* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] {
                if (S->stop) return true;
                if (S->queue.empty()) return false;
                const Req* f = S->queue.front();
                // FIFO admission: the head runs when it fits, or alone when nothing else does
                return S->running == 0 || S->in_use + f->fixed + f->allowance <= S->opts.hbm_budget;
            });
            if (S->stop && S->queue.empty()) break;
            if (S->queue.empty()) continue;
            r = S->queue.front();
            S->queue.pop_front();
            S->in_use += r->fixed + r->allowance;
            S->peak_in_use = std::max(S->peak_in_use, S->in_use);
            S->running++;
            r->state = 1;
            r->t_admit = now_s();
        }
        hj_status s = HJ_OK;
        void* d_db = nullptr;
        const size_t bytes = (size_t)r->n * r->d * (r->dtype == HJ_F64 ? 8 : 4);
        hj_index* ix = nullptr;
        if (cudaMallocAsync(&d_db, bytes, st) != cudaSuccess ||
            cudaMemcpyAsync(d_db, r->h_db, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            s = HJ_ERR_CUDA;
            snprintf(r->err, sizeof(r->err), "copy-in failed");
        }
        if (s == HJ_OK) s = hj_index_create(d_db, r->n, r->d, r->k, r->dtype, r->eps, nullptr, nullptr, st, &ix);
        if (d_db) cudaFreeAsync(d_db, st);
        if (s == HJ_OK) s = hj_sort_by_workload(ix, st, nullptr);
        if (s == HJ_OK) {
            hj_join_opts o;
            hj_join_opts_default(&o);
            o.refine = S->opts.refine;
            o.mem_fraction = 0.6 / std::max<uint32_t>(1, S->opts.workers);
            o.device_bytes_cap = r->allowance;
            s = hj_join(ix, &o, st, &r->result, &r->stats);
            // refused by its cap: give the allowance back, wait until the larger one it
            // asked for fits (or nothing else runs), and join again on the same index
            for (int tries = 0; s == HJ_ERR_OOM && r->stats.bytes_wanted > r->allowance && tries < 3; ++tries) {
                const uint64_t want = r->stats.bytes_wanted + r->stats.bytes_wanted / 16;
                {
                    std::unique_lock<std::mutex> lk(S->mu);
                    S->in_use -= r->allowance;
                    S->running--;
                    S->cv_work.notify_all();
                    S->cv_work.wait(lk, [&] { return S->running == 0 || S->in_use + want <= S->opts.hbm_budget; });
                    S->in_use += want;
                    S->peak_in_use = std::max(S->peak_in_use, S->in_use);
                    S->running++;
                    r->allowance = want;
                    r->regrants++;
                }
                r->err[0] = 0;
                o.device_bytes_cap = r->allowance;
                s = hj_join(ix, &o, st, &r->result, &r->stats);
            }
        }
        if (s != HJ_OK && !r->err[0]) snprintf(r->err, sizeof(r->err), "%s", hj_last_error());
        if (ix) hj_index_destroy(ix);
        cudaStreamSynchronize(st);
        // the worker's stream dies with the server; the finished result's later
        // frees go to the legacy default stream (all its work is complete)
        if (r->result) hj::result_set_stream(r->result, nullptr);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            r->status = s;
            r->result_bytes = r->result ? r->stats.total_pairs * 4ull + 16ull * r->n : 0;
            S->in_use = S->in_use - r->fixed - r->allowance + r->result_bytes;
            S->peak_in_use = std::max(S->peak_in_use, S->in_use);
            S->running--;
            r->state = 2;
            r->t_done = now_s();
        }
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
    hj::set_current_workspace(nullptr);
    if (ws.base) cudaFreeAsync(ws.base, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
}

}  // namespace

extern "C" {

void hj_server_opts_default(hj_server_opts* o) {
    if (!o) return;
    *o = hj_server_opts{};
    o->hbm_budget = 150ull << 30;
    o->workers = 4;
    o->refine = HJ_REFINE_AUTO;
}

hj_status hj_server_create(const hj_server_opts* opts, hj_server** out) {
    if (!out) return HJ_ERR_INVALID;
    hj_server* S = new hj_server();
    if (opts) S->opts = *opts; else hj_server_opts_default(&S->opts);
    if (S->opts.workers == 0) S->opts.workers = 1;
    if (S->opts.hbm_budget == 0) S->opts.hbm_budget = 150ull << 30;
    cudaGetDevice(&S->device);
    S->in_use = (uint64_t)S->opts.workers * kWorkspaceBytes;   // the workers' workspaces
    S->peak_in_use = S->in_use;
    for (uint32_t i = 0; i < S->opts.workers; ++i) S->workers.emplace_back(worker_main, S);
    *out = S;
    return HJ_OK;
}

hj_status hj_server_submit(hj_server* S, const void* h_db, uint32_t n, uint32_t d, uint32_t k, int dtype, double eps,
                           uint64_t* ticket) {
    if (!S || !h_db || !ticket || n == 0 || d == 0 || k == 0 || k > d || (dtype != HJ_F32 && dtype != HJ_F64))
        return HJ_ERR_INVALID;
    Req* r = new Req();
    r->h_db = h_db; r->n = n; r->d = d; r->k = k; r->dtype = dtype; r->eps = eps;
    r->fixed = fixed_bytes(*r);
    r->allowance = first_allowance(*r);
    r->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(S->mu);
        r->ticket = S->next_ticket++;
        S->reqs[r->ticket] = r;
        S->queue.push_back(r);
    }
    S->cv_work.notify_all();
    *ticket = r->ticket;
    return HJ_OK;
}

hj_status hj_server_wait(hj_server* S, uint64_t ticket, double timeout_s, hj_result** result, hj_serve_info* info) {
    if (!S) return HJ_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return HJ_ERR_INVALID;
    Req* r = it->second;
    bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9),
                                  [&] { return r->state == 2; });
    if (!ok) return HJ_ERR_TIMEOUT;
    if (info) {
        info->status = r->status;
        info->t_submit = r->t_submit;
        info->t_admit = r->t_admit;
        info->t_done = r->t_done;
        info->stats = r->stats;
        info->reserved_bytes = r->fixed + r->allowance;
        info->regrants = r->regrants;
    }
    hj_status st = r->status;
    if (result) {
        *result = r->result;       // ownership passes to the caller
    } else if (r->result) {
        hj_result_destroy(r->result);
    }
    S->in_use -= r->result_bytes;
    S->reqs.erase(it);
    delete r;
    lk.unlock();
    S->cv_work.notify_all();
    return st;
}

hj_status hj_server_usage(hj_server* S, uint64_t* in_use, uint64_t* peak_in_use) {
    if (!S) return HJ_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    if (in_use) *in_use = S->in_use;
    if (peak_in_use) *peak_in_use = S->peak_in_use;
    return HJ_OK;
}

hj_status hj_server_destroy(hj_server* S) {
    if (!S) return HJ_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    for (auto& t : S->workers) t.join();
    for (auto& kv : S->reqs) {
        if (kv.second->result) hj_result_destroy(kv.second->result);
        delete kv.second;
    }
    delete S;
    return HJ_OK;
}

}  // extern "C"
