// jfg_server.cu -- device-resident request loop over model families.
//
// Serving pattern of the reference's optimisation worker
// (tools/jfem_worker_jsonl.jl:132-148, manifest_batch_core.jl:283-409): many
// property-update requests against a few models.  Here each family's mesh,
// CSC pattern and scatter maps stay on the GPU in its jfg_model handle; a
// request carries a new shell-thickness vector and asks for K and KG of that
// family (membrane stress recovery from the family's displacement field is
// part of KG).  Results stay on the device until the client releases them.
//
// Policies:
//   JFG_SERVE_BATCHED  continuous batching.  A scheduler thread takes every
//                      request of a family that is waiting when a result
//                      slot of that family frees up (up to the family's batch
//                      limit) and runs them as one batched launch
//                      (jfg_assemble_batch_device) on the family's stream;
//                      families run on separate streams, so their work
//                      overlaps on the device, and a family keeps up to two
//                      batches queued so its stream never idles.  Requests
//                      that arrive while others run join the next batch.
//   JFG_SERVE_SERIAL   the plain path: one request per launch, in arrival
//                      order, each waited for before the next starts.
// Admission: at creation every family gets batch workspace and result slots
// sized to an equal share of the HBM budget; a request waits in its family's
// queue until a slot is free.  Completion times come from a host function
// enqueued behind each batch on its stream.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/jfem_gpu.h"

namespace {

constexpr int kSlotsPerFamily = 2;

struct SrvRequest {
    int64_t ticket = 0;
    int family = 0;
    std::vector<double> h;      // thickness vector, copied at submit
    bool keep = true;           // results kept until jfg_server_release
    bool freed = false;         // keep == false: its slot share was returned at completion
    int state = 0;              // 0 queued, 1 launched, 2 done
    int slot = -1, var = -1;
    double t_submit = 0, t_launch = 0, t_done = 0;
};

struct Batch;

struct Slot {
    double *h_dev = nullptr, *nzk = nullptr, *nzkg = nullptr, *max = nullptr;
    double *h_pin = nullptr;    // pinned staging of the batch's thickness vectors
    bool busy = false;
    int unreleased = 0;
    Batch *batch = nullptr;
};

struct Family {
    jfg_model *m = nullptr;
    cudaStream_t stream = nullptr;
    int64_t ndof = 0, nnz = 0, n_shell = 0;
    double *u_dev = nullptr;    // the family's displacement field for KG (or null: K only)
    int B = 1;                  // batch limit
    std::vector<Slot> slots;
    std::deque<int64_t> pending;
    int inflight = 0;
};

}  // namespace

struct jfg_server;

namespace {
struct Batch {
    jfg_server *s = nullptr;
    int family = 0, slot = 0;
    std::vector<int64_t> tickets;
};
}  // namespace

struct jfg_server {
    std::vector<Family> fam;
    int policy = JFG_SERVE_BATCHED;
    std::mutex mu;
    std::condition_variable cv;        // wakes the scheduler
    std::condition_variable done_cv;   // wakes waiting clients
    std::thread th;
    bool stop = false;
    bool hold = false;                 // queue requests without launching (jfg_server_hold)
    std::unordered_map<int64_t, SrvRequest> reqs;
    std::deque<int64_t> fifo;          // arrival order (serial policy)
    int64_t next_ticket = 1;
    int64_t n_done = 0, n_batches = 0, max_batch_seen = 0, reserved_bytes = 0;
    std::chrono::steady_clock::time_point t0;
    std::string err;
    std::vector<void *> allocs, pinned;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

jfg_status sfail(jfg_server *s, jfg_status st, const std::string &msg) {
    if (s) s->err = msg;
    return st;
}

#define SCK(call)                                                                                             \
    do {                                                                                                      \
        cudaError_t _e = (call);                                                                              \
        if (_e != cudaSuccess)                                                                                \
            return sfail(s, _e == cudaErrorMemoryAllocation ? JFG_ERR_NOMEM : JFG_ERR_CUDA,                    \
                         std::string(#call) + ": " + cudaGetErrorString(_e));                                  \
    } while (0)

// Runs on a CUDA host thread once the batch's kernels have finished.  No
// CUDA calls here: it only stamps the completion time and wakes waiters.
void CUDART_CB batch_done(void *p) {
    Batch *b = static_cast<Batch *>(p);
    jfg_server *s = b->s;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const double t = s->now();
        Family &f = s->fam[b->family];
        Slot &sl = f.slots[b->slot];
        for (int64_t tk : b->tickets) {
            auto it = s->reqs.find(tk);
            if (it == s->reqs.end()) continue;
            it->second.state = 2;
            it->second.t_done = t;
            if (!it->second.keep) {  // results dropped now; the record (times) stays until released
                it->second.freed = true;
                sl.unreleased -= 1;
            }
        }
        s->n_done += (int64_t)b->tickets.size();
        f.inflight -= 1;
        sl.batch = nullptr;
        if (sl.unreleased == 0) sl.busy = false;
    }
    s->cv.notify_all();
    s->done_cv.notify_all();
    delete b;
}

// Launch one batch (the lock is held by the caller while the batch is formed,
// released for the CUDA calls).
jfg_status launch_batch(jfg_server *s, Batch *b) {
    Family &f = s->fam[b->family];
    Slot &sl = f.slots[b->slot];
    const int n = (int)b->tickets.size();
    SCK(cudaMemcpyAsync(sl.h_dev, sl.h_pin, sizeof(double) * f.n_shell * n, cudaMemcpyHostToDevice, f.stream));
    jfg_status st = jfg_assemble_batch_device(f.m, n, sl.h_dev, nullptr, f.u_dev, 0, sl.nzk, sl.max, nullptr,
                                              f.u_dev ? sl.nzkg : nullptr);
    if (st) return sfail(s, st, std::string("batched assembly: ") + jfg_last_error(f.m));
    SCK(cudaLaunchHostFunc(f.stream, batch_done, b));
    return JFG_OK;
}

// Form a batch of up to f.B queued requests of family fi in a free slot.
// Called with the lock held; returns null when nothing can start.
Batch *form_batch(jfg_server *s, int fi, int limit) {
    Family &f = s->fam[fi];
    if (f.pending.empty()) return nullptr;
    int si = -1;
    for (int k = 0; k < (int)f.slots.size(); ++k)
        if (!f.slots[k].busy) { si = k; break; }
    if (si < 0) return nullptr;
    Slot &sl = f.slots[si];
    Batch *b = new Batch;
    b->s = s;
    b->family = fi;
    b->slot = si;
    const double t = s->now();
    while (!f.pending.empty() && (int)b->tickets.size() < limit) {
        int64_t tk = f.pending.front();
        f.pending.pop_front();
        SrvRequest &r = s->reqs[tk];
        const int v = (int)b->tickets.size();
        std::memcpy(sl.h_pin + v * f.n_shell, r.h.data(), sizeof(double) * f.n_shell);
        std::vector<double>().swap(r.h);  // the pinned copy is the one the launch reads
        r.state = 1;
        r.slot = si;
        r.var = v;
        r.t_launch = t;
        b->tickets.push_back(tk);
    }
    sl.busy = true;
    sl.unreleased = (int)b->tickets.size();
    sl.batch = b;
    f.inflight += 1;
    s->n_batches += 1;
    s->max_batch_seen = std::max<int64_t>(s->max_batch_seen, (int64_t)b->tickets.size());
    return b;
}

void scheduler(jfg_server *s) {
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        if (s->hold) {
            s->cv.wait_for(lk, std::chrono::milliseconds(50));
            continue;
        }
        std::vector<Batch *> ready;
        if (s->policy == JFG_SERVE_SERIAL) {
            // one request per launch, in arrival order, each completed before the next
            if (!s->fifo.empty()) {
                int64_t tk = s->fifo.front();
                auto it = s->reqs.find(tk);
                if (it == s->reqs.end()) { s->fifo.pop_front(); continue; }
                Family &f = s->fam[it->second.family];
                if (f.inflight == 0 && !f.pending.empty() && f.pending.front() == tk) {
                    Batch *b = form_batch(s, it->second.family, 1);
                    if (b) {
                        s->fifo.pop_front();
                        lk.unlock();
                        jfg_status st = launch_batch(s, b);
                        if (st == JFG_OK) cudaStreamSynchronize(f.stream);
                        lk.lock();
                        if (st) s->stop = true;
                        continue;
                    }
                }
            }
        } else {
            for (int fi = 0; fi < (int)s->fam.size(); ++fi) {
                Family &f = s->fam[fi];
                while (f.inflight < 2) {
                    Batch *b = form_batch(s, fi, f.B);
                    if (!b) break;
                    ready.push_back(b);
                }
            }
            if (!ready.empty()) {
                lk.unlock();
                bool bad = false;
                for (Batch *b : ready)
                    if (launch_batch(s, b)) bad = true;
                lk.lock();
                if (bad) s->stop = true;
                continue;
            }
        }
        s->cv.wait_for(lk, std::chrono::milliseconds(50));
    }
}

}  // namespace

extern "C" {

jfg_status jfg_server_create(jfg_model *const *families, const double *const *u_host, int32_t n_families,
                             int64_t hbm_budget_bytes, int32_t max_batch, int32_t policy, jfg_server **out) {
    if (!families || n_families < 1 || !out || max_batch < 1 || hbm_budget_bytes <= 0 ||
        (policy != JFG_SERVE_BATCHED && policy != JFG_SERVE_SERIAL))
        return JFG_ERR_INVALID;
    *out = nullptr;
    jfg_server *s = new jfg_server;
    s->policy = policy;
    s->t0 = std::chrono::steady_clock::now();
    s->fam.resize(n_families);
    const int64_t share = hbm_budget_bytes / n_families;
    auto fail_free = [&](jfg_status st) {
        jfg_server_destroy(s);
        return st;
    };
    for (int i = 0; i < n_families; ++i) {
        Family &f = s->fam[i];
        f.m = families[i];
        if (!f.m) return fail_free(JFG_ERR_INVALID);
        int64_t counts[4];
        if (jfg_model_counts(f.m, counts) || jfg_pattern(f.m, &f.ndof, &f.nnz)) return fail_free(JFG_ERR_STATE);
        f.n_shell = counts[1] + counts[2];
        int64_t ws1 = 0;
        if (jfg_batch_workspace_bytes(f.m, 1, &ws1)) return fail_free(JFG_ERR_STATE);
        const bool kg = u_host && u_host[i];
        // per variant: workspace + its share of every result slot (K, KG, max, h)
        const int64_t out1 = 8 * (f.nnz * (kg ? 2 : 1) + 1 + f.n_shell);
        const int64_t per = ws1 + kSlotsPerFamily * out1;
        int64_t B = std::min<int64_t>(max_batch, share / std::max<int64_t>(per, 1));
        if (B < 1) {
            jfg_server_destroy(s);
            return JFG_ERR_NOMEM;
        }
        f.B = (int)std::min<int64_t>(B, 65535);
        if (jfg_batch_reserve(f.m, f.B)) return fail_free(JFG_ERR_NOMEM);
        if (cudaStreamCreateWithFlags(&f.stream, cudaStreamNonBlocking) != cudaSuccess) return fail_free(JFG_ERR_CUDA);
        if (jfg_set_stream(f.m, f.stream)) return fail_free(JFG_ERR_STATE);
        if (kg) {
            if (cudaMalloc((void **)&f.u_dev, sizeof(double) * f.ndof) != cudaSuccess) return fail_free(JFG_ERR_NOMEM);
            s->allocs.push_back(f.u_dev);
            if (cudaMemcpy(f.u_dev, u_host[i], sizeof(double) * f.ndof, cudaMemcpyHostToDevice) != cudaSuccess)
                return fail_free(JFG_ERR_CUDA);
        }
        f.slots.resize(kSlotsPerFamily);
        for (Slot &sl : f.slots) {
            double *blk = nullptr;
            const int64_t nd = (int64_t)f.B * (f.nnz * (kg ? 2 : 1) + 1 + f.n_shell);
            if (cudaMalloc((void **)&blk, sizeof(double) * std::max<int64_t>(nd, 1)) != cudaSuccess)
                return fail_free(JFG_ERR_NOMEM);
            s->allocs.push_back(blk);
            sl.nzk = blk;
            sl.nzkg = kg ? blk + f.B * f.nnz : nullptr;
            sl.max = blk + f.B * f.nnz * (kg ? 2 : 1);
            sl.h_dev = sl.max + f.B;
            if (cudaMallocHost((void **)&sl.h_pin, sizeof(double) * std::max<int64_t>(f.B * f.n_shell, 1)) != cudaSuccess)
                return fail_free(JFG_ERR_NOMEM);
            s->pinned.push_back(sl.h_pin);
        }
        s->reserved_bytes += (int64_t)f.B * per;
    }
    s->th = std::thread(scheduler, s);
    *out = s;
    return JFG_OK;
}

jfg_status jfg_server_submit(jfg_server *s, int32_t family, const double *h_host, int32_t keep, int64_t *ticket) {
    if (!s) return JFG_ERR_INVALID;
    if (family < 0 || family >= (int)s->fam.size() || !h_host || !ticket)
        return sfail(s, JFG_ERR_INVALID, "bad family, thickness pointer or ticket pointer");
    const Family &f = s->fam[family];
    for (int64_t e = 0; e < f.n_shell; ++e)
        if (!(h_host[e] > 0.0)) return sfail(s, JFG_ERR_INVALID, "shell thickness must be positive");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return sfail(s, JFG_ERR_STATE, "server stopped: " + s->err);
        const int64_t tk = s->next_ticket++;
        SrvRequest &r = s->reqs[tk];
        r.ticket = tk;
        r.family = family;
        r.h.assign(h_host, h_host + f.n_shell);
        r.keep = keep != 0;
        r.t_submit = s->now();
        s->fam[family].pending.push_back(tk);
        if (s->policy == JFG_SERVE_SERIAL) s->fifo.push_back(tk);
        *ticket = tk;
    }
    s->cv.notify_all();
    return JFG_OK;
}

jfg_status jfg_server_wait(jfg_server *s, int64_t ticket, double timeout_s, int32_t *done) {
    if (!s || !done) return JFG_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] {
        auto it = s->reqs.find(ticket);
        return s->stop || it == s->reqs.end() || it->second.state == 2;
    };
    if (timeout_s < 0) s->done_cv.wait(lk, ready);
    else s->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
    auto it = s->reqs.find(ticket);
    *done = (it == s->reqs.end() || it->second.state == 2) ? 1 : 0;
    if (s->stop && !*done) return sfail(s, JFG_ERR_STATE, "server stopped: " + s->err);
    return JFG_OK;
}

jfg_status jfg_server_result(jfg_server *s, int64_t ticket, double **nzk_dev, double **nzkg_dev, double **max_dev,
                             double *times3) {
    if (!s) return JFG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return sfail(s, JFG_ERR_INVALID, "unknown or released ticket");
    const SrvRequest &r = it->second;
    if (r.state != 2) return sfail(s, JFG_ERR_STATE, "request not finished");
    const Family &f = s->fam[r.family];
    const Slot &sl = f.slots[r.slot];
    if (nzk_dev) *nzk_dev = r.freed ? nullptr : sl.nzk + (int64_t)r.var * f.nnz;
    if (nzkg_dev) *nzkg_dev = (r.freed || !sl.nzkg) ? nullptr : sl.nzkg + (int64_t)r.var * f.nnz;
    if (max_dev) *max_dev = r.freed ? nullptr : sl.max + r.var;
    if (times3) { times3[0] = r.t_submit; times3[1] = r.t_launch; times3[2] = r.t_done; }
    return JFG_OK;
}

jfg_status jfg_server_release(jfg_server *s, int64_t ticket) {
    if (!s) return JFG_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return sfail(s, JFG_ERR_INVALID, "unknown or released ticket");
        if (it->second.state != 2) return sfail(s, JFG_ERR_STATE, "request not finished");
        Slot &sl = s->fam[it->second.family].slots[it->second.slot];
        const bool freed = it->second.freed;
        s->reqs.erase(it);
        if (!freed) {
            sl.unreleased -= 1;
            if (sl.unreleased == 0 && !sl.batch) sl.busy = false;
        }
    }
    s->cv.notify_all();
    return JFG_OK;
}

jfg_status jfg_server_stats(jfg_server *s, int64_t *out6) {
    if (!s || !out6) return JFG_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    out6[0] = s->next_ticket - 1;       // submitted
    out6[1] = s->n_done;                // completed
    out6[2] = s->n_batches;             // launches (batches)
    out6[3] = s->max_batch_seen;        // largest batch so far
    out6[4] = s->reserved_bytes;        // device bytes held for batches and result slots
    int64_t q = 0;
    for (const Family &f : s->fam) q += (int64_t)f.pending.size();
    out6[5] = q;                        // queued, not yet launched
    return JFG_OK;
}

jfg_status jfg_server_family_batch(jfg_server *s, int32_t family, int32_t *batch_limit) {
    if (!s || family < 0 || family >= (int)s->fam.size() || !batch_limit) return JFG_ERR_INVALID;
    *batch_limit = s->fam[family].B;
    return JFG_OK;
}

jfg_status jfg_server_hold(jfg_server *s, int32_t hold) {
    if (!s) return JFG_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->hold = hold != 0;
    }
    s->cv.notify_all();
    return JFG_OK;
}

const char *jfg_server_last_error(jfg_server *s) { return s ? s->err.c_str() : "null server"; }

void jfg_server_destroy(jfg_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    s->done_cv.notify_all();
    if (s->th.joinable()) s->th.join();
    for (Family &f : s->fam) {
        if (f.stream) {
            cudaStreamSynchronize(f.stream);   // lets pending host functions run
            if (f.m) jfg_set_stream(f.m, nullptr);
            cudaStreamDestroy(f.stream);
        }
    }
    for (void *p : s->allocs) cudaFree(p);
    for (void *p : s->pinned) cudaFreeHost(p);
    delete s;
}

}  // extern "C"
