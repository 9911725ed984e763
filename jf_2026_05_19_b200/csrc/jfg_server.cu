// jfg_server.cu -- device-resident request loop over model families.
//
// Serving pattern of the reference's optimisation worker
// (tools/jfem_worker_jsonl.jl:132-148, manifest_batch_core.jl:283-409): many
// property-update requests against a few models.  Here each family's mesh,
// CSC pattern and scatter maps stay on the GPU; a request carries a new
// shell-thickness vector and asks for K and KG of that family (membrane
// stress recovery from the family's displacement field is part of KG).
// Results stay on the device until the client releases them.
//
// Launch units.  A family is served through a unit: its own jfg_model handle,
// or one member of a group handle (jfg_group_create) shared with other
// families.  A batch is one batched launch sequence on one unit
// (jfg_assemble_batch_device_ws): n variants, each variant a full thickness
// vector of the unit.  For a group unit, variant v carries the v-th queued
// request of every member family that has one; members with nothing queued
// are computed at their current thickness (the handle's own) and discarded.
// So requests of different (small) families share one launch.
//
// Admission by HBM budget.  One device pool of hbm_budget_bytes holds every
// batch's workspace (element staging per variant) and results (K, KG, max,
// thickness per variant).  A batch takes both out of the pool when it is
// formed, as many variants as are queued (up to max_batch) and fit; the
// workspace goes back when the batch's kernels finish, the results when the
// last of its requests is released.  A request waits only while its unit has
// two batches in flight or the pool lacks room, so memory freed by any family
// admits the next batch of any other.
//
// Policies:
//   JFG_SERVE_BATCHED  continuous batching as above; units run on their own
//                      streams, so their batches overlap on the device.
//   JFG_SERVE_SERIAL   the plain path: one request per launch, in arrival
//                      order, each finished before the next starts.
// Completion times come from a host function enqueued behind each batch.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/jfem_gpu.h"

namespace {

constexpr int kInflightPerUnit = 2;
constexpr int64_t kAlign = 256;

inline int64_t align_up(int64_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

// First-fit allocator over the offsets of one device region, with
// neighbouring free ranges merged on release.  Host bookkeeping only.
class Pool {
  public:
    void reset(int64_t size) {
        size_ = size;
        free_.clear();
        free_[0] = size;
        used_ = peak_ = 0;
    }
    bool alloc(int64_t bytes, int64_t *off) {
        bytes = align_up(std::max<int64_t>(bytes, 1));
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= bytes) {
                *off = it->first;
                const int64_t rest = it->second - bytes;
                const int64_t o = it->first;
                free_.erase(it);
                if (rest) free_[o + bytes] = rest;
                used_ += bytes;
                peak_ = std::max(peak_, used_);
                return true;
            }
        return false;
    }
    void release(int64_t off, int64_t bytes) {
        bytes = align_up(std::max<int64_t>(bytes, 1));
        used_ -= bytes;
        auto next = free_.lower_bound(off);
        int64_t o = off, n = bytes;
        if (next != free_.end() && next->first == off + bytes) { n += next->second; next = free_.erase(next); }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) { o = prev->first; n += prev->second; free_.erase(prev); }
        }
        free_[o] = n;
    }
    int64_t peak() const { return peak_; }

  private:
    int64_t size_ = 0, used_ = 0, peak_ = 0;
    std::map<int64_t, int64_t> free_;
};

struct SrvRequest {
    int64_t ticket = 0;
    int family = 0;
    std::vector<double> h;      // thickness vector, copied at submit
    bool keep = true;           // results kept until jfg_server_release
    bool freed = false;         // keep == false: results dropped at completion
    int state = 0;              // 0 queued, 1 launched, 2 done
    int64_t batch = 0;          // batch id while its results are held
    int var = -1;
    double t_submit = 0, t_launch = 0, t_done = 0;
};

struct Family {
    int unit = 0, member = 0;             // member index inside a group unit (0 for a plain handle)
    int64_t nq = 0, nt = 0;               // the family's CQUAD4 / CTRIA3 counts
    int64_t q_off = 0, t_off = 0;         // offsets of its thicknesses in the unit's CQUAD4 / CTRIA3 sections
    int64_t nnz = 0, nnz_off = 0;         // its nonzeros inside the unit's value array
    int B = 1;                            // batch limit
    std::deque<int64_t> pending;
};

struct Unit {
    jfg_model *m = nullptr;
    cudaStream_t stream = nullptr;
    int64_t ndof = 0, nnz = 0, nq = 0, nt = 0;
    double *u_dev = nullptr;              // displacement field for KG, or null (K only)
    std::vector<int> fams;                // families in member order
    std::vector<double> base_h;           // the handle's own thicknesses: filler for idle members
    int64_t ws1 = 0;                      // workspace bytes per variant
    int B = 1;                            // variants per batch at most
    int inflight = 0;
    double *pin[kInflightPerUnit] = {nullptr, nullptr};   // pinned thickness staging, one per in-flight batch
    bool pin_busy[kInflightPerUnit] = {false, false};
    int64_t shell() const { return nq + nt; }
    int64_t out1() const { return 8 * (nnz * (u_dev ? 2 : 1) + 1 + shell()); }  // result bytes per variant
};

}  // namespace

struct jfg_server;

namespace {
struct SrvBatch {
    jfg_server *s = nullptr;
    int64_t id = 0;
    int unit = 0, n_var = 0, pin = 0;
    int64_t ws_off = 0, ws_bytes = 0, out_off = 0, out_bytes = 0;
    double *nzk = nullptr, *nzkg = nullptr, *max = nullptr, *h_dev = nullptr;
    std::vector<int64_t> tickets;
    int unreleased = 0;
    bool running = true;
};
}  // namespace

struct jfg_server {
    std::vector<Unit> units;
    std::vector<Family> fam;
    int policy = JFG_SERVE_BATCHED;
    std::mutex mu;
    std::condition_variable cv;        // wakes the scheduler
    std::condition_variable done_cv;   // wakes waiting clients
    std::thread th;
    bool stop = false;
    bool hold = false;                 // queue requests without launching (jfg_server_hold)
    std::unordered_map<int64_t, SrvRequest> reqs;
    std::unordered_map<int64_t, SrvBatch *> batches;
    std::deque<int64_t> fifo;          // arrival order (serial policy)
    int64_t next_ticket = 1, next_batch = 1;
    int64_t n_done = 0, n_batches = 0, max_batch_seen = 0;
    char *pool_base = nullptr;
    int64_t pool_bytes = 0;
    Pool pool;
    int rr = 0;                        // round-robin start among units
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

// Releases the batch's results once every request is released or dropped
// (lock held).
void maybe_free_results(jfg_server *s, SrvBatch *b) {
    if (b->running || b->unreleased > 0) return;
    s->pool.release(b->out_off, b->out_bytes);
    s->batches.erase(b->id);
    delete b;
}

// Runs on a CUDA host thread once the batch's kernels have finished.  No
// CUDA calls here: pool bookkeeping, completion times, wake-ups.
void CUDART_CB batch_done(void *p) {
    SrvBatch *b = static_cast<SrvBatch *>(p);
    jfg_server *s = b->s;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const double t = s->now();
        Unit &u = s->units[b->unit];
        for (int64_t tk : b->tickets) {
            auto it = s->reqs.find(tk);
            if (it == s->reqs.end()) continue;
            it->second.state = 2;
            it->second.t_done = t;
            if (!it->second.keep) {  // results dropped now; the record (times) stays until released
                it->second.freed = true;
                b->unreleased -= 1;
            }
        }
        s->n_done += (int64_t)b->tickets.size();
        s->pool.release(b->ws_off, b->ws_bytes);   // the workspace is free as soon as the kernels are done
        u.inflight -= 1;
        u.pin_busy[b->pin] = false;
        b->running = false;
        maybe_free_results(s, b);
    }
    s->cv.notify_all();
    s->done_cv.notify_all();
}

// Launches one batch (lock not held).
jfg_status launch_batch(jfg_server *s, SrvBatch *b) {
    Unit &u = s->units[b->unit];
    SCK(cudaMemcpyAsync(b->h_dev, u.pin[b->pin], sizeof(double) * u.shell() * b->n_var, cudaMemcpyHostToDevice, u.stream));
    jfg_status st = jfg_assemble_batch_device_ws(u.m, b->n_var, s->pool_base + b->ws_off, b->ws_bytes, b->h_dev, nullptr,
                                                 u.u_dev, 0, b->nzk, b->max, nullptr, u.u_dev ? b->nzkg : nullptr);
    if (st) return sfail(s, st, std::string("batched assembly: ") + jfg_last_error(u.m));
    SCK(cudaLaunchHostFunc(u.stream, batch_done, b));
    return JFG_OK;
}

// Variants a batch of unit ui would carry now: the largest queue among its
// families, at most the unit's limit (one for the serial policy).
int demand(const jfg_server *s, int ui, int limit) {
    size_t d = 0;
    for (int f : s->units[ui].fams) d = std::max(d, s->fam[f].pending.size());
    return (int)std::min<size_t>(d, (size_t)limit);
}

// Forms a batch of unit ui with up to `limit` variants that fit the pool
// (lock held); null when nothing can start now.
SrvBatch *form_batch(jfg_server *s, int ui, int limit) {
    Unit &u = s->units[ui];
    if (u.inflight >= kInflightPerUnit) return nullptr;
    int n = demand(s, ui, limit);
    if (n < 1) return nullptr;
    int pin = u.pin_busy[0] ? 1 : 0;
    if (u.pin_busy[pin]) return nullptr;
    int64_t ws_off = 0, out_off = 0;
    for (; n >= 1; n = n > 1 ? n / 2 : 0) {   // shrink until workspace and results both fit
        if (!s->pool.alloc(u.ws1 * n, &ws_off)) continue;
        if (s->pool.alloc(u.out1() * n, &out_off)) break;
        s->pool.release(ws_off, u.ws1 * n);
    }
    if (n < 1) return nullptr;
    SrvBatch *b = new SrvBatch;
    b->s = s;
    b->id = s->next_batch++;
    b->unit = ui;
    b->n_var = n;
    b->pin = pin;
    b->ws_off = ws_off;
    b->ws_bytes = u.ws1 * n;
    b->out_off = out_off;
    b->out_bytes = u.out1() * n;
    double *o = reinterpret_cast<double *>(s->pool_base + out_off);
    b->nzk = o;
    b->nzkg = u.u_dev ? o + (int64_t)n * u.nnz : nullptr;
    b->max = o + (int64_t)n * u.nnz * (u.u_dev ? 2 : 1);
    b->h_dev = b->max + n;
    u.pin_busy[pin] = true;
    // thickness of every variant: the queued requests of each member in
    // order, the member's current thickness where its queue runs out
    const double t = s->now();
    double *hp = u.pin[pin];
    for (int v = 0; v < n; ++v) {
        double *hv = hp + (int64_t)v * u.shell();
        for (int f : u.fams) {
            Family &fm = s->fam[f];
            const double *src = nullptr;
            if (!fm.pending.empty()) {
                const int64_t tk = fm.pending.front();
                fm.pending.pop_front();
                SrvRequest &r = s->reqs[tk];
                r.state = 1;
                r.batch = b->id;
                r.var = v;
                r.t_launch = t;
                b->tickets.push_back(tk);
                src = r.h.data();
                std::memcpy(hv + fm.q_off, src, sizeof(double) * fm.nq);
                std::memcpy(hv + u.nq + fm.t_off, src + fm.nq, sizeof(double) * fm.nt);
                std::vector<double>().swap(r.h);  // the pinned copy is the one the launch reads
            } else {
                std::memcpy(hv + fm.q_off, u.base_h.data() + fm.q_off, sizeof(double) * fm.nq);
                std::memcpy(hv + u.nq + fm.t_off, u.base_h.data() + u.nq + fm.t_off, sizeof(double) * fm.nt);
            }
        }
    }
    b->unreleased = (int)b->tickets.size();
    s->batches[b->id] = b;
    u.inflight += 1;
    s->n_batches += 1;
    s->max_batch_seen = std::max<int64_t>(s->max_batch_seen, (int64_t)n);
    return b;
}

void scheduler(jfg_server *s) {
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        if (s->hold) {
            s->cv.wait_for(lk, std::chrono::milliseconds(50));
            continue;
        }
        std::vector<SrvBatch *> ready;
        if (s->policy == JFG_SERVE_SERIAL) {
            // one request per launch, in arrival order, each completed before the next
            if (!s->fifo.empty()) {
                const int64_t tk = s->fifo.front();
                auto it = s->reqs.find(tk);
                if (it == s->reqs.end()) { s->fifo.pop_front(); continue; }
                const int ui = s->fam[it->second.family].unit;
                Unit &u = s->units[ui];
                if (u.inflight == 0) {
                    SrvBatch *b = form_batch(s, ui, 1);
                    if (b) {
                        s->fifo.pop_front();
                        lk.unlock();
                        jfg_status st = launch_batch(s, b);
                        if (st == JFG_OK) cudaStreamSynchronize(u.stream);
                        lk.lock();
                        if (st) s->stop = true;
                        continue;
                    }
                }
            }
        } else {
            const int nu = (int)s->units.size();
            for (int k = 0; k < nu; ++k) {
                const int ui = (s->rr + k) % nu;
                while (SrvBatch *b = form_batch(s, ui, s->units[ui].B)) ready.push_back(b);
            }
            s->rr = (s->rr + 1) % std::max(nu, 1);
            if (!ready.empty()) {
                lk.unlock();
                bool bad = false;
                for (SrvBatch *b : ready)
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

jfg_status jfg_server_create_units(jfg_model *const *units, const double *const *u_host, int32_t n_units,
                                   const int32_t *family_unit, const int32_t *family_member, int32_t n_families,
                                   int64_t hbm_budget_bytes, int32_t max_batch, int32_t policy, jfg_server **out) {
    if (!units || n_units < 1 || !family_unit || !family_member || n_families < 1 || !out || max_batch < 1 ||
        hbm_budget_bytes <= 0 || (policy != JFG_SERVE_BATCHED && policy != JFG_SERVE_SERIAL))
        return JFG_ERR_INVALID;
    *out = nullptr;
    jfg_server *s = new jfg_server;
    s->policy = policy;
    s->t0 = std::chrono::steady_clock::now();
    s->units.resize(n_units);
    s->fam.resize(n_families);
    auto fail_free = [&](jfg_status st) {
        jfg_server_destroy(s);
        return st;
    };
    for (int i = 0; i < n_units; ++i) {
        Unit &u = s->units[i];
        u.m = units[i];
        if (!u.m) return fail_free(JFG_ERR_INVALID);
        int64_t counts[4];
        if (jfg_model_counts(u.m, counts) || jfg_pattern(u.m, &u.ndof, &u.nnz)) return fail_free(JFG_ERR_STATE);
        u.nq = counts[1];
        u.nt = counts[2];
        if (jfg_batch_workspace_bytes(u.m, 1, &u.ws1)) return fail_free(JFG_ERR_STATE);
        u.ws1 = align_up(u.ws1);
        u.base_h.resize(std::max<int64_t>(u.shell(), 1));
        if (jfg_shell_thickness(u.m, u.base_h.data())) return fail_free(JFG_ERR_STATE);
        if (cudaStreamCreateWithFlags(&u.stream, cudaStreamNonBlocking) != cudaSuccess) return fail_free(JFG_ERR_CUDA);
        if (jfg_set_stream(u.m, u.stream)) return fail_free(JFG_ERR_STATE);
        if (u_host && u_host[i]) {
            if (cudaMalloc((void **)&u.u_dev, sizeof(double) * u.ndof) != cudaSuccess) return fail_free(JFG_ERR_NOMEM);
            s->allocs.push_back(u.u_dev);
            if (cudaMemcpy(u.u_dev, u_host[i], sizeof(double) * u.ndof, cudaMemcpyHostToDevice) != cudaSuccess)
                return fail_free(JFG_ERR_CUDA);
        }
        // the largest batch that fits the budget alone, at most max_batch
        const int64_t per = u.ws1 + align_up(u.out1());
        u.B = (int)std::min<int64_t>(std::min<int64_t>(max_batch, hbm_budget_bytes / std::max<int64_t>(per, 1)), 65535);
        if (u.B < 1) {
            jfg_server_destroy(s);
            return JFG_ERR_NOMEM;
        }
        for (auto &p : u.pin) {
            if (cudaMallocHost((void **)&p, sizeof(double) * std::max<int64_t>(u.B * u.shell(), 1)) != cudaSuccess)
                return fail_free(JFG_ERR_NOMEM);
            s->pinned.push_back(p);
        }
    }
    // families: a plain unit carries one; a group unit one per member
    for (int f = 0; f < n_families; ++f) {
        const int ui = family_unit[f], mi = family_member[f];
        if (ui < 0 || ui >= n_units) return fail_free(JFG_ERR_INVALID);
        Unit &u = s->units[ui];
        Family &fm = s->fam[f];
        fm.unit = ui;
        fm.member = mi;
        int64_t g[8];
        if (mi < 0) {
            if (!u.fams.empty()) return fail_free(JFG_ERR_INVALID);   // a plain handle serves one family
            fm.nq = u.nq; fm.nt = u.nt; fm.q_off = 0; fm.t_off = 0; fm.nnz = u.nnz; fm.nnz_off = 0;
        } else {
            if (jfg_group_member(u.m, mi, g)) return fail_free(JFG_ERR_INVALID);
            if (policy == JFG_SERVE_SERIAL) return fail_free(JFG_ERR_INVALID);  // the plain path serves plain handles
            // member counts: the next member's offsets (or the group's totals) minus its own
            int64_t next[8];
            const bool last = jfg_group_member(u.m, mi + 1, next) != JFG_OK;
            fm.nq = (last ? u.nq : next[4]) - g[4];
            fm.nt = (last ? u.nt : next[5]) - g[5];
            fm.q_off = g[4];
            fm.t_off = g[5];
            fm.nnz = g[2];
            fm.nnz_off = g[3];
        }
        u.fams.push_back(f);
        fm.B = u.B;
    }
    for (auto &u : s->units)
        if (u.fams.empty()) return fail_free(JFG_ERR_INVALID);
    if (cudaMalloc((void **)&s->pool_base, hbm_budget_bytes) != cudaSuccess) return fail_free(JFG_ERR_NOMEM);
    s->allocs.push_back(s->pool_base);
    s->pool_bytes = hbm_budget_bytes;
    s->pool.reset(hbm_budget_bytes);
    s->th = std::thread(scheduler, s);
    *out = s;
    return JFG_OK;
}

jfg_status jfg_server_create(jfg_model *const *families, const double *const *u_host, int32_t n_families,
                             int64_t hbm_budget_bytes, int32_t max_batch, int32_t policy, jfg_server **out) {
    if (n_families < 1) return JFG_ERR_INVALID;
    std::vector<int32_t> unit(n_families), member(n_families, -1);
    for (int i = 0; i < n_families; ++i) unit[i] = i;
    return jfg_server_create_units(families, u_host, n_families, unit.data(), member.data(), n_families, hbm_budget_bytes,
                                   max_batch, policy, out);
}

jfg_status jfg_server_submit(jfg_server *s, int32_t family, const double *h_host, int32_t keep, int64_t *ticket) {
    if (!s) return JFG_ERR_INVALID;
    if (family < 0 || family >= (int)s->fam.size() || !h_host || !ticket)
        return sfail(s, JFG_ERR_INVALID, "bad family, thickness pointer or ticket pointer");
    const Family &f = s->fam[family];
    const int64_t ns = f.nq + f.nt;
    for (int64_t e = 0; e < ns; ++e)
        if (!(h_host[e] > 0.0)) return sfail(s, JFG_ERR_INVALID, "shell thickness must be positive");
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return sfail(s, JFG_ERR_STATE, "server stopped: " + s->err);
        const int64_t tk = s->next_ticket++;
        SrvRequest &r = s->reqs[tk];
        r.ticket = tk;
        r.family = family;
        r.h.assign(h_host, h_host + ns);
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
    const Unit &u = s->units[f.unit];
    auto bi = s->batches.find(r.batch);
    const SrvBatch *b = (r.freed || bi == s->batches.end()) ? nullptr : bi->second;
    if (nzk_dev) *nzk_dev = b ? b->nzk + (int64_t)r.var * u.nnz + f.nnz_off : nullptr;
    if (nzkg_dev) *nzkg_dev = (b && b->nzkg) ? b->nzkg + (int64_t)r.var * u.nnz + f.nnz_off : nullptr;
    if (max_dev) *max_dev = b ? b->max + r.var : nullptr;
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
        const bool freed = it->second.freed;
        const int64_t bid = it->second.batch;
        s->reqs.erase(it);
        if (!freed) {
            auto bi = s->batches.find(bid);
            if (bi != s->batches.end()) {
                bi->second->unreleased -= 1;
                maybe_free_results(s, bi->second);
            }
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
    out6[4] = s->pool.peak();           // most pool bytes in use at once
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
    for (Unit &u : s->units) {
        if (u.stream) {
            cudaStreamSynchronize(u.stream);   // lets pending host functions run
            if (u.m) jfg_set_stream(u.m, nullptr);
            cudaStreamDestroy(u.stream);
        }
    }
    for (auto &kv : s->batches) delete kv.second;
    for (void *p : s->allocs) cudaFree(p);
    for (void *p : s->pinned) cudaFreeHost(p);
    delete s;
}

}  // extern "C"
