// serve.cu -- continuous-batching request loop over libchy_pot3 plans.
//
// Requests (a grid descriptor, host RHO in, host PHI out) are queued by
// chy_server_submit from any thread.  One dispatcher thread:
//   * keeps one size class per distinct grid: plans (tables + work space) that
//     stay resident on the device and are reused by every later request of
//     that grid, two "lanes" per class, each with up to two batches in flight
//     on three streams (copies in, solves, copies out), so that a batch's
//     copies overlap the solves and copies of the others;
//   * admits waiting requests into a free lane as soon as device buffers for
//     them fit in the arena (the HBM budget left after the plans), up to the
//     plan's batch size -- requests that arrive while others are on the GPU
//     join the next batch of their class instead of waiting for the queue to
//     drain;
//   * runs every class on its own streams, so batches of different grids run
//     concurrently on the device;
//   * retires a batch when its event completes and wakes the waiters.
// A solve's result does not depend on what it is batched with: every kernel
// reduces in a fixed order per solve.
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
#include <unordered_map>
#include <vector>

#include "chy_pot3.h"
#include "planimpl.h"

using namespace chy;

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kLanes = 2;
constexpr int kLaneDepth = 2;   // batches in flight per lane

struct Request {
    long long id = 0;
    std::string key;
    chy_grid g{};
    std::vector<double> r, z, rhf, zhf;   // copies of the caller's grid arrays (if given)
    const double *rho = nullptr;
    double *phi = nullptr;
    Clock::time_point t_submit;
    double latency_ms = 0.0;
    int status = CHY_OK;
    bool done = false;
    size_t buf_off = 0;                   // device buffers [rho | phi] in the arena
};

// One batch in flight: its requests, the events that order its copies in,
// solve and copies out, and the pinned word its mode solve's error word is
// read back into.
struct Slot {
    std::vector<Request *> batch;
    cudaEvent_t in = nullptr, solved = nullptr, done = nullptr;
    int *err = nullptr;
};

struct Lane {
    chy_plan *plan = nullptr;
    cudaStream_t stream = nullptr;                 // solves (in order: they share the plan's work space)
    cudaStream_t s_in = nullptr, s_out = nullptr;  // host -> device, device -> host copies
    Slot slots[kLaneDepth];
    bool idle() const
    {
        for (const Slot &sl : slots)
            if (!sl.batch.empty()) return false;
        return true;
    }
};

int lane_streams(Lane &ln)
{
    if (cudaStreamCreateWithFlags(&ln.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ln.s_in, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ln.s_out, cudaStreamNonBlocking) != cudaSuccess)
        return CHY_ERR_CUDA;
    for (Slot &sl : ln.slots)
        if (cudaEventCreateWithFlags(&sl.in, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.solved, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost(&sl.err, sizeof(int)) != cudaSuccess)
            return CHY_ERR_CUDA;
    return CHY_OK;
}

void lane_free(Lane &ln)
{
    if (ln.plan) chy_plan_destroy(ln.plan);
    for (cudaStream_t st : {ln.stream, ln.s_in, ln.s_out})
        if (st) cudaStreamDestroy(st);
    for (Slot &sl : ln.slots) {
        for (cudaEvent_t ev : {sl.in, sl.solved, sl.done})
            if (ev) cudaEventDestroy(ev);
        if (sl.err) cudaFreeHost(sl.err);
    }
    ln = Lane{};
}

struct SizeClass {
    std::string key;
    size_t nvol = 0, req_bytes = 0;
    int J = 0, K = 0, L = 0;
    Lane lanes[kLanes];
    std::deque<Request *> waiting;
    Clock::time_point last_use;
};

// First-fit allocator over one device arena (offsets, 256-byte granules).
class Arena {
  public:
    size_t size = 0;
    std::map<size_t, size_t> free_;   // offset -> bytes
    void reset(size_t bytes)
    {
        size = bytes;
        free_.clear();
        if (bytes) free_[0] = bytes;
    }
    bool alloc(size_t bytes, size_t *off)
    {
        bytes = (bytes + 255) & ~(size_t)255;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes, o = it->first + bytes;
            free_.erase(it);
            if (rest) free_[o] = rest;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes)
    {
        bytes = (bytes + 255) & ~(size_t)255;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

std::string grid_key(const chy_grid &g, int precision)
{
    // every field that shapes the plan (field by field: no padding bytes);
    // grid arrays by content
    std::string k;
    auto put = [&](const void *p, size_t n) { k.append((const char *)p, n); };
    put(&g.jmax, sizeof g.jmax);
    put(&g.kmax, sizeof g.kmax);
    put(&g.lmax, sizeof g.lmax);
    put(&g.rof3n, sizeof g.rof3n);
    put(&g.zof3n, sizeof g.zof3n);
    put(&g.pi, sizeof g.pi);
    put(&g.grav, sizeof g.grav);
    put(&g.isym, sizeof g.isym);
    put(&g.maxtrm, sizeof g.maxtrm);
    put(&g.redge, sizeof g.redge);
    put(&g.npoint, sizeof g.npoint);
    put(&g.literal_kind, sizeof g.literal_kind);
    put(&precision, sizeof precision);
    auto add = [&](const double *a, int n) {
        if (a) k.append((const char *)a, sizeof(double) * n);
        k.push_back(a ? 'a' : 'u');
    };
    add(g.r, g.jmax + 2);
    add(g.z, g.kmax + 2);
    add(g.rhf, g.jmax + 2);
    add(g.zhf, g.kmax + 2);
    return k;
}

}  // namespace

struct chy_server {
    int device = 0;
    int precision = CHY_PREC_MIXED;
    int max_batch = 8;
    size_t budget = 0, plan_bytes = 0;
    char *arena_base = nullptr;
    Arena arena;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> incoming;
    std::unordered_map<long long, std::unique_ptr<Request>> requests;
    std::map<std::string, std::unique_ptr<SizeClass>> classes;
    long long next_id = 1;
    bool stop = false;
    long long completed = 0, batches = 0;
    std::thread worker;

    void run();
    int launch(SizeClass &c, Lane &ln, Slot &sl);
    void retire(SizeClass &c, Slot &sl, int status);
    int make_class(Request *rq, SizeClass **out);
};

int chy_server::make_class(Request *rq, SizeClass **out)
{
    auto c = std::make_unique<SizeClass>();
    c->key = rq->key;
    c->J = rq->g.jmax;
    c->K = rq->g.kmax;
    c->L = rq->g.lmax;
    c->nvol = (size_t)(c->J + 2) * (c->K + 2) * c->L;
    c->req_bytes = 2 * c->nvol * sizeof(double);
    chy_grid g = rq->g;
    g.r = rq->r.empty() ? nullptr : rq->r.data();
    g.z = rq->z.empty() ? nullptr : rq->z.data();
    g.rhf = rq->rhf.empty() ? nullptr : rq->rhf.data();
    g.zhf = rq->zhf.empty() ? nullptr : rq->zhf.data();
    for (int i = 0; i < kLanes; i++) {
        Lane &ln = c->lanes[i];
        int prec = precision;
        int st = chy_plan_create(&g, prec, max_batch, &ln.plan);
        if (st == CHY_ERR_UNSUPPORTED && prec == CHY_PREC_MIXED) {   // grids the mixed path does not cover
            prec = CHY_PREC_FP64;
            st = chy_plan_create(&g, prec, max_batch, &ln.plan);
        }
        if (st == CHY_OK) {
            plan_bytes += (size_t)chy_plan_device_bytes(ln.plan);
            st = lane_streams(ln);
        }
        if (st != CHY_OK) {
            for (int k = 0; k <= i; k++) {
                if (c->lanes[k].plan) plan_bytes -= (size_t)chy_plan_device_bytes(c->lanes[k].plan);
                lane_free(c->lanes[k]);
            }
            return st;
        }
    }
    c->last_use = Clock::now();
    // plans count against the budget left after the arena: drop idle classes
    // (least recently used first) to make room, else give up on this grid
    while (plan_bytes > budget - arena.size) {
        SizeClass *victim = nullptr;
        for (auto &kv : classes) {
            SizeClass &o = *kv.second;
            bool idle = o.waiting.empty();
            for (Lane &ln : o.lanes) idle = idle && ln.idle();
            if (idle && (!victim || o.last_use < victim->last_use)) victim = &o;
        }
        if (!victim) break;
        for (Lane &ln : victim->lanes) {
            plan_bytes -= (size_t)chy_plan_device_bytes(ln.plan);
            lane_free(ln);
        }
        classes.erase(victim->key);
    }
    if (plan_bytes > budget - arena.size || c->req_bytes > arena.size) {
        for (Lane &ln : c->lanes) {
            plan_bytes -= (size_t)chy_plan_device_bytes(ln.plan);
            lane_free(ln);
        }
        return CHY_ERR_CAPACITY;
    }
    *out = c.get();
    classes[c->key] = std::move(c);
    return CHY_OK;
}

// Copies the slot's batch in (s_in), solves it (the lane's solve stream, after
// the lane's earlier batches) and copies it out (s_out).
int chy_server::launch(SizeClass &c, Lane &ln, Slot &sl)
{
    BatchPtrs bp{};
    const int nb = (int)sl.batch.size();
    const double *mapped[kMaxBatchPtrs] = {};
    for (int i = 0; i < nb; i++) {
        Request *rq = sl.batch[i];
        double *dr = reinterpret_cast<double *>(arena_base + rq->buf_off), *df = dr + c.nvol;
        if (copy_rho_in(dr, rq->rho, c.J, c.K, c.L, ln.s_in) != cudaSuccess) return CHY_ERR_CUDA;
        // the cells the solve leaves alone go back with the rest of PHI: read
        // by a kernel from pinned (mapped) host memory, else copied
        mapped[i] = chy_internal_mapped_view(rq->phi);
        if (!mapped[i] && copy_phi_rim(df, rq->phi, c.J, c.K, c.L, cudaMemcpyHostToDevice, ln.s_in) != cudaSuccess)
            return CHY_ERR_CUDA;
        bp.rho[i] = dr;
        bp.phi[i] = df;
    }
    if (cudaEventRecord(sl.in, ln.s_in) != cudaSuccess || cudaStreamWaitEvent(ln.stream, sl.in, 0) != cudaSuccess)
        return CHY_ERR_CUDA;
    for (int i = 0; i < nb; i++)
        if (mapped[i] && chy_internal_rim_in(bp.phi[i], mapped[i], c.J, c.K, c.L, ln.stream) != cudaSuccess)
            return CHY_ERR_CUDA;
    int st = chy_internal_run_batch(ln.plan, bp, nb, ln.stream);
    if (st != CHY_OK) return st;
    // the mode solve's error word, read back with the batch into the slot's own
    // word (checked at retirement; no-op for other precisions)
    *sl.err = 0;
    st = chy_mixed_read_error(ln.plan, sl.err, ln.stream);
    if (st != CHY_OK) return st;
    if (cudaEventRecord(sl.solved, ln.stream) != cudaSuccess ||
        cudaStreamWaitEvent(ln.s_out, sl.solved, 0) != cudaSuccess)
        return CHY_ERR_CUDA;
    for (int i = 0; i < nb; i++)
        if (copy_phi_out(sl.batch[i]->phi, bp.phi[i], c.J, c.K, c.L, ln.s_out) != cudaSuccess)
            return CHY_ERR_CUDA;
    if (cudaEventRecord(sl.done, ln.s_out) != cudaSuccess) return CHY_ERR_CUDA;
    return CHY_OK;
}

void chy_server::retire(SizeClass &c, Slot &sl, int status)
{
    const auto now = Clock::now();
    for (Request *rq : sl.batch) {
        arena.release(rq->buf_off, c.req_bytes);
        rq->status = status;
        rq->latency_ms = std::chrono::duration<double, std::milli>(now - rq->t_submit).count();
        rq->done = true;
        completed++;
    }
    sl.batch.clear();
    c.last_use = now;
}

void chy_server::run()
{
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        bool progress = false;
        // new requests -> their size class (created on first use)
        while (!incoming.empty()) {
            Request *rq = incoming.front();
            incoming.pop_front();
            auto it = classes.find(rq->key);
            SizeClass *c = nullptr;
            if (it != classes.end()) {
                c = it->second.get();
            } else {
                const int st = make_class(rq, &c);
                if (st != CHY_OK) {
                    rq->status = st;
                    rq->done = true;
                    completed++;
                    progress = true;
                    continue;
                }
            }
            if (rq->g.jmax != c->J || rq->g.kmax != c->K || rq->g.lmax != c->L) {
                rq->status = CHY_ERR_ARG;
                rq->done = true;
                completed++;
                progress = true;
                continue;
            }
            c->waiting.push_back(rq);
        }
        // retire finished batches
        for (auto &kv : classes)
            for (Lane &ln : kv.second->lanes)
                for (Slot &sl : ln.slots)
                    if (!sl.batch.empty()) {
                        const cudaError_t e = cudaEventQuery(sl.done);
                        if (e == cudaErrorNotReady) continue;
                        retire(*kv.second, sl, e != cudaSuccess ? CHY_ERR_CUDA : *sl.err ? CHY_ERR_TIMEOUT : CHY_OK);
                        progress = true;
                    }
        // admit waiting requests into free slots while their buffers fit: the
        // lanes' first slots before their second ones, so that batches spread
        // over both lanes' solve streams
        for (auto &kv : classes) {
            SizeClass &c = *kv.second;
            bool full = false;
            for (int d = 0; d < kLaneDepth && !full; d++)
                for (Lane &ln : c.lanes) {
                    if (c.waiting.empty()) break;
                    Slot &sl = ln.slots[d];
                    if (!sl.batch.empty()) continue;
                    while (!c.waiting.empty() && (int)sl.batch.size() < max_batch) {
                        size_t off = 0;
                        if (!arena.alloc(c.req_bytes, &off)) break;
                        Request *rq = c.waiting.front();
                        c.waiting.pop_front();
                        rq->buf_off = off;
                        sl.batch.push_back(rq);
                    }
                    if (sl.batch.empty()) {   // arena full: retry after a retirement
                        full = true;
                        break;
                    }
                    lk.unlock();
                    const int st = launch(c, ln, sl);
                    if (st != CHY_OK) {   // nothing may still use the buffers
                        cudaStreamSynchronize(ln.s_in);
                        cudaStreamSynchronize(ln.stream);
                        cudaStreamSynchronize(ln.s_out);
                    }
                    lk.lock();
                    if (st != CHY_OK) retire(c, sl, st);
                    else batches++;
                    progress = true;
                }
        }
        if (progress) cv_done.notify_all();
        if (stop && incoming.empty()) {
            bool idle = true;
            for (auto &kv : classes) {
                if (!kv.second->waiting.empty()) idle = false;
                for (Lane &ln : kv.second->lanes)
                    if (!ln.idle()) idle = false;
            }
            if (idle) break;
        }
        if (!progress) cv_work.wait_for(lk, std::chrono::microseconds(50));
    }
}

extern "C" {

int chy_server_create(const chy_server_opts *o, chy_server **out)
{
    if (!out) return chy_internal_fail(CHY_ERR_ARG, "chy_server_create: null output pointer");
    *out = nullptr;
    auto s = std::make_unique<chy_server>();
    s->precision = o ? o->precision : CHY_PREC_MIXED;
    if (s->precision != CHY_PREC_FP64 && s->precision != CHY_PREC_MIXED && s->precision != CHY_PREC_FP64_BLKTRI)
        return chy_internal_fail(CHY_ERR_ARG, "chy_server_create: precision must be CHY_PREC_FP64, _MIXED or _FP64_BLKTRI");
    if (cudaGetDevice(&s->device) != cudaSuccess) return chy_internal_fail(CHY_ERR_CUDA, "chy_server_create: no device");
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
        return chy_internal_fail(CHY_ERR_CUDA, "chy_server_create: cudaMemGetInfo failed");
    s->budget = (o && o->hbm_budget > 0) ? (size_t)o->hbm_budget : free_b / 4 * 3;
    s->max_batch = (o && o->max_batch > 0) ? std::min(o->max_batch, (int)kMaxBatchPtrs) : 8;
    // request buffers get the arena fraction of the budget; plans the rest
    const double frac = (o && o->arena_fraction > 0.0 && o->arena_fraction < 1.0) ? o->arena_fraction : 0.5;
    const size_t arena = ((size_t)(s->budget * frac)) & ~(size_t)255;
    if (arena > free_b) return chy_internal_fail(CHY_ERR_NOMEM, "chy_server_create: arena larger than free device memory");
    if (cudaMalloc(&s->arena_base, arena) != cudaSuccess) {
        cudaGetLastError();
        return chy_internal_fail(CHY_ERR_NOMEM, "chy_server_create: arena allocation failed");
    }
    s->arena.reset(arena);
    chy_server *raw = s.release();
    raw->worker = std::thread([raw] { raw->run(); });
    *out = raw;
    return CHY_OK;
}

int chy_server_submit(chy_server *s, const chy_grid *g, const double *rho, double *phi, long long *ticket)
{
    if (!s || !g || !rho || !phi || !ticket) return CHY_ERR_ARG;
    auto rq = std::make_unique<Request>();
    rq->g = *g;
    auto copy = [](const double *a, int n, std::vector<double> &v) {
        if (a) v.assign(a, a + n);
    };
    copy(g->r, g->jmax + 2, rq->r);
    copy(g->z, g->kmax + 2, rq->z);
    copy(g->rhf, g->jmax + 2, rq->rhf);
    copy(g->zhf, g->kmax + 2, rq->zhf);
    rq->key = grid_key(*g, s->precision);
    rq->rho = rho;
    rq->phi = phi;
    rq->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return CHY_ERR_ARG;
        rq->id = s->next_id++;
        *ticket = rq->id;
        s->incoming.push_back(rq.get());
        s->requests[rq->id] = std::move(rq);
    }
    s->cv_work.notify_one();
    return CHY_OK;
}

int chy_server_wait(chy_server *s, long long ticket, double *latency_ms)
{
    if (!s) return CHY_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return CHY_ERR_ARG;
    Request *rq = it->second.get();
    s->cv_done.wait(lk, [&] { return rq->done; });
    const int st = rq->status;
    if (latency_ms) *latency_ms = rq->latency_ms;
    s->requests.erase(it);
    return st;
}

int chy_server_get_stats(chy_server *s, chy_server_stats *out)
{
    if (!s || !out) return CHY_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    out->completed = s->completed;
    out->batches = s->batches;
    out->size_classes = (int)s->classes.size();
    out->plan_bytes = (long long)s->plan_bytes;
    out->arena_bytes = (long long)s->arena.size;
    return CHY_OK;
}

void chy_server_destroy(chy_server *s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_one();
    if (s->worker.joinable()) s->worker.join();
    for (auto &kv : s->classes)
        for (Lane &ln : kv.second->lanes) lane_free(ln);
    cudaFree(s->arena_base);
    delete s;
}

}  // extern "C"
