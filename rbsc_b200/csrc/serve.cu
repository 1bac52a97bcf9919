// serve.cu -- refinement as a service: continuous batching of jobs on one GPU.
//
// No counterpart in the reference, which refines one graph per process run
// (src/rbsc/rbsc.cu:182-497).  A server owns `slots` executors; each is a host
// thread with its own context (stream, buffer pool), so the refinements of
// different slots overlap on the device.  One mutex guards the queue and the
// accounting.  The scheduling step (dispatch) runs whenever a job arrives and
// whenever an executor finishes:
//
//   while an executor is idle and jobs wait:
//     head = the oldest waiting job; but when head is large, every other
//            executor runs a large job and a small job waits, head = the
//            oldest small job (a lane for small jobs: with two or more
//            executors, large jobs hold at most all but one while small jobs
//            wait, so a burst of large jobs does not hold up the small ones;
//            large jobs still start in arrival order as executors free up)
//     head small -> take it and the small jobs waiting behind it, in arrival
//                   order (large ones are passed over), up to the pack limits
//     otherwise  -> take head alone
//     footprint  =  rbsc_serve_footprint(nodes, arcs, weighted, jobs taken)
//     if reserved + footprint > budget: shrink the pack; if even head alone
//        does not fit, stop -- head waits for memory and nothing overtakes
//        it, so no job starves
//     reserved += footprint; hand the work to the idle executor
//
// A pack is refined as the disjoint union of its graphs (rbsc_batch_refine):
// each job receives its graph's local canonical labels and block count, which
// are those of a refinement of the graph alone.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/rbsc.h"
#include "internal.h"

namespace {

using Clock = std::chrono::steady_clock;

thread_local std::string t_serve_error;

rbsc_status serve_fail(rbsc_status code, const char* fmt, ...)
{
    char buf[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_serve_error = buf;
    return code;
}

double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

uint64_t pow2_at_least(uint64_t x)
{
    uint64_t r = 1;
    while (r < x) r <<= 1;
    return r;
}

struct Job {
    uint64_t id = 0;
    rbsc_csr g{};
    const uint32_t* init = nullptr;
    uint32_t* out = nullptr;
    bool small = false;
    bool done = false;
    rbsc_serve_result res{};
    Clock::time_point t_submit, t_start;
};

struct Slot {
    uint32_t index = 0;
    rbsc_ctx* ctx = nullptr;
    std::thread th;
    std::condition_variable cv;
    bool busy = false;            // work handed over and not finished
    bool large = false;           // the work is one large job
    std::vector<Job*> work;
    uint64_t footprint = 0;
    void* stage = nullptr;        // pinned staging of packed batches
    size_t stage_bytes = 0;
};

}  // namespace

struct rbsc_server {
    rbsc_serve_opts o{};
    std::mutex mu;
    std::condition_variable cv_done;
    std::deque<Job*> queue;
    std::unordered_map<uint64_t, Job*> jobs;
    std::vector<Slot*> slots;
    uint64_t next_id = 1;
    bool stopping = false;
    uint32_t busy = 0;
    uint32_t busy_large = 0;      // executors running one large job
    rbsc_serve_stats st{};
};

extern "C" void rbsc_serve_opts_default(rbsc_serve_opts* o)
{
    std::memset(o, 0, sizeof *o);
    o->device = 0;
    o->slots = 2;
    o->hbm_budget = 0;
    o->pack_max_arcs = 1ull << 18;
    o->pack_max_graphs = 4096;
    o->pack_arc_budget = 1ull << 22;
    o->queue_cap = 65536;
    rbsc_opts_default(&o->opts);
}

// Upper estimate of the device bytes one refinement allocates (rbsc.cu:
// graph_alloc_csr, graph_prepare, ensure_refine_bufs, verify_fixpoint; batch.cu
// for packs), with the pool's rounding and the scan / sort temporaries.
extern "C" uint64_t rbsc_serve_footprint(uint64_t n, uint64_t m, int32_t weighted, uint32_t graphs)
{
    const uint64_t N = std::max<uint64_t>(n, 1);
    const uint64_t mpad = (m + 511) / 512 * 512 + 512;
    const uint64_t tab = std::max<uint64_t>(1024, pow2_at_least(2 * N));
    uint64_t b = 0;
    // resident graph: offsets, rows, row offsets, the non-empty scan, tiles, head bitmap, heads
    b += 8 * (N + 1) + 4 * N + 8 * (N + 1) + 4 * (N + 1) + mpad / 128 + mpad / 8 + 4 * mpad;
    // per node: colours, initial labels, signatures, slots, output, ranks, follower
    // pairs, group representatives and counts, two node lists, uploaded colours
    b += N * (4 + 4 + 16 + 4 + 4 + 2 + 8 + 4 + 4 + 8 + 4);
    // relabel tables: 16-B and 8-B entries, 4-B class ranks
    b += tab * 28;
    // compacted arc sets: two copies of heads, bitmap, row data
    b += 2 * (4 * mpad + mpad / 8 + 12 * N + mpad / 128);
    // exact check: per-node lists, and at worst one 8-B key (twice) per arc
    b += N * 32 + 16 * m;
    if (weighted) b += 3 * 8 * mpad + 16 * m;
    // packed batch: sort keys and values, segment heads, histogram, local labels
    if (graphs > 1) b += N * 48 + 24 * (uint64_t)graphs;
    // temporaries and pool rounding
    b += b / 8 + (8ull << 20);
    return b;
}

namespace {

void finish_error(Job* j, rbsc_status s, const char* msg)
{
    j->res.status = s;
    snprintf(j->res.error, sizeof j->res.error, "%s", msg ? msg : "");
}

void run_single(Slot* sl, Job* j)
{
    rbsc_stats st;
    const rbsc_status s = rbsc_refine(sl->ctx, &j->g, j->init, j->out, &st);
    if (s != RBSC_OK) {
        finish_error(j, s, rbsc_last_error(sl->ctx));
        return;
    }
    j->res.status = RBSC_OK;
    j->res.blocks = st.blocks;
    j->res.rounds = st.rounds;
}

template <typename T>
void shift_offsets(const void* src, uint32_t n, uint64_t base, uint64_t* dst)
{
    const T* s = static_cast<const T*>(src);
    for (uint32_t u = 0; u < n; ++u) dst[u] = base + (uint64_t)s[u];
}

// The jobs side by side in pinned staging (global node ids), one batch
// refinement of the union, each job's local labels copied to its output.
void run_pack(Slot* sl, const std::vector<Job*>& js)
{
    rbsc_ctx* ctx = sl->ctx;
    const uint32_t G = (uint32_t)js.size();
    uint64_t N = 0, M = 0;
    bool any_init = false;
    for (Job* j : js) {
        N += j->g.n;
        M += j->g.m;
        any_init |= j->init != nullptr;
    }
    auto al = [](size_t b) { return (b + 63) & ~(size_t)63; };
    const size_t b_off = al(8 * (N + 1)), b_gn = al(8 * ((size_t)G + 1)), b_idx = al(4 * M), b_init = al(4 * N),
                 b_local = al(4 * N), b_blocks = al(4 * (size_t)G);
    const size_t bytes = b_off + b_gn + b_idx + b_init + b_local + b_blocks;
    if (bytes > sl->stage_bytes) {
        // grown in powers of two: pinning host memory is slow, so it happens
        // a few times per slot, not whenever a larger pack comes along
        host_free(ctx, sl->stage);
        sl->stage_bytes = 0;
        const size_t want = (size_t)pow2_at_least(std::max<size_t>(bytes, (size_t)8 << 20));
        if (host_alloc(ctx, &sl->stage, want) != RBSC_OK) {
            for (Job* j : js) finish_error(j, RBSC_ERR_OOM, rbsc_last_error(ctx));
            return;
        }
        sl->stage_bytes = want;
    }
    char* p = static_cast<char*>(sl->stage);
    uint64_t* off = reinterpret_cast<uint64_t*>(p);
    uint64_t* gn = reinterpret_cast<uint64_t*>(p + b_off);
    uint32_t* idx = reinterpret_cast<uint32_t*>(p + b_off + b_gn);
    uint32_t* init = reinterpret_cast<uint32_t*>(p + b_off + b_gn + b_idx);
    uint32_t* local = reinterpret_cast<uint32_t*>(p + b_off + b_gn + b_idx + b_init);
    uint32_t* blocks = reinterpret_cast<uint32_t*>(p + b_off + b_gn + b_idx + b_init + b_local);
    // node and arc bases, then the copies in parallel over contiguous job ranges
    std::vector<uint64_t> ab((size_t)G + 1, 0);
    gn[0] = 0;
    for (uint32_t i = 0; i < G; ++i) {
        gn[i + 1] = gn[i] + js[i]->g.n;
        ab[i + 1] = ab[i] + js[i]->g.m;
    }
    auto copy_jobs = [&](uint32_t i0, uint32_t i1) {
        for (uint32_t i = i0; i < i1; ++i) {
            const rbsc_csr& g = js[i]->g;
            const uint64_t nb = gn[i];
            if (g.offset_bytes == 8) shift_offsets<uint64_t>(g.offsets, g.n, ab[i], off + nb);
            else shift_offsets<uint32_t>(g.offsets, g.n, ab[i], off + nb);
            const uint32_t base = (uint32_t)nb;
            uint32_t* dst = idx + ab[i];
            for (uint64_t k = 0; k < g.m; ++k) dst[k] = g.indices[k] + base;
            if (any_init) {
                if (js[i]->init) std::memcpy(init + nb, js[i]->init, 4 * (size_t)g.n);
                else std::memset(init + nb, 0, 4 * (size_t)g.n);
            }
        }
    };
    const uint32_t T = (uint32_t)std::min<uint64_t>(8, std::max<uint64_t>(1, (M + N) >> 18));
    if (T <= 1 || G < 2) {
        copy_jobs(0, G);
    } else {
        // split the jobs into T ranges of about equal arcs + nodes
        std::vector<std::thread> ts;
        uint32_t i0 = 0;
        for (uint32_t t = 1; t <= T && i0 < G; ++t) {
            const uint64_t goal = (M + N) * t / T;
            uint32_t i1 = i0;
            while (i1 < G && (t == T || ab[i1] + gn[i1] < goal)) ++i1;
            if (i1 == i0) i1 = i0 + 1;
            ts.emplace_back(copy_jobs, i0, i1);
            i0 = i1;
        }
        if (i0 < G) copy_jobs(i0, G);
        for (auto& x : ts) x.join();
    }
    off[N] = M;
    rbsc_csr u{(uint32_t)N, M, off, 8, idx, nullptr};
    rbsc_batch_result r;
    std::memset(&r, 0, sizeof r);
    r.local = local;
    r.blocks = blocks;
    rbsc_stats st;
    const rbsc_status s = rbsc_batch_refine(ctx, &u, gn, G, any_init ? init : nullptr, &r, &st);
    if (s != RBSC_OK) {
        for (Job* j : js) finish_error(j, s, rbsc_last_error(ctx));
        return;
    }
    for (uint32_t i = 0; i < G; ++i) {
        Job* j = js[i];
        if (j->out) std::memcpy(j->out, local + gn[i], 4 * (size_t)j->g.n);
        j->res.status = RBSC_OK;
        j->res.blocks = blocks[i];
        j->res.rounds = st.rounds;
    }
}

void dispatch(rbsc_server* srv);

void slot_main(rbsc_server* srv, Slot* sl)
{
    if (!srv->o.dry_run) cudaSetDevice(srv->o.device);
    std::unique_lock<std::mutex> lk(srv->mu);
    for (;;) {
        sl->cv.wait(lk, [&] { return sl->busy || srv->stopping; });
        if (!sl->busy) break;  // stopping with nothing handed over
        std::vector<Job*> work;
        work.swap(sl->work);
        const uint64_t fp = sl->footprint;
        lk.unlock();
        uint64_t arcs = 0;
        for (Job* j : work) arcs += j->g.m;
        if (srv->o.dry_run) {
            std::this_thread::sleep_for(std::chrono::nanoseconds(20000 + (uint64_t)srv->o.dry_run_ns_per_arc * arcs));
            for (Job* j : work) j->res.status = RBSC_OK;
        } else if (work.size() == 1) {
            run_single(sl, work[0]);
        } else {
            run_pack(sl, work);
        }
        const auto t1 = Clock::now();
        lk.lock();
        for (Job* j : work) {
            j->res.packed = (uint32_t)work.size();
            j->res.slot = sl->index;
            j->res.footprint = fp;
            j->res.queue_ms = ms_between(j->t_submit, j->t_start);
            j->res.service_ms = ms_between(j->t_start, t1);
            j->res.latency_ms = ms_between(j->t_submit, t1);
            j->done = true;
            if (j->res.status == RBSC_OK) ++srv->st.completed;
            else ++srv->st.failed;
        }
        srv->st.reserved -= fp;
        srv->st.running -= work.size();
        --srv->busy;
        if (sl->large) --srv->busy_large;
        sl->busy = false;
        sl->large = false;
        dispatch(srv);
        srv->cv_done.notify_all();
    }
}

// Hands waiting jobs to idle executors (lock held).
void dispatch(rbsc_server* srv)
{
    if (srv->stopping) return;
    for (Slot* sl : srv->slots) {
        if (sl->busy) continue;
        if (srv->queue.empty()) return;
        size_t h = 0;  // queue position of the work's first job
        if (!srv->queue.front()->small && srv->slots.size() >= 2 && srv->busy_large + 1 >= srv->slots.size()) {
            // the last executor goes to the oldest small job, if one waits
            for (size_t i = 1; i < srv->queue.size(); ++i)
                if (srv->queue[i]->small) {
                    h = i;
                    break;
                }
        }
        Job* head = srv->queue[h];
        std::vector<size_t> take{h};
        std::vector<uint64_t> cn{head->g.n}, cm{head->g.m};  // running totals
        if (head->small && srv->o.pack_max_graphs > 1) {
            for (size_t i = h + 1; i < srv->queue.size() && take.size() < srv->o.pack_max_graphs; ++i) {
                const Job* j = srv->queue[i];
                if (!j->small) continue;
                if (cm.back() + j->g.m > srv->o.pack_arc_budget || cn.back() + j->g.n > srv->o.pack_arc_budget) continue;
                take.push_back(i);
                cn.push_back(cn.back() + j->g.n);
                cm.push_back(cm.back() + j->g.m);
            }
        }
        // the largest prefix of the pack that fits in the budget
        size_t k = take.size();
        uint64_t fp = 0;
        for (; k > 0; --k) {
            fp = rbsc_serve_footprint(cn[k - 1], cm[k - 1], head->g.weights != nullptr, (uint32_t)k);
            if (srv->st.reserved + fp <= srv->o.hbm_budget) break;
        }
        if (k == 0) return;  // the chosen job waits for memory (nothing else overtakes it)
        take.resize(k);
        std::vector<Job*> work;
        work.reserve(k);
        std::deque<Job*> rest;
        size_t t = 0;
        for (size_t i = 0; i < srv->queue.size(); ++i) {
            if (t < take.size() && take[t] == i) {
                work.push_back(srv->queue[i]);
                ++t;
            } else {
                rest.push_back(srv->queue[i]);
            }
        }
        srv->queue.swap(rest);
        const auto now = Clock::now();
        for (Job* j : work) j->t_start = now;
        srv->st.reserved += fp;
        srv->st.peak_reserved = std::max(srv->st.peak_reserved, srv->st.reserved);
        srv->st.queued -= work.size();
        srv->st.running += work.size();
        ++srv->st.batches;
        if (work.size() > 1) srv->st.packed_jobs += work.size();
        ++srv->busy;
        srv->st.peak_busy_slots = std::max(srv->st.peak_busy_slots, srv->busy);
        sl->large = !head->small;
        if (sl->large) ++srv->busy_large;
        sl->work.swap(work);
        sl->footprint = fp;
        sl->busy = true;
        sl->cv.notify_one();
    }
}

void destroy_slots(rbsc_server* srv)
{
    for (Slot* sl : srv->slots) {
        if (sl->th.joinable()) sl->th.join();
        if (sl->ctx) {
            host_free(sl->ctx, sl->stage);
            rbsc_ctx_destroy(sl->ctx);
        }
        delete sl;
    }
    srv->slots.clear();
}

}  // namespace

extern "C" rbsc_status rbsc_serve_create(const rbsc_serve_opts* opts, rbsc_server** out)
{
    if (!out) return serve_fail(RBSC_ERR_INVALID, "null output");
    *out = nullptr;
    rbsc_server* srv = new (std::nothrow) rbsc_server();
    if (!srv) return serve_fail(RBSC_ERR_OOM, "out of host memory");
    if (opts) srv->o = *opts;
    else rbsc_serve_opts_default(&srv->o);
    rbsc_serve_opts& o = srv->o;
    if (o.slots == 0) o.slots = 2;
    if (o.slots > 64) {
        delete srv;
        return serve_fail(RBSC_ERR_INVALID, "slots = %u (at most 64)", o.slots);
    }
    if (o.pack_max_arcs == 0) o.pack_max_arcs = 1ull << 18;
    if (o.pack_max_graphs == 0) o.pack_max_graphs = 4096;
    if (o.pack_arc_budget == 0) o.pack_arc_budget = 1ull << 22;
    o.pack_arc_budget = std::min<uint64_t>(o.pack_arc_budget, 1ull << 30);
    if (o.queue_cap == 0) o.queue_cap = 65536;
    o.opts.no_persist = 1;
    if (!o.dry_run) {
        cudaError_t e = cudaSetDevice(o.device);
        size_t free_b = 0, total_b = 0;
        if (e == cudaSuccess) e = cudaMemGetInfo(&free_b, &total_b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            delete srv;
            return serve_fail(RBSC_ERR_CUDA, "device %d: %s", o.device, cudaGetErrorString(e));
        }
        if (o.hbm_budget == 0) o.hbm_budget = free_b / 2;
    } else if (o.hbm_budget == 0) {
        o.hbm_budget = 64ull << 30;
    }
    srv->st.slots = o.slots;
    srv->st.hbm_budget = o.hbm_budget;
    for (uint32_t i = 0; i < o.slots; ++i) {
        Slot* sl = new (std::nothrow) Slot();
        if (!sl) {
            destroy_slots(srv);
            delete srv;
            return serve_fail(RBSC_ERR_OOM, "out of host memory");
        }
        sl->index = i;
        srv->slots.push_back(sl);
        if (!o.dry_run) {
            sl->ctx = rbsc_ctx_create(o.device, &o.opts);
            if (!sl->ctx) {
                const rbsc_status s = serve_fail(RBSC_ERR_CUDA, "slot %u: %s", i, rbsc_last_error(nullptr));
                destroy_slots(srv);
                delete srv;
                return s;
            }
            // unused cached blocks of a slot count against nobody's budget, but
            // giving them back costs a cudaFree, which waits for every slot's
            // work on the device: a slot keeps up to its share of the budget
            sl->ctx->dpool.cap = std::max<size_t>((size_t)64 << 20, o.hbm_budget / (uint64_t)o.slots);
        }
    }
    for (Slot* sl : srv->slots) sl->th = std::thread(slot_main, srv, sl);
    *out = srv;
    return RBSC_OK;
}

extern "C" void rbsc_serve_destroy(rbsc_server* srv)
{
    if (!srv) return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stopping = true;
        for (Job* j : srv->queue) {
            finish_error(j, RBSC_ERR_INVALID, "server shut down before the job started");
            j->done = true;
        }
        srv->queue.clear();
        for (Slot* sl : srv->slots) sl->cv.notify_one();
    }
    destroy_slots(srv);
    for (auto& kv : srv->jobs) delete kv.second;
    delete srv;
}

extern "C" const char* rbsc_serve_last_error(const rbsc_server*)
{
    return t_serve_error.c_str();
}

extern "C" rbsc_status rbsc_serve_submit(rbsc_server* srv, const rbsc_csr* g, const uint32_t* init_colors, uint32_t* out_labels,
                                         uint64_t* job_id)
{
    if (!srv || !g || !job_id) return serve_fail(RBSC_ERR_INVALID, "null argument");
    if (g->n >= 0x80000000u) return serve_fail(RBSC_ERR_TOO_LARGE, "N = %u: node ids must be < 2^31", g->n);
    if (g->offset_bytes != 4 && g->offset_bytes != 8) return serve_fail(RBSC_ERR_INVALID, "offset_bytes must be 4 or 8");
    if (g->offset_bytes == 4 && g->m >= (1ull << 32)) return serve_fail(RBSC_ERR_INVALID, "M >= 2^32 needs 8-byte offsets");
    if (!g->offsets) return serve_fail(RBSC_ERR_INVALID, "null offsets");
    if (g->m > 0 && !g->indices) return serve_fail(RBSC_ERR_INVALID, "null indices");
    const uint64_t fp = rbsc_serve_footprint(g->n, g->m, g->weights != nullptr, 1);
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stopping) return serve_fail(RBSC_ERR_INVALID, "server is shutting down");
    if (fp > srv->o.hbm_budget) {
        ++srv->st.rejected;
        return serve_fail(RBSC_ERR_TOO_LARGE, "job needs about %llu bytes of device memory, budget %llu",
                          (unsigned long long)fp, (unsigned long long)srv->o.hbm_budget);
    }
    if (srv->queue.size() >= srv->o.queue_cap) {
        ++srv->st.rejected;
        return serve_fail(RBSC_ERR_BUSY, "queue full (%u jobs waiting)", srv->o.queue_cap);
    }
    Job* j = new (std::nothrow) Job();
    if (!j) return serve_fail(RBSC_ERR_OOM, "out of host memory");
    j->id = srv->next_id++;
    j->g = *g;
    j->init = init_colors;
    j->out = out_labels;
    j->small = g->n >= 1 && g->n <= srv->o.pack_max_arcs && g->m <= srv->o.pack_max_arcs && g->weights == nullptr;
    j->t_submit = Clock::now();
    srv->jobs.emplace(j->id, j);
    srv->queue.push_back(j);
    ++srv->st.submitted;
    ++srv->st.queued;
    *job_id = j->id;
    dispatch(srv);
    return RBSC_OK;
}

namespace {

rbsc_status collect(rbsc_server* srv, uint64_t id, int64_t timeout_ms, rbsc_serve_result* r)
{
    std::unique_lock<std::mutex> lk(srv->mu);
    auto ready = [&] {
        auto it = srv->jobs.find(id);
        return it == srv->jobs.end() || it->second->done;
    };
    if (!ready() && timeout_ms != 0) {
        if (timeout_ms < 0) srv->cv_done.wait(lk, ready);
        else srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    }
    auto it = srv->jobs.find(id);
    if (it == srv->jobs.end()) return serve_fail(RBSC_ERR_INVALID, "unknown job %llu (or its result was collected)",
                                                 (unsigned long long)id);
    Job* j = it->second;
    if (!j->done) return RBSC_PENDING;
    if (r) *r = j->res;
    srv->jobs.erase(it);
    delete j;
    return RBSC_OK;
}

}  // namespace

extern "C" rbsc_status rbsc_serve_poll(rbsc_server* srv, uint64_t job_id, rbsc_serve_result* result)
{
    if (!srv) return serve_fail(RBSC_ERR_INVALID, "null server");
    return collect(srv, job_id, 0, result);
}

extern "C" rbsc_status rbsc_serve_wait(rbsc_server* srv, uint64_t job_id, int64_t timeout_ms, rbsc_serve_result* result)
{
    if (!srv) return serve_fail(RBSC_ERR_INVALID, "null server");
    return collect(srv, job_id, timeout_ms, result);
}

extern "C" rbsc_status rbsc_serve_stats_get(rbsc_server* srv, rbsc_serve_stats* stats)
{
    if (!srv || !stats) return serve_fail(RBSC_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    *stats = srv->st;
    return RBSC_OK;
}
