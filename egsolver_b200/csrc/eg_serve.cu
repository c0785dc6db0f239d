/*
 * eg_serve.cu -- serving mean-payoff threshold queries with continuous
 * batching.
 *
 * A query asks for the credits of every vertex of a registered game at K
 * thresholds p_k (weights w*d - p_k).  One worker thread runs the loop:
 *
 *   1. completions: micro-batches whose event fired hand their credits to
 *      their queries (device -> host) and release the queries' buffers;
 *   2. admission, in submission order: a query is admitted when fewer than
 *      max_inflight queries are admitted and the free device memory (from
 *      cudaMemGetInfo) minus hbm_reserve_bytes covers its credits and, if
 *      its game is not resident yet, the game's packed layout; idle resident
 *      games are evicted oldest-first when memory is short.  A game stays
 *      resident across all its queries until it is evicted or removed;
 *   3. launch: every admitted query not yet launched goes into one
 *      micro-batch, i.e. one launch of the unit kernel (eg_batch.cu: one CTA
 *      per game x threshold group, credits in shared memory), on the next of
 *      `streams` streams.  Earlier micro-batches keep running; as their CTAs
 *      run out of units and exit, the new launch's CTAs take the freed SMs,
 *      so the work of queries that arrived at different times overlaps on
 *      the device.  Each launch records its first CTA start and last CTA end
 *      on the device clock (eg_serve_trace).
 *
 * Routing: games above the batched layout's limit (2^19 vertices), and games
 * whose credits do not fit one CTA's shared memory while the queue is
 * shallow, are solved by a second thread one threshold at a time on the
 * persistent grid solver, capped at `large_ctas` CTAs so that micro-batches
 * keep SMs to run on.  With a deep queue such games run as units with their
 * credits in global memory, for throughput.
 *
 * Every result equals the solve of the same game and threshold alone: a
 * unit's work depends only on its own game and thresholds.
 */
#include "eg_batch.cuh"
#include "../../include/egsolver_b200_serve.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

using namespace eg;

namespace {

using clk = std::chrono::steady_clock;

double ms_since(clk::time_point a, clk::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); }

struct ServedGame {
    int64_t id;
    int n, n0;
    long long m;
    std::vector<int64_t> rp;
    std::vector<int32_t> succ, w;
    std::vector<uint8_t> own;
    bool has_owner = false;
    bool large = false;          /* above the batched layout's limit         */
    bool fits_smem = true;       /* one threshold's credits fit shared memory */
    bool resident = false;
    bool removed = false;
    HostPacked hp;               /* packed layout (host image)               */
    PackedDev pd;                /* its device copy while resident           */
    int active = 0; /* admitted queries still running */
    uint64_t last_use = 0;
    eg_game view() const
    {
        eg_game g;
        g.num_nodes = n;
        g.num_nodes0 = n0;
        g.num_edges = m;
        g.row_ptr = rp.data();
        g.succ = succ.data();
        g.weight = w.data();
        g.owner = has_owner ? own.data() : nullptr;
        return g;
    }
};

struct Query {
    int64_t id, game;
    int K, d;
    std::vector<int> p;
    int state = EG_QUERY_QUEUED;
    eg_status status = EG_OK;
    clk::time_point t_submit, t_done;
    long long rounds = 0;
    std::vector<int64_t> result; /* threshold-major */
    std::vector<long long> mg;   /* MG per threshold                         */
    /* device buffers while admitted: credits n*K (threshold-major),
     * thresholds, MG, per-unit rounds and status, global credit scratch */
    long long *dF = nullptr;
    int *dthr = nullptr;
    long long *dmg = nullptr;
    long long *drounds = nullptr;
    int *dstatus = nullptr;
    void *dscratch = nullptr;
    size_t dbytes = 0;
    std::vector<UnitDesc> units; /* planned at admission                     */
    std::vector<long long> cost;
    int smem = 16;
    cudaEvent_t ready = nullptr; /* buffers allocated and thresholds copied */
};

struct Launch {
    int stream;
    int64_t number = 0;
    int units = 0;
    cudaEvent_t ev = nullptr;
    std::vector<int64_t> qids;
    UnitDesc *dunits = nullptr;
    LaunchCtrl *dctrl = nullptr;
    void *dtails = nullptr;
    void *dscratch = nullptr;   /* hybrid tail regions */
};

}  // namespace

struct eg_server {
    eg_serve_opts o;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker, large_worker;
    bool stop = false;
    int64_t next_game = 1, next_query = 1;
    std::map<int64_t, std::unique_ptr<ServedGame>> games;
    std::map<int64_t, std::unique_ptr<Query>> queries;
    std::deque<int64_t> pending, large_pending;
    std::vector<int64_t> ready;
    std::vector<Launch> inflight;
    std::vector<cudaStream_t> streams;
    std::vector<UnitLauncher> launchers; /* side streams of each micro-batch stream */
    cudaStream_t upload_stream = nullptr;
    int next_stream = 0;
    int admitted_now = 0;
    uint64_t tick = 0;
    int sms = 148;
    int smem_budget = 0;
    std::vector<eg_serve_span> spans;   /* device-clock span of every micro-batch */
    unsigned long long clock0 = 0;      /* device clock of the first micro-batch  */
    /* statistics */
    int64_t submitted = 0, admitted = 0, completed = 0, failed = 0, uploads = 0, evictions = 0;
    int64_t micro_batches = 0, threshold_solves = 0;
    std::vector<double> latencies;
    clk::time_point t0, t_last_done;
    int64_t device_bytes = 0;
};

namespace {

/* credits | thresholds | MG | per-unit rounds | per-unit status | scratch */
size_t query_bytes(const ServedGame &g, int K, size_t scratch)
{
    return sizeof(long long) * (size_t)g.n * K + 4 * 64 * sizeof(long long) + 1024 + scratch;
}

void free_query_device(Query &q, cudaStream_t st)
{
    if (q.dF) cudaFreeAsync(q.dF, st);
    if (q.ready) cudaEventDestroy(q.ready);
    q.ready = nullptr;
    q.dF = nullptr;
    q.dthr = nullptr;
    q.dmg = nullptr;
    q.drounds = nullptr;
    q.dstatus = nullptr;
    q.dscratch = nullptr;
}

void drop_resident(eg_server *s, ServedGame &g)
{
    s->device_bytes -= (int64_t)g.pd.bytes;
    if (g.pd.block) cudaFreeAsync(g.pd.block, s->upload_stream);
    cudaStreamSynchronize(s->upload_stream);
    g.pd = PackedDev();
    g.resident = false;
}

/* Frees resident games nobody uses, oldest first, until `need` bytes fit. */
bool make_room(eg_server *s, size_t need)
{
    for (;;) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        const size_t reserve = (size_t)s->o.hbm_reserve_bytes;
        if (free_b > reserve && free_b - reserve >= need) return true;
        ServedGame *victim = nullptr;
        for (auto &kv : s->games) {
            ServedGame &g = *kv.second;
            if (g.resident && g.active == 0 && (!victim || g.last_use < victim->last_use)) victim = &g;
        }
        if (!victim) return false;
        drop_resident(s, *victim);
        s->evictions++;
    }
}

void finish_query(eg_server *s, Query &q, eg_status st, clk::time_point now)
{
    q.status = st;
    q.state = st == EG_OK ? EG_QUERY_DONE : EG_QUERY_FAILED;
    q.t_done = now;
    s->t_last_done = now;
    if (st == EG_OK) {
        s->completed++;
        s->threshold_solves += q.K;
    } else {
        s->failed++;
    }
    s->latencies.push_back(ms_since(q.t_submit, now));
}

/* Completion of finished micro-batches (lock held). */
bool reap(eg_server *s)
{
    bool any = false;
    for (size_t i = 0; i < s->inflight.size();) {
        Launch &l = s->inflight[i];
        const cudaError_t e = cudaEventQuery(l.ev);
        if (e == cudaErrorNotReady) {
            i++;
            continue;
        }
        any = true;
        const clk::time_point now = clk::now();
        UnitCtrl c;
        LaunchCtrl cv;
        memset(&c, 0, sizeof c);
        if (e == cudaSuccess && cudaMemcpy(&cv, l.dctrl, sizeof cv, cudaMemcpyDeviceToHost) == cudaSuccess) {
            sum_ctrl(cv, &c);
            if (!s->clock0) s->clock0 = c.t_begin;
            eg_serve_span sp;
            memset(&sp, 0, sizeof sp);
            sp.batch = l.number;
            sp.queries = (int32_t)l.qids.size();
            sp.units = l.units;
            sp.begin_ms = ((double)c.t_begin - (double)s->clock0) * 1e-6;
            sp.end_ms = ((double)c.t_end - (double)s->clock0) * 1e-6;
            s->spans.push_back(sp);
        }
        for (int64_t qid : l.qids) {
            Query &q = *s->queries[qid];
            ServedGame &g = *s->games[q.game];
            eg_status st = e == cudaSuccess ? EG_OK : EG_ERR_CUDA;
            if (st == EG_OK) {
                const size_t nu = q.units.size();
                std::vector<long long> rr(nu);
                std::vector<int> ss(nu);
                q.result.assign((size_t)g.n * q.K, 0);
                cudaError_t cp = cudaMemcpy(q.result.data(), q.dF, sizeof(long long) * q.result.size(),
                                            cudaMemcpyDeviceToHost);
                if (cp == cudaSuccess) cp = cudaMemcpy(ss.data(), q.dstatus, sizeof(int) * nu, cudaMemcpyDeviceToHost);
                if (cp == cudaSuccess) cp = cudaMemcpy(rr.data(), q.drounds, sizeof(long long) * nu, cudaMemcpyDeviceToHost);
                if (cp != cudaSuccess) {
                    st = EG_ERR_CUDA;
                } else {
                    q.rounds = 0;
                    for (size_t u = 0; u < nu; u++) {
                        q.rounds = std::max(q.rounds, rr[u]);
                        if (st == EG_OK && ss[u] != EG_OK) st = (eg_status)ss[u];
                    }
                }
            }
            s->device_bytes -= (int64_t)q.dbytes;
            free_query_device(q, s->streams[l.stream]);
            g.active--;
            s->admitted_now--;
            finish_query(s, q, st, now);
        }
        cudaEventDestroy(l.ev);
        cudaFreeAsync(l.dunits, s->streams[l.stream]);
        cudaFreeAsync(l.dctrl, s->streams[l.stream]);
        cudaFreeAsync(l.dtails, s->streams[l.stream]);
        if (l.dscratch) cudaFreeAsync(l.dscratch, s->streams[l.stream]);
        s->inflight.erase(s->inflight.begin() + (long)i);
    }
    if (any) s->cv_done.notify_all();
    return any;
}

/* Admission in submission order (lock held; releases it around uploads). */
bool admit(eg_server *s, std::unique_lock<std::mutex> &lk)
{
    bool any = false;
    while (!s->pending.empty() && s->admitted_now < s->o.max_inflight) {
        const int64_t qid = s->pending.front();
        Query &q = *s->queries[qid];
        ServedGame &g = *s->games[q.game];
        /* routing: the grid solver for games the batched layout cannot hold,
         * and for games whose credits miss shared memory while the queue is
         * shallow (lower latency); units otherwise */
        if (g.large || (!g.fits_smem && s->pending.size() + s->ready.size() <= 2)) {
            s->pending.pop_front();
            s->large_pending.push_back(qid);
            s->cv_work.notify_all();
            any = true;
            continue;
        }
        /* plan the query's units (device pointers are filled in below) */
        q.mg.assign((size_t)q.K, 0);
        for (int k = 0; k < q.K; k++) q.mg[(size_t)k] = threshold_mg(g.hp, q.p[(size_t)k], q.d);
        std::vector<UnitDesc> units;
        std::vector<size_t> gneed;
        std::vector<long long> cost;
        int smem = 16;
        eg_status ps = make_units(g.hp, PackedDev(), q.K, q.d, q.p.data(), q.mg.data(), nullptr, nullptr, nullptr,
                                  s->smem_budget, 8, &units, &gneed, &cost, &smem);
        if (ps != EG_OK) {
            s->pending.pop_front();
            finish_query(s, q, ps, clk::now());
            s->cv_done.notify_all();
            any = true;
            continue;
        }
        size_t scratch = 0;
        for (size_t x : gneed) scratch += x;
        const size_t qbytes = query_bytes(g, q.K, scratch) + units.size() * 16;
        size_t need = qbytes;
        if (!g.resident) need += packed_dev_bytes(g.hp);
        if (!make_room(s, need)) {
            if (s->admitted_now == 0 && s->inflight.empty()) { /* can never fit */
                s->pending.pop_front();
                finish_query(s, q, EG_ERR_OOM, clk::now());
                s->cv_done.notify_all();
                any = true;
                continue;
            }
            break; /* wait for memory to come back */
        }
        if (!g.resident) {
            void *blk = nullptr;
            const size_t pb = packed_dev_bytes(g.hp);
            eg_status st = EG_OK;
            lk.unlock();
            if (cudaMallocAsync(&blk, pb, s->upload_stream) != cudaSuccess) {
                cudaGetLastError();
                st = eg_set_error(EG_ERR_OOM, "device allocation of a game failed");
            }
            PackedDev pd;
            if (st == EG_OK) st = packed_upload(g.hp, blk, s->upload_stream, &pd);
            if (st == EG_OK && cudaStreamSynchronize(s->upload_stream) != cudaSuccess)
                st = eg_set_error(EG_ERR_CUDA, "game upload failed");
            lk.lock();
            if (st != EG_OK) {
                if (blk) cudaFreeAsync(blk, s->upload_stream);
                s->pending.pop_front();
                finish_query(s, q, st, clk::now());
                s->cv_done.notify_all();
                any = true;
                continue;
            }
            g.pd = pd;
            g.resident = true;
            s->uploads++;
            s->device_bytes += (int64_t)pd.bytes;
        }
        /* one device block per query: credits | thresholds | MG | rounds | status | scratch */
        const size_t nu = units.size();
        const size_t fbytes = sizeof(long long) * (size_t)g.n * q.K;
        const size_t o_thr = (fbytes + 255) & ~(size_t)255;
        const size_t o_mg = o_thr + (((size_t)q.K * sizeof(int) + 255) & ~(size_t)255);
        const size_t o_rounds = o_mg + (((size_t)q.K * sizeof(long long) + 255) & ~(size_t)255);
        const size_t o_status = o_rounds + ((nu * sizeof(long long) + 255) & ~(size_t)255);
        const size_t o_scr = o_status + ((nu * sizeof(int) + 255) & ~(size_t)255);
        const size_t total = o_scr + scratch;
        char *blk = nullptr;
        if (cudaMallocAsync((void **)&blk, total, s->upload_stream) != cudaSuccess) {
            cudaGetLastError();
            break;
        }
        q.dF = (long long *)blk;
        q.dthr = (int *)(blk + o_thr);
        q.dmg = (long long *)(blk + o_mg);
        q.drounds = (long long *)(blk + o_rounds);
        q.dstatus = (int *)(blk + o_status);
        q.dscratch = scratch ? (void *)(blk + o_scr) : nullptr;
        q.dbytes = total;
        size_t goff = 0;
        for (size_t u = 0; u < nu; u++) {
            UnitDesc &d = units[u];
            d.E = g.pd.E;
            d.slice_off = g.pd.slice_off;
            d.orig = g.pd.orig;
            d.p = q.dthr;
            d.mg = q.dmg;
            d.F = q.dF;
            d.rounds = q.drounds + u;
            d.status = q.dstatus + u;
            if (gneed[u]) {
                d.gscratch = (char *)q.dscratch + goff;
                goff += gneed[u];
            }
        }
        q.units.swap(units);
        q.cost.swap(cost);
        q.smem = smem;
        cudaMemcpyAsync(q.dthr, q.p.data(), sizeof(int) * (size_t)q.K, cudaMemcpyHostToDevice, s->upload_stream);
        cudaMemcpyAsync(q.dmg, q.mg.data(), sizeof(long long) * (size_t)q.K, cudaMemcpyHostToDevice, s->upload_stream);
        cudaEventCreateWithFlags(&q.ready, cudaEventDisableTiming);
        cudaEventRecord(q.ready, s->upload_stream);
        cudaStreamSynchronize(s->upload_stream); /* q.p / q.mg are host memory that may go away */
        s->device_bytes += (int64_t)q.dbytes;
        g.active++;
        g.last_use = ++s->tick;
        q.state = EG_QUERY_RUNNING;
        s->admitted++;
        s->admitted_now++;
        s->pending.pop_front();
        s->ready.push_back(qid);
        any = true;
    }
    return any;
}

/* One micro-batch of every admitted, not yet launched query (lock held). */
bool launch_ready(eg_server *s)
{
    if (s->ready.empty() || (int)s->inflight.size() >= s->o.streams) return false;
    std::vector<UnitDesc> all;
    std::vector<long long> cost;
    Launch l;
    for (int64_t qid : s->ready) {
        Query &q = *s->queries[qid];
        all.insert(all.end(), q.units.begin(), q.units.end());
        cost.insert(cost.end(), q.cost.begin(), q.cost.end());
        l.qids.push_back(qid);
    }
    UnitSet S;
    group_units(all, cost, std::vector<size_t>(all.size(), 0), &S, nullptr);
    l.stream = s->next_stream;
    l.number = s->micro_batches;
    l.units = (int)S.units.size();
    s->next_stream = (s->next_stream + 1) % s->o.streams;
    cudaStream_t st = s->streams[l.stream];
    for (int64_t qid : l.qids) cudaStreamWaitEvent(st, s->queries[qid]->ready, 0);
    cudaError_t e = cudaMallocAsync((void **)&l.dunits, sizeof(UnitDesc) * S.units.size(), st);
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&l.dctrl, sizeof(LaunchCtrl), st);
    if (e == cudaSuccess) e = cudaMallocAsync(&l.dtails, tail_bytes(S), st);
    const size_t tsb = tail_scratch_bytes(S, s->sms);
    if (e == cudaSuccess && tsb) e = cudaMallocAsync(&l.dscratch, tsb, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(l.dunits, S.units.data(), sizeof(UnitDesc) * S.units.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&l.ev, cudaEventDisableTiming);
    eg_status ls = EG_OK;
    TailList *tl = nullptr;
    if (e == cudaSuccess) ls = tail_upload(S, l.dtails, st, &tl);
    if (e == cudaSuccess && ls == EG_OK) {
        int grid = 0;
        ls = launch_unit_set(s->launchers[(size_t)l.stream], st, S, l.dunits, tl, l.dscratch, l.dctrl, s->o.block,
                             s->sms, s->o.max_rounds, 0, &grid);
        if (ls == EG_OK) e = cudaEventRecord(l.ev, st);
        /* the tail list's host image is copied from pageable memory: wait for
         * the copy before S goes out of scope */
        if (ls == EG_OK && e == cudaSuccess) e = cudaStreamSynchronize(s->upload_stream);
    }
    if (e != cudaSuccess || ls != EG_OK) {
        cudaGetLastError();
        const clk::time_point now = clk::now();
        for (int64_t qid : l.qids) {
            Query &q = *s->queries[qid];
            s->device_bytes -= (int64_t)q.dbytes;
            free_query_device(q, st);
            s->games[q.game]->active--;
            s->admitted_now--;
            finish_query(s, q, ls != EG_OK ? ls : EG_ERR_CUDA, now);
        }
        if (l.ev) cudaEventDestroy(l.ev);
        if (l.dunits) cudaFreeAsync(l.dunits, st);
        if (l.dctrl) cudaFreeAsync(l.dctrl, st);
        if (l.dtails) cudaFreeAsync(l.dtails, st);
        if (l.dscratch) cudaFreeAsync(l.dscratch, st);
        s->ready.clear();
        s->cv_done.notify_all();
        return true;
    }
    s->ready.clear();
    s->inflight.push_back(l);
    s->micro_batches++;
    return true;
}

void worker_main(eg_server *s)
{
    cudaSetDevice(s->o.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        bool progress = reap(s);
        progress |= admit(s, lk);
        progress |= launch_ready(s);
        if (s->stop && s->pending.empty() && s->ready.empty() && s->inflight.empty()) break;
        if (!progress) s->cv_work.wait_for(lk, std::chrono::microseconds(200));
    }
}

/* Large games: one threshold at a time on the capped persistent grid. */
void large_main(eg_server *s)
{
    cudaSetDevice(s->o.device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        if (s->large_pending.empty()) {
            if (s->stop) break;
            s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
            continue;
        }
        const int64_t qid = s->large_pending.front();
        s->large_pending.pop_front();
        Query &q = *s->queries[qid];
        ServedGame &g = *s->games[q.game];
        g.active++;
        q.state = EG_QUERY_RUNNING;
        s->admitted++;
        eg_game base = g.view();
        const int K = q.K, d = q.d;
        const std::vector<int> p = q.p;
        lk.unlock();
        std::vector<int64_t> result((size_t)g.n * K);
        std::vector<int32_t> wt((size_t)g.m);
        eg_status st = EG_OK;
        long long rounds = 0;
        for (int k = 0; k < K && st == EG_OK; k++) {
            for (long long j = 0; j < g.m; j++) {
                const long long x = (long long)base.weight[j] * d - p[(size_t)k];
                if (x < INT32_MIN || x > INT32_MAX) {
                    st = eg_set_error(EG_ERR_OVERFLOW, "shifted weight out of int32 range");
                    break;
                }
                wt[(size_t)j] = (int32_t)x;
            }
            if (st != EG_OK) break;
            eg_game tg = base;
            tg.weight = wt.data();
            eg_opts o;
            eg_opts_default(&o);
            o.device = s->o.device;
            o.credit_bits = 64;
            o.max_rounds = s->o.max_rounds;
            o.grid_ctas = s->o.large_ctas;
            eg_dgame *dg = nullptr;
            st = eg_dgame_upload(&tg, &o, &dg);
            eg_stats ss;
            if (st == EG_OK) st = eg_dgame_solve(dg, &o, &ss);
            if (st == EG_OK) st = eg_dgame_credits_i64(dg, result.data() + (size_t)k * g.n);
            if (st == EG_OK) rounds = std::max(rounds, (long long)ss.rounds);
            eg_dgame_free(dg);
        }
        lk.lock();
        q.result.swap(result);
        q.rounds = rounds;
        g.active--;
        finish_query(s, q, st, clk::now());
        s->cv_done.notify_all();
    }
}

}  // namespace

extern "C" eg_status eg_serve_create(const eg_serve_opts *opts, eg_server **out)
{
    if (!out) return eg_set_error(EG_ERR_INVALID, "out is NULL");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return eg_set_error(EG_ERR_NO_DEVICE, "no CUDA device available");
    }
    eg_server *s = new eg_server();
    memset(&s->o, 0, sizeof s->o);
    if (opts) s->o = *opts;
    if (s->o.device < 0 || s->o.device >= count) {
        delete s;
        return eg_set_error(EG_ERR_INVALID, "device %d not available", opts ? opts->device : 0);
    }
    if (s->o.max_inflight <= 0) s->o.max_inflight = 1024;
    if (s->o.streams <= 0) s->o.streams = 4;
    if (s->o.block <= 0) s->o.block = 1024;
    if (s->o.hbm_reserve_bytes <= 0) s->o.hbm_reserve_bytes = 1ll << 30;
    if (s->o.large_ctas <= 0) s->o.large_ctas = 148;
    if (s->o.max_rounds == 0) s->o.max_rounds = -1;
    cudaSetDevice(s->o.device);
    cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->o.device);
    {
        eg_status ks = unit_kernel_setup(s->o.device);
        if (ks != EG_OK) {
            delete s;
            return ks;
        }
        s->smem_budget = unit_smem_budget(s->o.device);
    }
    for (int i = 0; i < s->o.streams; i++) {
        cudaStream_t st;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
            for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
            delete s;
            return eg_set_error(EG_ERR_CUDA, "stream creation failed");
        }
        s->streams.push_back(st);
        s->launchers.emplace_back();
        if (s->launchers.back().init() != EG_OK) {
            for (UnitLauncher &L : s->launchers) L.destroy();
            for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
            delete s;
            return eg_set_error(EG_ERR_CUDA, "stream creation failed");
        }
    }
    if (cudaStreamCreateWithFlags(&s->upload_stream, cudaStreamNonBlocking) != cudaSuccess) {
        for (UnitLauncher &L : s->launchers) L.destroy();
        for (cudaStream_t x : s->streams) cudaStreamDestroy(x);
        delete s;
        return eg_set_error(EG_ERR_CUDA, "stream creation failed");
    }
    s->t0 = s->t_last_done = clk::now();
    s->worker = std::thread(worker_main, s);
    s->large_worker = std::thread(large_main, s);
    *out = s;
    return EG_OK;
}

extern "C" eg_status eg_serve_add_game(eg_server *s, const eg_game *game, int64_t *game_id)
{
    if (!s || !game || !game_id) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    eg_status v = eg_validate(game);
    if (v != EG_OK) return v;
    auto g = std::make_unique<ServedGame>();
    g->n = game->num_nodes;
    g->n0 = game->num_nodes0;
    g->m = game->num_edges;
    g->rp.assign(game->row_ptr, game->row_ptr + game->num_nodes + 1);
    g->succ.assign(game->succ, game->succ + game->num_edges);
    g->w.assign(game->weight, game->weight + game->num_edges);
    if (game->owner) {
        g->own.assign(game->owner, game->owner + game->num_nodes);
        g->has_owner = true;
    }
    g->large = game->num_nodes > kBatchMaxGameNodes;
    if (!g->large) {
        /* the packed layout the unit kernel reads (host image, uploaded on admission) */
        eg_status ps = pack_game(*game, &g->hp);
        if (ps != EG_OK) return ps;
        g->fits_smem = (long long)g->hp.rows() * 4 <= (long long)s->smem_budget;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    g->id = s->next_game++;
    *game_id = g->id;
    s->games[g->id] = std::move(g);
    return EG_OK;
}

extern "C" eg_status eg_serve_remove_game(eg_server *s, int64_t game_id)
{
    if (!s) return eg_set_error(EG_ERR_INVALID, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->games.find(game_id);
    if (it == s->games.end()) return eg_set_error(EG_ERR_NOT_FOUND, "no game %lld", (long long)game_id);
    for (auto &kv : s->queries)
        if (kv.second->game == game_id && kv.second->state <= EG_QUERY_RUNNING)
            return eg_set_error(EG_ERR_BUSY, "game %lld still has queries in flight", (long long)game_id);
    if (it->second->resident) drop_resident(s, *it->second);
    s->games.erase(it);
    return EG_OK;
}

extern "C" eg_status eg_serve_submit(eg_server *s, int64_t game_id, const int32_t *p, int32_t K, int32_t d,
                                     int64_t *query_id)
{
    if (!s || !p || !query_id) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    if (K < 1 || K > EG_BATCH_MAX_K) return eg_set_error(EG_ERR_INVALID, "K must be in [1, %d]", EG_BATCH_MAX_K);
    if (d < 1) return eg_set_error(EG_ERR_INVALID, "scale d must be >= 1");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return eg_set_error(EG_ERR_BUSY, "server is shutting down");
    if (!s->games.count(game_id)) return eg_set_error(EG_ERR_NOT_FOUND, "no game %lld", (long long)game_id);
    auto q = std::make_unique<Query>();
    q->id = s->next_query++;
    q->game = game_id;
    q->K = K;
    q->d = d;
    q->p.assign(p, p + K);
    q->t_submit = clk::now();
    *query_id = q->id;
    s->pending.push_back(q->id);
    s->queries[q->id] = std::move(q);
    s->submitted++;
    s->cv_work.notify_all();
    return EG_OK;
}

extern "C" eg_status eg_serve_poll(eg_server *s, int64_t query_id, int32_t *state, double *latency_ms)
{
    if (!s) return eg_set_error(EG_ERR_INVALID, "server is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->queries.find(query_id);
    if (it == s->queries.end()) return eg_set_error(EG_ERR_NOT_FOUND, "no query %lld", (long long)query_id);
    const Query &q = *it->second;
    if (state) *state = q.state;
    if (latency_ms) *latency_ms = q.state >= EG_QUERY_DONE ? ms_since(q.t_submit, q.t_done) : ms_since(q.t_submit, clk::now());
    return EG_OK;
}

extern "C" eg_status eg_serve_wait(eg_server *s, int64_t query_id, double timeout_ms)
{
    if (!s) return eg_set_error(EG_ERR_INVALID, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    const clk::time_point until = clk::now() + std::chrono::microseconds((long long)(timeout_ms * 1000));
    for (;;) {
        auto it = s->queries.find(query_id);
        if (it == s->queries.end()) return eg_set_error(EG_ERR_NOT_FOUND, "no query %lld", (long long)query_id);
        if (it->second->state >= EG_QUERY_DONE) return EG_OK;
        if (timeout_ms >= 0 && clk::now() >= until) return eg_set_error(EG_ERR_TIMEOUT, "query %lld not finished", (long long)query_id);
        s->cv_done.wait_for(lk, std::chrono::milliseconds(5));
    }
}

extern "C" eg_status eg_serve_result(eg_server *s, int64_t query_id, int64_t *credits, int64_t *rounds)
{
    if (!s || !credits) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->queries.find(query_id);
    if (it == s->queries.end()) return eg_set_error(EG_ERR_NOT_FOUND, "no query %lld", (long long)query_id);
    Query &q = *it->second;
    if (q.state == EG_QUERY_FAILED) {
        const eg_status st = q.status;
        s->queries.erase(it);
        return eg_set_error(st, "query %lld failed with status %d", (long long)query_id, (int)st);
    }
    if (q.state != EG_QUERY_DONE) return eg_set_error(EG_ERR_BUSY, "query %lld not finished", (long long)query_id);
    memcpy(credits, q.result.data(), sizeof(int64_t) * q.result.size());
    if (rounds) *rounds = q.rounds;
    s->queries.erase(it);
    return EG_OK;
}

extern "C" eg_status eg_serve_stats_get(eg_server *s, eg_serve_stats *out)
{
    if (!s || !out) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(out, 0, sizeof *out);
    out->submitted = s->submitted;
    out->admitted = s->admitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->games_registered = (int64_t)s->games.size();
    for (auto &kv : s->games) out->games_resident += kv.second->resident;
    out->game_uploads = s->uploads;
    out->evictions = s->evictions;
    out->micro_batches = s->micro_batches;
    out->threshold_solves = s->threshold_solves;
    std::vector<double> lat = s->latencies;
    if (!lat.empty()) {
        std::sort(lat.begin(), lat.end());
        auto pct = [&](double q) { return lat[std::min(lat.size() - 1, (size_t)(q * (double)(lat.size() - 1) + 0.5))]; };
        out->latency_p50_ms = pct(0.50);
        out->latency_p99_ms = pct(0.99);
        out->latency_max_ms = lat.back();
        double sum = 0;
        for (double x : lat) sum += x;
        out->latency_mean_ms = sum / (double)lat.size();
    }
    out->elapsed_s = std::chrono::duration<double>(s->t_last_done - s->t0).count();
    if (out->elapsed_s > 0) {
        out->queries_per_s = (double)s->completed / out->elapsed_s;
        out->solves_per_s = (double)s->threshold_solves / out->elapsed_s;
    }
    out->device_bytes = s->device_bytes;
    return EG_OK;
}

extern "C" eg_status eg_serve_trace(eg_server *s, eg_serve_span *spans, int32_t cap, int32_t *count)
{
    if (!s || !count || (cap > 0 && !spans)) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    const int32_t n = (int32_t)s->spans.size();
    for (int32_t i = 0; i < n && i < cap; i++) spans[i] = s->spans[(size_t)i];
    *count = n;
    return EG_OK;
}

extern "C" eg_status eg_serve_destroy(eg_server *s)
{
    if (!s) return EG_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    s->worker.join();
    s->large_worker.join();
    cudaSetDevice(s->o.device);
    for (auto &kv : s->queries) free_query_device(*kv.second, s->upload_stream);
    for (auto &kv : s->games)
        if (kv.second->resident && kv.second->pd.block) cudaFreeAsync(kv.second->pd.block, s->upload_stream);
    cudaStreamSynchronize(s->upload_stream);
    for (UnitLauncher &L : s->launchers) L.destroy();
    for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
    cudaStreamDestroy(s->upload_stream);
    delete s;
    return EG_OK;
}
