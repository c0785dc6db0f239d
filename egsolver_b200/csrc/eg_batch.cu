/*
 * eg_batch.cu -- batched solving of many games at K mean-payoff thresholds
 * in one persistent launch.
 *
 * Layout: the games are packed into one device-resident multi-CSR (global
 * vertex ids, no edge crosses games), with one CSC built by the same stable
 * counting sort as the single-game path.  Credits are stored vertex-major
 * with the K thresholds contiguous, f[(v * K) + k], so the K lanes that
 * lift vertex v for the K thresholds read one successor's K credits as a
 * single contiguous row.
 *
 * Kernel: every CTA takes a game from a device queue (largest games first),
 * computes MG_k = sum_v max(0, p_k - d * min_w(v)), then runs dense rounds
 * of that game alone with CTA barriers: every vertex lifted at every
 * threshold per round, eight independent credit gathers in flight per lane.
 * Mean-payoff threshold games take thousands of rounds in which most
 * vertices rise, so a frontier would hold nearly every vertex anyway.  The
 * lift of vertex v for threshold k is the reference's (reference
 * src/dev_EG_alg.cu:84-109) on the weights w * d - p_k.  No wait in this
 * kernel spins: rounds end at __syncthreads and games come from an atomic
 * counter.
 */
#include "eg_batch.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

using namespace eg;

#define EG_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t _e = (call);                                                                       \
        if (_e != cudaSuccess)                                                                         \
            return eg_set_error(_e == cudaErrorMemoryAllocation ? EG_ERR_OOM : EG_ERR_CUDA,             \
                                "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

#define EG_TRY(call)                                                                                   \
    do {                                                                                               \
        eg_status _s = (call);                                                                         \
        if (_s != EG_OK) return _s;                                                                    \
    } while (0)

namespace {

/* OMINUS on 64-bit credits for the weight b = w * d - p (reference
 * src/common.h:270-272); the difference is formed without overflow and only
 * used when a is finite. */
__device__ __forceinline__ long long ominus64(long long a, long long b, long long mg)
{
    const long long t = (long long)INT64_MAX;
    const long long x = (long long)((unsigned long long)a - (unsigned long long)b);
    return (a < t && x <= mg) ? (x > 0 ? x : 0) : t;
}

/* Edges of a vertex taken together per step of the lift loop: independent
 * credit gathers in flight per lane. */
constexpr int kBatchUnroll = 8;

/* KP lanes per vertex (KP >= K, a power of two); lane k serves threshold k.
 * Dense rounds: each round lifts every vertex of the game at every
 * threshold in place (no frontier), and the game is solved after a round
 * without a raise.  Every lift reads credits that are the round's start
 * values or values raised since, all below the least fixed point, so this is
 * a fair chaotic iteration of the same operator and the credits equal the
 * worklist solver's. */
template <int KP>
__global__ void __launch_bounds__(1024) k_batch_solve(const __grid_constant__ BatchParams p)
{
    __shared__ int s_game;
    __shared__ long long s_mg[KP];
    __shared__ int s_p[KP];
    const int tid = threadIdx.x, lane = tid & 31;
    const int gl = lane % KP;
    const int group = tid / KP, ngroups = blockDim.x / KP;
    const long long TOP = (long long)INT64_MAX;
    unsigned long long lifts = 0, edges = 0, ntop = 0;
    if (blockIdx.x == 0 && tid == 0) p.ctrl->t_start = globaltimer_ns();
    for (;;) {
        if (tid == 0) s_game = atomicAdd(&p.ctrl->next_game, 1);
        __syncthreads();
        const int gi = s_game;
        if (gi >= p.num_games) break;
        const GameDesc gd = p.games[p.order ? p.order[gi] : gi];
        const long long base = gd.base;
        const int n = gd.n;
        const int K = gd.K;
        const long long d = gd.d;
        const int *P = gd.P;
        const int2 *E = gd.E;
        const unsigned char *owner = gd.owner;
        long long *F = gd.F - base * K; /* indexed by id * K + k with ids base-relative */
        if (tid < KP) {
            s_p[tid] = gd.thr[tid < K ? tid : 0];
            s_mg[tid] = 0;
        }
        for (long long i = tid; i < (long long)n * K; i += blockDim.x) gd.F[i] = 0;
        __syncthreads();
        /* MG per threshold: sum_v max(0, p_k - d * min_w(v)) */
        for (int k = 0; k < K; k++) {
            long long s = 0;
            for (int v = tid; v < n; v += blockDim.x) {
                const long long x = (long long)s_p[k] - (long long)gd.minw[v] * d;
                s += x > 0 ? x : 0;
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
            if (lane == 0 && s) atomicAdd((unsigned long long *)&s_mg[k], (unsigned long long)s);
        }
        __syncthreads();
        const long long pk = s_p[gl];
        const long long mgk = s_mg[gl];
        const bool valid = gl < K;
        long long r = 0;
        int st = EG_OK;
        for (;;) {
            int raised = 0;
            /* the next vertex's row and owner load while this one is lifted */
            int eb = 0, ee = 0, own = 0;
            if (group < n) {
                eb = P[group];
                ee = P[group + 1];
                own = owner[group];
            }
            for (int v = group; v < n; v += ngroups) {
                const long long gv = base + v;
                const int vn = v + ngroups;
                int ebn = 0, een = 0, ownn = 0;
                if (vn < n) {
                    ebn = P[vn];
                    een = P[vn + 1];
                    ownn = owner[vn];
                }
                /* only this lane writes F[v][k] in a round: read it early */
                const long long old = valid ? F[gv * K + gl] : 0;
                long long acc = own ? 0 : TOP;
                for (int e = eb; e < ee; e += kBatchUnroll) {
                    int2 q[kBatchUnroll];
                    long long f[kBatchUnroll];
#pragma unroll
                    for (int j = 0; j < kBatchUnroll; j++)
                        if (e + j < ee) q[j] = __ldg(E + e + j);
#pragma unroll
                    for (int j = 0; j < kBatchUnroll; j++)
                        f[j] = (valid && e + j < ee) ? F[(long long)q[j].x * K + gl] : 0;
#pragma unroll
                    for (int j = 0; j < kBatchUnroll; j++) {
                        if (valid && e + j < ee) {
                            const long long val = ominus64(f[j], (long long)q[j].y * d - pk, mgk);
                            acc = own ? (val > acc ? val : acc) : (val < acc ? val : acc);
                        }
                    }
                }
                if (valid && old < acc) {
                    F[gv * K + gl] = acc;
                    raised = 1;
                }
                if (gl == 0) {
                    lifts++;
                    edges += (unsigned long long)(ee - eb) * (unsigned long long)K;
                }
                eb = ebn;
                ee = een;
                own = ownn;
            }
            r++;
            if (!__syncthreads_or(raised)) break;
            if (p.max_rounds >= 0 && r >= p.max_rounds) {
                st = EG_ERR_LOOPCAP;
                break;
            }
            const int late = __syncthreads_or(tid == 0 && p.timeout_ns &&
                                              globaltimer_ns() - p.ctrl->t_start > p.timeout_ns);
            if (late) {
                st = EG_ERR_TIMEOUT;
                break;
            }
        }
        /* TOP count of this game (all thresholds) */
        for (long long i = tid; i < (long long)n * K; i += blockDim.x) ntop += (gd.F[i] == TOP);
        if (tid == 0) {
            *gd.rounds = r;
            *gd.status = st;
        }
        __syncthreads();
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        lifts += __shfl_xor_sync(0xffffffffu, lifts, off);
        edges += __shfl_xor_sync(0xffffffffu, edges, off);
        ntop += __shfl_xor_sync(0xffffffffu, ntop, off);
    }
    if (lane == 0) {
        atomicAdd(&p.ctrl->lifts, lifts);
        atomicAdd(&p.ctrl->edges, edges);
        atomicAdd(&p.ctrl->num_top, ntop);
    }
}

}  // namespace

namespace eg {

/* one warp per vertex of the packed graph: CSC sort input and in-degrees */
__global__ void k_batch_expand(long long total_nodes, const int *P, const int2 *E, int *key, int *val, int *indeg)
{
    const int lane = threadIdx.x & 31;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long v = w0; v < total_nodes; v += nw) {
        for (int e = P[v] + lane; e < P[v + 1]; e += 32) {
            const int s = E[e].x;
            key[e] = s;
            val[e] = (int)v;
            atomicAdd(&indeg[s], 1);
        }
    }
}

size_t layout_bytes(int n, long long m)
{
    return sizeof(int) * ((size_t)n + 1) * 2 + sizeof(int) * (size_t)m + sizeof(int2) * (size_t)m + (size_t)n +
           2 * sizeof(int) * (size_t)n + 4096;
}

size_t layout_build_bytes(int n, long long m)
{
    return sizeof(int) * 4 * (size_t)(m + 1) + sizeof(int) * (size_t)(radix_scratch_ints(m) + scan_scratch_ints(n + 1) + 64);
}

void layout_free(GameLayout *l, cudaStream_t st)
{
    void *ptrs[] = {l->P, l->CP, l->CS, l->minw, l->maxw, l->E, l->owner};
    for (void *q : ptrs)
        if (q) cudaFreeAsync(q, st);
    memset(l, 0, sizeof *l);
}

eg_status layout_upload(const eg_game &G, cudaStream_t st, GameLayout *out)
{
    GameLayout L;
    memset(&L, 0, sizeof L);
    const int n = G.num_nodes;
    const long long m = G.num_edges;
    L.n = n;
    L.m = m;
    std::vector<int> P((size_t)n + 1), minw((size_t)n), maxw((size_t)n);
    std::vector<int2> E((size_t)m);
    std::vector<unsigned char> own((size_t)n);
    for (int v = 0; v < n; v++) {
        P[(size_t)v] = (int)G.row_ptr[v];
        own[(size_t)v] = G.owner ? G.owner[v] : (unsigned char)(v >= G.num_nodes0);
        int mn = INT32_MAX, mx = INT32_MIN;
        for (long long j = G.row_ptr[v]; j < G.row_ptr[v + 1]; j++) {
            E[(size_t)j] = make_int2(G.succ[j], G.weight[j]);
            mn = std::min(mn, G.weight[j]);
            mx = std::max(mx, G.weight[j]);
        }
        minw[(size_t)v] = mn;
        maxw[(size_t)v] = mx;
    }
    P[(size_t)n] = (int)m;
    cudaError_t e = cudaSuccess;
    /* stream-ordered allocations: no device-wide synchronisation, so kernels
     * already running on other streams keep running during an upload */
#define LA(ptr, cnt)                                                         \
    if (e == cudaSuccess) {                                                  \
        e = cudaMallocAsync((void **)&ptr, std::max<size_t>(sizeof(*ptr) * (size_t)(cnt), 16), st); \
    }
    LA(L.P, n + 1);
    LA(L.CP, n + 1);
    LA(L.CS, m);
    LA(L.E, m);
    LA(L.owner, n);
    LA(L.minw, n);
    LA(L.maxw, n);
    int *k0 = nullptr, *v0 = nullptr, *k1 = nullptr, *v1 = nullptr, *scr = nullptr;
    LA(k0, m + 1);
    LA(v0, m + 1);
    LA(k1, m + 1);
    LA(v1, m + 1);
    LA(scr, radix_scratch_ints(m) + scan_scratch_ints((long long)n + 1) + 64);
#undef LA
    if (e == cudaSuccess) e = cudaMemcpyAsync(L.P, P.data(), sizeof(int) * ((size_t)n + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(L.E, E.data(), sizeof(int2) * (size_t)m, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(L.owner, own.data(), (size_t)n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(L.minw, minw.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(L.maxw, maxw.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(L.CP, 0, sizeof(int) * ((size_t)n + 1), st);
    if (e == cudaSuccess) {
        long long gr = ((long long)n * 32 + 255) / 256;
        if (gr > 148 * 32) gr = 148 * 32;
        k_batch_expand<<<(unsigned)gr, 256, 0, st>>>(n, L.P, L.E, k0, v0, L.CP);
        excl_scan(L.CP, (long long)n + 1, scr, st);
        int *sk, *sv;
        radix_sort_pairs(k0, v0, k1, v1, m, bits_for(n), scr, st, &sk, &sv);
        e = cudaMemcpyAsync(L.CS, sv, sizeof(int) * (size_t)m, cudaMemcpyDeviceToDevice, st);
    }
    if (k0) cudaFreeAsync(k0, st);
    if (v0) cudaFreeAsync(v0, st);
    if (k1) cudaFreeAsync(k1, st);
    if (v1) cudaFreeAsync(v1, st);
    if (scr) cudaFreeAsync(scr, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        layout_free(&L, st);
        cudaStreamSynchronize(st);
        return eg_set_error(e == cudaErrorMemoryAllocation ? EG_ERR_OOM : EG_ERR_CUDA, "game upload failed: %s",
                            cudaGetErrorString(e));
    }
    L.bytes = layout_bytes(n, m);
    *out = L;
    return EG_OK;
}

GameDesc layout_desc(const GameLayout &l, const int *thr, long long *F, long long *rounds, int *status, int K, int d)
{
    GameDesc D;
    memset(&D, 0, sizeof D);
    D.P = l.P;
    D.E = l.E;
    D.CP = l.CP;
    D.CS = l.CS;
    D.owner = l.owner;
    D.minw = l.minw;
    D.maxw = l.maxw;
    D.thr = thr;
    D.F = F;
    D.rounds = rounds;
    D.status = status;
    D.base = 0;
    D.n = l.n;
    D.K = K;
    D.d = d;
    return D;
}

}  // namespace eg

namespace {

}  // namespace

namespace eg {

typedef void (*batch_kernel_t)(BatchParams);

batch_kernel_t kernel_for(int kp)
{
    switch (kp) {
    case 1: return k_batch_solve<1>;
    case 2: return k_batch_solve<2>;
    case 4: return k_batch_solve<4>;
    case 8: return k_batch_solve<8>;
    case 16: return k_batch_solve<16>;
    default: return k_batch_solve<32>;
    }
}

eg_status launch_batch(const BatchParams &p, int KP, int block, int num_sms, cudaStream_t st, int *grid_out)
{
    batch_kernel_t fn = kernel_for(KP);
    const size_t smem = 0; /* dense rounds keep no frontier */
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, block, smem);
    if (e != cudaSuccess || per_sm < 1)
        return eg_set_error(EG_ERR_CUDA, "batch kernel does not fit (block %d, %zu B shared)", block, smem);
    int grid = num_sms * per_sm;
    if (grid > p.num_games) grid = p.num_games;
    if (grid < 1) grid = 1;
    e = cudaMemsetAsync(p.ctrl, 0, sizeof(BatchCtrl), st);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    void *args[] = {(void *)&p};
    e = cudaLaunchKernel((const void *)fn, dim3(grid), dim3(block), args, smem, st);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "batch kernel launch failed: %s", cudaGetErrorString(e));
    *grid_out = grid;
    return EG_OK;
}

}  // namespace eg

namespace {

int pow2_at_least(int k)
{
    int x = 1;
    while (x < k) x <<= 1;
    return x;
}

}  // namespace

struct eg_batch {
    int device;
    cudaStream_t st;
    cudaEvent_t ev0, ev1;
    int num_games, K, KP, d;
    long long total_nodes, total_edges;
    int words_max;
    int block;
    long long max_rounds;
    double timeout_ms;
    std::vector<long long> node_off_h;
    long long *node_off;
    int *order, *P, *CP, *CS, *minw, *maxw, *thr, *status;
    int2 *E;
    unsigned char *owner;
    long long *F, *rounds;
    BatchCtrl *ctrl;
    GameDesc *desc;
    size_t bytes;
    bool thresholds_set, solved;
    bool use_graph;
    cudaGraph_t graph;
    cudaGraphExec_t graph_exec;
    int graph_block;
};

template <class T>
static eg_status balloc(eg_batch *b, T **p, size_t count)
{
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return eg_set_error(EG_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    b->bytes += bytes;
    return EG_OK;
}

extern "C" void eg_batch_free(eg_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    void *ptrs[] = {b->node_off, b->order, b->P, b->CP, b->CS, b->minw, b->maxw, b->thr,
                    b->status, b->E, b->owner, b->F, b->rounds, b->ctrl, b->desc};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

extern "C" int64_t eg_batch_device_bytes(const eg_batch *b) { return b ? (int64_t)b->bytes : 0; }

extern "C" eg_status eg_batch_create(const eg_game *games, int32_t num_games, const eg_batch_opts *opts, eg_batch **out)
{
    if (!games || num_games <= 0 || !opts || !out) return eg_set_error(EG_ERR_INVALID, "bad batch arguments");
    if (opts->thresholds < 1 || opts->thresholds > EG_BATCH_MAX_K)
        return eg_set_error(EG_ERR_INVALID, "thresholds must be in [1, %d]", EG_BATCH_MAX_K);
    if (opts->scale < 1) return eg_set_error(EG_ERR_INVALID, "scale d must be >= 1");
    if (opts->block && (opts->block < 64 || opts->block > 1024 || (opts->block & 31)))
        return eg_set_error(EG_ERR_INVALID, "block must be a multiple of 32 in [64, 1024]");
    long long tn = 0, tm = 0;
    int nmax = 0;
    for (int g = 0; g < num_games; g++) {
        eg_status s = eg_validate(&games[g]);
        if (s != EG_OK) return eg_set_error(s, "game %d: %s", g, eg_last_error());
        if (games[g].num_nodes > kBatchMaxGameNodes)
            return eg_set_error(EG_ERR_INVALID, "game %d has %d vertices; the batch path holds at most %d per game",
                                g, games[g].num_nodes, kBatchMaxGameNodes);
        tn += games[g].num_nodes;
        tm += games[g].num_edges;
        nmax = std::max(nmax, games[g].num_nodes);
    }
    if (tn >= (long long)INT32_MAX - 64 || tm >= (long long)INT32_MAX - 64)
        return eg_set_error(EG_ERR_INVALID, "batch too large (%lld vertices, %lld edges)", tn, tm);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return eg_set_error(EG_ERR_NO_DEVICE, "no CUDA device available");
    }
    EG_CUDA(cudaSetDevice(opts->device));
    eg_batch *b = new eg_batch();
    b->device = opts->device;
    b->num_games = num_games;
    b->K = opts->thresholds;
    b->KP = pow2_at_least(opts->thresholds);
    b->d = opts->scale;
    b->total_nodes = tn;
    b->total_edges = tm;
    b->words_max = (nmax + 31) / 32;
    b->block = opts->block ? opts->block : 1024;
    b->max_rounds = opts->max_rounds;
    b->timeout_ms = opts->timeout_ms;
    b->use_graph = opts->use_graph != 0;
    /* host packing: global ids, owners, min/max out-weight */
    std::vector<int> P((size_t)tn + 1), minw((size_t)tn), maxw((size_t)tn);
    std::vector<int2> E((size_t)tm);
    std::vector<unsigned char> own((size_t)tn);
    b->node_off_h.assign((size_t)num_games + 1, 0);
    long long vb = 0, eb = 0;
    for (int g = 0; g < num_games; g++) {
        const eg_game &G = games[g];
        b->node_off_h[g] = vb;
        for (int v = 0; v < G.num_nodes; v++) {
            P[(size_t)(vb + v)] = (int)(eb + G.row_ptr[v]);
            own[(size_t)(vb + v)] = G.owner ? G.owner[v] : (unsigned char)(v >= G.num_nodes0);
            int mn = INT32_MAX, mx = INT32_MIN;
            for (long long j = G.row_ptr[v]; j < G.row_ptr[v + 1]; j++) {
                const int w = G.weight[j];
                E[(size_t)(eb + j)] = make_int2((int)(vb + G.succ[j]), w);
                mn = std::min(mn, w);
                mx = std::max(mx, w);
            }
            minw[(size_t)(vb + v)] = mn;
            maxw[(size_t)(vb + v)] = mx;
        }
        vb += G.num_nodes;
        eb += G.num_edges;
    }
    b->node_off_h[num_games] = vb;
    P[(size_t)tn] = (int)tm;
    std::vector<int> order((size_t)num_games);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return games[a].num_edges > games[c].num_edges; });

    eg_status s = EG_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e != cudaSuccess) s = eg_set_error(EG_ERR_CUDA, "stream/event creation failed: %s", cudaGetErrorString(e));
    if (s == EG_OK) s = balloc(b, &b->node_off, (size_t)num_games + 1);
    if (s == EG_OK) s = balloc(b, &b->order, (size_t)num_games);
    if (s == EG_OK) s = balloc(b, &b->P, (size_t)tn + 1);
    if (s == EG_OK) s = balloc(b, &b->CP, (size_t)tn + 1);
    if (s == EG_OK) s = balloc(b, &b->CS, (size_t)tm);
    if (s == EG_OK) s = balloc(b, &b->E, (size_t)tm);
    if (s == EG_OK) s = balloc(b, &b->owner, (size_t)tn);
    if (s == EG_OK) s = balloc(b, &b->minw, (size_t)tn);
    if (s == EG_OK) s = balloc(b, &b->maxw, (size_t)tn);
    if (s == EG_OK) s = balloc(b, &b->thr, (size_t)num_games * b->K);
    if (s == EG_OK) s = balloc(b, &b->F, (size_t)tn * b->K);
    if (s == EG_OK) s = balloc(b, &b->rounds, (size_t)num_games);
    if (s == EG_OK) s = balloc(b, &b->status, (size_t)num_games);
    if (s == EG_OK) s = balloc(b, &b->ctrl, 1);
    if (s == EG_OK) s = balloc(b, &b->desc, (size_t)num_games);
    if (s != EG_OK) {
        eg_batch_free(b);
        return s;
    }
    /* one descriptor per game, pointing into the packed arrays */
    std::vector<GameDesc> desc((size_t)num_games);
    for (int g = 0; g < num_games; g++) {
        const long long base = b->node_off_h[g];
        GameDesc &D = desc[(size_t)g];
        D.P = b->P + base;
        D.E = b->E;
        D.CP = b->CP + base;
        D.CS = b->CS;
        D.owner = b->owner + base;
        D.minw = b->minw + base;
        D.maxw = b->maxw + base;
        D.thr = b->thr + (long long)g * b->K;
        D.F = b->F + base * b->K;
        D.rounds = b->rounds + g;
        D.status = b->status + g;
        D.base = base;
        D.n = games[g].num_nodes;
        D.K = b->K;
        D.d = b->d;
        D.pad = 0;
    }
    cudaStream_t st = b->st;
    e = cudaMemcpyAsync(b->node_off, b->node_off_h.data(), sizeof(long long) * ((size_t)num_games + 1),
                        cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->order, order.data(), sizeof(int) * (size_t)num_games, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->desc, desc.data(), sizeof(GameDesc) * desc.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->P, P.data(), sizeof(int) * ((size_t)tn + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->E, E.data(), sizeof(int2) * (size_t)tm, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->owner, own.data(), (size_t)tn, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->minw, minw.data(), sizeof(int) * (size_t)tn, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b->maxw, maxw.data(), sizeof(int) * (size_t)tn, cudaMemcpyHostToDevice, st);
    /* CSC by the stable counting sort, with temporary sort buffers */
    int *k0 = nullptr, *v0 = nullptr, *k1 = nullptr, *v1 = nullptr, *scr = nullptr;
    const long long scr_ints = radix_scratch_ints(tm) + scan_scratch_ints(tn + 1) + 64;
    if (e == cudaSuccess) e = cudaMalloc(&k0, sizeof(int) * (size_t)std::max<long long>(tm, 1));
    if (e == cudaSuccess) e = cudaMalloc(&v0, sizeof(int) * (size_t)std::max<long long>(tm, 1));
    if (e == cudaSuccess) e = cudaMalloc(&k1, sizeof(int) * (size_t)std::max<long long>(tm, 1));
    if (e == cudaSuccess) e = cudaMalloc(&v1, sizeof(int) * (size_t)std::max<long long>(tm, 1));
    if (e == cudaSuccess) e = cudaMalloc(&scr, sizeof(int) * (size_t)scr_ints);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->CP, 0, sizeof(int) * ((size_t)tn + 1), st);
    if (e == cudaSuccess) {
        long long gr = (tn * 32 + 255) / 256;
        if (gr > 148 * 32) gr = 148 * 32;
        k_batch_expand<<<(unsigned)gr, 256, 0, st>>>(tn, b->P, b->E, k0, v0, b->CP);
        excl_scan(b->CP, tn + 1, scr, st);
        int *sk, *sv;
        radix_sort_pairs(k0, v0, k1, v1, tm, bits_for(tn), scr, st, &sk, &sv);
        e = cudaMemcpyAsync(b->CS, sv, sizeof(int) * (size_t)tm, cudaMemcpyDeviceToDevice, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(k0);
    cudaFree(v0);
    cudaFree(k1);
    cudaFree(v1);
    cudaFree(scr);
    if (e != cudaSuccess) {
        s = eg_set_error(e == cudaErrorMemoryAllocation ? EG_ERR_OOM : EG_ERR_CUDA, "batch upload failed: %s",
                         cudaGetErrorString(e));
        cudaGetLastError();
        eg_batch_free(b);
        return s;
    }
    *out = b;
    return EG_OK;
}

extern "C" eg_status eg_batch_set_thresholds(eg_batch *b, const int32_t *p)
{
    if (!b || !p) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    EG_CUDA(cudaSetDevice(b->device));
    EG_CUDA(cudaMemcpyAsync(b->thr, p, sizeof(int) * (size_t)b->num_games * b->K, cudaMemcpyHostToDevice, b->st));
    EG_CUDA(cudaStreamSynchronize(b->st));
    b->thresholds_set = true;
    return EG_OK;
}

static eg_status batch_params(eg_batch *b, BatchParams *p)
{
    memset(p, 0, sizeof *p);
    p->games = b->desc;
    p->order = b->order;
    p->ctrl = b->ctrl;
    p->num_games = b->num_games;
    p->words_max = b->words_max;
    p->max_rounds = b->max_rounds;
    p->timeout_ns = b->timeout_ms > 0 ? (unsigned long long)(b->timeout_ms * 1e6) : 0ull;
    return EG_OK;
}

/* Enqueues one solve (control reset + persistent kernel) on the stream. */
static eg_status batch_enqueue(eg_batch *b, int block, int *grid_out)
{
    BatchParams p;
    batch_params(b, &p);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    return launch_batch(p, b->KP, block, sms, b->st, grid_out);
}

extern "C" eg_status eg_batch_solve(eg_batch *b, eg_batch_stats *stats)
{
    if (!b) return eg_set_error(EG_ERR_INVALID, "batch is NULL");
    if (!b->thresholds_set) return eg_set_error(EG_ERR_INVALID, "thresholds not set");
    EG_CUDA(cudaSetDevice(b->device));
    int grid = 0;
    bool replay = false;
    EG_CUDA(cudaEventRecord(b->ev0, b->st));
    if (b->use_graph) {
        if (!b->graph_exec || b->graph_block != b->block) {
            if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
            if (b->graph) cudaGraphDestroy(b->graph);
            b->graph_exec = nullptr;
            b->graph = nullptr;
            /* capture on a side stream so that the timing events stay outside the graph */
            cudaStream_t cs;
            EG_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            EG_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            cudaStream_t keep = b->st;
            b->st = cs;
            eg_status s = batch_enqueue(b, b->block, &grid);
            b->st = keep;
            cudaGraph_t gph = nullptr;
            cudaError_t e = cudaStreamEndCapture(cs, &gph);
            cudaStreamDestroy(cs);
            if (s != EG_OK) {
                if (gph) cudaGraphDestroy(gph);
                return s;
            }
            if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
            b->graph = gph;
            EG_CUDA(cudaGraphInstantiate(&b->graph_exec, b->graph, 0));
            b->graph_block = b->block;
        } else {
            replay = true;
        }
        EG_CUDA(cudaGraphLaunch(b->graph_exec, b->st));
    } else {
        EG_TRY(batch_enqueue(b, b->block, &grid));
    }
    EG_CUDA(cudaEventRecord(b->ev1, b->st));
    BatchCtrl c;
    EG_CUDA(cudaMemcpyAsync(&c, b->ctrl, sizeof c, cudaMemcpyDeviceToHost, b->st));
    std::vector<long long> rounds((size_t)b->num_games);
    std::vector<int> status((size_t)b->num_games);
    EG_CUDA(cudaMemcpyAsync(rounds.data(), b->rounds, sizeof(long long) * rounds.size(), cudaMemcpyDeviceToHost, b->st));
    EG_CUDA(cudaMemcpyAsync(status.data(), b->status, sizeof(int) * status.size(), cudaMemcpyDeviceToHost, b->st));
    EG_CUDA(cudaStreamSynchronize(b->st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->solved = true;
    int failed = 0;
    long long rmax = 0, rsum = 0;
    eg_status first = EG_OK;
    for (int g = 0; g < b->num_games; g++) {
        rmax = std::max(rmax, rounds[g]);
        rsum += rounds[g];
        if (status[g] != EG_OK) {
            failed++;
            if (first == EG_OK) first = (eg_status)status[g];
        }
    }
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->num_games = b->num_games;
        stats->thresholds = b->K;
        stats->total_nodes = b->total_nodes;
        stats->total_edges = b->total_edges;
        stats->rounds_max = rmax;
        stats->rounds_sum = rsum;
        stats->lifts = (int64_t)c.lifts;
        stats->edges = (int64_t)c.edges;
        stats->num_top = (int64_t)c.num_top;
        stats->solve_ms = ms;
        stats->block = b->block;
        stats->grid = grid;
        stats->games_failed = failed;
        stats->graph_replayed = replay ? 1 : 0;
    }
    if (first != EG_OK) return eg_set_error(first, "%d game(s) stopped early (status %d)", failed, (int)first);
    return EG_OK;
}

extern "C" eg_status eg_batch_credits(eg_batch *b, int32_t game, int64_t *credits)
{
    if (!b || !credits || game < 0 || game >= b->num_games) return eg_set_error(EG_ERR_INVALID, "bad arguments");
    if (!b->solved) return eg_set_error(EG_ERR_INVALID, "batch not solved");
    EG_CUDA(cudaSetDevice(b->device));
    const long long base = b->node_off_h[game], n = b->node_off_h[game + 1] - base;
    std::vector<long long> rows((size_t)(n * b->K));
    EG_CUDA(cudaMemcpyAsync(rows.data(), b->F + base * b->K, sizeof(long long) * rows.size(), cudaMemcpyDeviceToHost, b->st));
    EG_CUDA(cudaStreamSynchronize(b->st));
    for (long long v = 0; v < n; v++)
        for (int k = 0; k < b->K; k++) credits[(size_t)k * n + v] = rows[(size_t)(v * b->K + k)];
    return EG_OK;
}

extern "C" eg_status eg_batch_game_result(eg_batch *b, int32_t game, int64_t *rounds, int32_t *status)
{
    if (!b || game < 0 || game >= b->num_games) return eg_set_error(EG_ERR_INVALID, "bad arguments");
    EG_CUDA(cudaSetDevice(b->device));
    long long r = 0;
    int s = 0;
    EG_CUDA(cudaMemcpyAsync(&r, b->rounds + game, sizeof r, cudaMemcpyDeviceToHost, b->st));
    EG_CUDA(cudaMemcpyAsync(&s, b->status + game, sizeof s, cudaMemcpyDeviceToHost, b->st));
    EG_CUDA(cudaStreamSynchronize(b->st));
    if (rounds) *rounds = r;
    if (status) *status = s;
    return EG_OK;
}

/* Autotuner: each candidate CTA size solves the batch under a round cap
 * (enough rounds to reach steady state, few enough to be quick); the one
 * with the most edge relaxations per second is kept. */
extern "C" eg_status eg_batch_tune(eg_batch *b, int32_t *block_out)
{
    if (!b) return eg_set_error(EG_ERR_INVALID, "batch is NULL");
    if (!b->thresholds_set) return eg_set_error(EG_ERR_INVALID, "thresholds not set");
    const int cands[] = {256, 512, 1024};
    const long long keep_cap = b->max_rounds;
    const bool keep_graph = b->use_graph;
    b->use_graph = false;
    b->max_rounds = 64;
    double best = -1.0;
    int best_block = b->block;
    for (int c : cands) {
        b->block = c;
        eg_batch_stats st;
        eg_status s = eg_batch_solve(b, &st);
        if (s != EG_OK && s != EG_ERR_LOOPCAP) continue;
        const double rate = st.solve_ms > 0 ? (double)st.edges / st.solve_ms : 0.0;
        if (rate > best) {
            best = rate;
            best_block = c;
        }
    }
    b->block = best_block;
    b->max_rounds = keep_cap;
    b->use_graph = keep_graph;
    b->solved = false;
    if (block_out) *block_out = best_block;
    if (best < 0) return eg_set_error(EG_ERR_CUDA, "no candidate CTA size ran");
    return EG_OK;
}
