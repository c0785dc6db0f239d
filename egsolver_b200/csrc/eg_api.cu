/*
 * eg_api.cu -- host orchestration and the C-ABI entry points of the solver:
 * resident games (upload, solve, credits), the one-call solve, the
 * standalone CSR -> CSC transpose and cancel flags.
 *
 * The reference's GPU boundary (reference src/dev_solver.cu:81-266) keeps
 * one packed device allocation per process and addresses it through
 * __device__ globals set with cudaMemcpyToSymbol; here every resident game
 * is a handle that owns its device arrays, so several games can be resident
 * at once and no global state is shared between solves.
 */
#include "eg_lift.cuh"
#include "eg_prep.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
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

constexpr unsigned long long kWaitLimitNs = 5ull * 1000ull * 1000ull * 1000ull; /* 5 s per barrier wait */
constexpr int kPrepBlock = 256;
/* AUTO lifts a game with one CTA (frontier in shared memory) up to this
 * many edges; larger games use the persistent grid. */
constexpr long long kSmallGameEdges = 1 << 17;
/* default round-kind thresholds, raises per thousand vertices */
constexpr long long kDensePermille = 40;
constexpr long long kSparsePermille = 15;
constexpr int kSmallGameMaxPad = 1 << 19;

inline unsigned grid_for(long long items, int block, int cap = 148 * 32)
{
    long long g = (items + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

inline int align32(long long x) { return (int)((x + 31) & ~31LL); }

}  // namespace

struct eg_dgame {
    int device;
    cudaStream_t st;
    cudaEvent_t ev[6]; /* solve start, lift start, lift end, solve end; dense launch start / end */
    int n, n0;
    long long m;
    bool has_owner;
    /* input CSR (device copy) */
    long long *d_rowptr;
    int *d_succ, *d_w;
    unsigned char *d_owner;
    /* capacities */
    int n_pad_cap;
    long long m_pad_cap, tmp_cap, scratch_ints;
    /* layout of the last preprocessing */
    bool prepared;
    BucketBounds bb;
    int groups[EG_MAX_CLASSES / 2];
    ClassTable ct;
    int n_pad, words;
    long long m_pad;
    int *d_perm, *d_iperm, *d_P, *d_CP, *d_CS;
    int2 *d_E;
    unsigned char *d_active0;
    int *d_k0, *d_v0, *d_k1, *d_v1, *d_scratch;
    int *d_counts;
    unsigned long long *d_mg;
    void *d_F, *d_out;
    uint32_t *d_B;
    Ctrl *d_ctrl;
    /* heavy vertices cut into edge tasks (AUTO layout) */
    int4 *d_tasks;
    void *d_hacc;
    int *d_hrem, *d_toff;
    long long task_cap;
    int num_tasks, heavy_begin, heavy_bucket, task_pairs;
    /* dense rounds: pair-stream metadata and cut-vertex accumulators */
    uint16_t *d_PM;
    int *d_CB, *d_merr, *d_drem;
    void *d_dacc;
    int npairs;
    bool meta_ok;
    /* the same pairs in 8 bytes when successor and weight fit 32 bits:
     * (succ << wbits) | (w + wmax) per out-edge */
    int2 *d_E8;
    int wbits; /* 0: not packed */
    long long wmax;
    size_t bytes;
    long long mg;
    int solved_bits;
    bool solved;
    long long launches;
};

/* ------------------------------------------------------------------ */
/* Devices and options                                                  */
/* ------------------------------------------------------------------ */

extern "C" eg_status eg_device_count(int32_t *count)
{
    int n = 0;
    *count = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return eg_set_error(EG_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    }
    int ok = 0;
    for (int d = 0; d < n; d++) {
        int major = 0;
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d);
        if (major == 10) ok++;
    }
    *count = ok;
    return EG_OK;
}

/* Degree buckets and the lane-group size of each bucket.
 * AUTO / SMEM: deg <= small_max_deg (8) thread-per-vertex, up to
 * large_min_deg - 1 (64) eight lanes, from large_min_deg (65) on "heavy":
 * cut into edge tasks on the grid, a warp per vertex in the one-CTA kernel.
 * Forced variants keep the reference-style buckets below. */
static void choose_layout(const eg_opts *o, BucketBounds *bb, int *groups)
{
    const int v = o ? o->variant : EG_VARIANT_AUTO;
    if (v == EG_VARIANT_AUTO || v == EG_VARIANT_SMEM) {
        /* light vertices (deg < large_min_deg, default 17) in warp-cooperative
         * words; heavy ones as edge tasks (a warp each in the one-CTA kernel).
         * small_max_deg > 0 splits off a thread-per-vertex bucket. */
        const int heavy = o && o->large_min_deg > 1 ? o->large_min_deg : 17;
        const int small = o && o->small_max_deg > 0 ? o->small_max_deg : 0;
        int nb = 0;
        if (small > 0 && small < heavy - 1) {
            bb->upper[nb] = small;
            groups[nb++] = 1;
        }
        bb->upper[nb] = heavy - 1;
        groups[nb++] = EG_GROUP_LIGHT;
        groups[nb++] = 32;
        bb->nb = nb;
        return;
    }
    const int small = o && o->small_max_deg > 0 ? o->small_max_deg : 8;
    const int large = o && o->large_min_deg > 0 ? o->large_min_deg : 1024;
    if (v == EG_VARIANT_THREAD || v == EG_VARIANT_WARP || v == EG_VARIANT_CTA) {
        bb->nb = 1;
        int g = 1;
        if (v == EG_VARIANT_WARP) g = (o->lanes_per_vertex > 0) ? o->lanes_per_vertex : 32;
        if (v == EG_VARIANT_CTA) g = EG_GROUP_CTA;
        groups[0] = g;
        return;
    }
    int nb = 0;
    bb->upper[nb] = small;
    groups[nb++] = 1;
    if (small < 64 && large > 65) {
        bb->upper[nb] = 64;
        groups[nb++] = 8;
    }
    const int prev = bb->upper[nb - 1];
    if (large - 1 > prev) {
        bb->upper[nb] = large - 1;
        groups[nb++] = 32;
    }
    groups[nb++] = EG_GROUP_CTA;
    bb->nb = nb;
}

static eg_status check_lanes(const eg_opts *o)
{
    if (o && o->variant == EG_VARIANT_WARP && o->lanes_per_vertex) {
        const int k = o->lanes_per_vertex;
        if (k != 1 && k != 2 && k != 4 && k != 8 && k != 16 && k != 32)
            return eg_set_error(EG_ERR_INVALID, "lanes_per_vertex must be 1, 2, 4, 8, 16 or 32 (got %d)", k);
    }
    if (o && (o->variant < 0 || o->variant > EG_VARIANT_SMEM))
        return eg_set_error(EG_ERR_INVALID, "unknown variant %d", o->variant);
    if (o && o->credit_bits != 0 && o->credit_bits != 32 && o->credit_bits != 64)
        return eg_set_error(EG_ERR_INVALID, "credit_bits must be 32 or 64 (got %d)", o->credit_bits);
    if (o && (o->direction < EG_DIRECTION_SWITCH || o->direction > EG_DIRECTION_DENSE))
        return eg_set_error(EG_ERR_INVALID, "unknown direction %d", o->direction);
    if (o && (o->dense_sweeps < 0 || o->dense_sweeps > kMaxDenseSweeps))
        return eg_set_error(EG_ERR_INVALID, "dense_sweeps must be in [0, %d] (got %d)", kMaxDenseSweeps, o->dense_sweeps);
    if (o && (o->dense_depth < 0 || o->dense_depth > 2))
        return eg_set_error(EG_ERR_INVALID, "dense_depth must be 0, 1 or 2 (got %d)", o->dense_depth);
    if (o && (o->dense_permille < 0 || o->dense_permille > 1000 || o->sparse_permille < 0 || o->sparse_permille > 1000))
        return eg_set_error(EG_ERR_INVALID, "round-kind thresholds must be 0..1000 per mille");
    return EG_OK;
}

/* ------------------------------------------------------------------ */
/* Resident games                                                       */
/* ------------------------------------------------------------------ */

template <class P>
static eg_status dalloc(eg_dgame *g, P **p, size_t count)
{
    size_t bytes = count * sizeof(P);
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc((void **)p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return eg_set_error(EG_ERR_OOM, "cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    g->bytes += bytes;
    return EG_OK;
}

extern "C" void eg_dgame_free(eg_dgame *g)
{
    if (!g) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    if (g->st) cudaStreamSynchronize(g->st);
    void *ptrs[] = {g->d_rowptr, g->d_succ, g->d_w, g->d_owner, g->d_perm, g->d_iperm, g->d_P, g->d_CP,
                    g->d_CS, g->d_E, g->d_active0, g->d_k0, g->d_v0, g->d_k1, g->d_v1, g->d_scratch,
                    g->d_counts, g->d_mg, g->d_F, g->d_out, g->d_B, g->d_ctrl, g->d_tasks, g->d_hacc,
                    g->d_hrem, g->d_toff, g->d_PM, g->d_CB, g->d_merr, g->d_drem, g->d_dacc, g->d_E8};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (int i = 0; i < 6; i++)
        if (g->ev[i]) cudaEventDestroy(g->ev[i]);
    if (g->st) cudaStreamDestroy(g->st);
    cudaSetDevice(prev);
    free(g);
}

static eg_status dgame_alloc(const eg_game *game, const eg_opts *opts, eg_dgame **out)
{
    {
        /* the padded row offsets (up to one pad pair per vertex) and the
         * padded predecessor offsets (up to three pads per vertex) are int */
        const long long npc = align32(game->num_nodes) + 32LL * (EG_MAX_CLASSES + 1);
        if (game->num_edges + 3 * npc + 64 > (long long)INT32_MAX)
            return eg_set_error(EG_ERR_INVALID,
                                "game too large: %lld edges plus padding for %d vertices exceed 32-bit offsets",
                                (long long)game->num_edges, game->num_nodes);
    }
    const int dev = opts ? opts->device : 0;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return eg_set_error(EG_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (dev < 0 || dev >= count) return eg_set_error(EG_ERR_INVALID, "device %d not available (%d devices)", dev, count);
    EG_CUDA(cudaSetDevice(dev));
    int major = 0;
    EG_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) return eg_set_error(EG_ERR_NO_DEVICE, "device %d is sm_%d0, this library is built for sm_100a", dev, major);
    eg_dgame *g = (eg_dgame *)calloc(1, sizeof(eg_dgame));
    if (!g) return eg_set_error(EG_ERR_OOM, "host allocation failed");
    g->device = dev;
    g->n = game->num_nodes;
    g->n0 = game->num_nodes0;
    g->m = game->num_edges;
    g->has_owner = game->owner != nullptr;
    g->n_pad_cap = align32(g->n) + 32 * (EG_MAX_CLASSES + 1);
    g->m_pad_cap = g->m + g->n_pad_cap;
    g->tmp_cap = std::max<long long>(g->m, g->n) + 1;
    g->scratch_ints = radix_scratch_ints(g->tmp_cap) + scan_scratch_ints(g->n_pad_cap + 1) + 64;
    eg_status s = EG_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) s = eg_set_error(EG_ERR_CUDA, "cudaStreamCreate failed: %s", cudaGetErrorString(e));
    for (int i = 0; i < 6 && s == EG_OK; i++)
        if (cudaEventCreate(&g->ev[i]) != cudaSuccess) s = eg_set_error(EG_ERR_CUDA, "cudaEventCreate failed");
    const long long words = g->n_pad_cap / 32 + 2;
    if (s == EG_OK) s = dalloc(g, &g->d_rowptr, (size_t)g->n + 1);
    if (s == EG_OK) s = dalloc(g, &g->d_succ, (size_t)g->m);
    if (s == EG_OK) s = dalloc(g, &g->d_w, (size_t)g->m);
    if (s == EG_OK && g->has_owner) s = dalloc(g, &g->d_owner, (size_t)g->n);
    if (s == EG_OK) s = dalloc(g, &g->d_perm, (size_t)g->n_pad_cap);
    if (s == EG_OK) s = dalloc(g, &g->d_iperm, (size_t)g->n);
    if (s == EG_OK) s = dalloc(g, &g->d_P, (size_t)g->n_pad_cap + 1);
    if (s == EG_OK) s = dalloc(g, &g->d_CP, (size_t)g->n_pad_cap + 1);
    if (s == EG_OK) s = dalloc(g, &g->d_CS, (size_t)g->m + 3 * (size_t)g->n_pad_cap + 8);
    if (s == EG_OK) s = dalloc(g, &g->d_E, (size_t)g->m_pad_cap);
    if (s == EG_OK) s = dalloc(g, &g->d_active0, (size_t)g->n);
    if (s == EG_OK) s = dalloc(g, &g->d_k0, (size_t)g->tmp_cap);
    if (s == EG_OK) s = dalloc(g, &g->d_v0, (size_t)g->tmp_cap);
    if (s == EG_OK) s = dalloc(g, &g->d_k1, (size_t)g->tmp_cap);
    if (s == EG_OK) s = dalloc(g, &g->d_v1, (size_t)g->tmp_cap);
    if (s == EG_OK) s = dalloc(g, &g->d_scratch, (size_t)g->scratch_ints);
    if (s == EG_OK) s = dalloc(g, &g->d_counts, (size_t)EG_MAX_CLASSES);
    if (s == EG_OK) s = dalloc(g, &g->d_mg, 2); /* MG, largest |weight| */
    if (s == EG_OK) s = dalloc(g, (int64_t **)&g->d_F, (size_t)g->n_pad_cap + 64);
    if (s == EG_OK) s = dalloc(g, (int64_t **)&g->d_out, (size_t)g->n);
    if (s == EG_OK) s = dalloc(g, &g->d_B, (size_t)(4 * words)); /* two frontiers, two raised-maps */
    if (s == EG_OK) s = dalloc(g, &g->d_ctrl, 1);
    g->task_cap = g->m_pad_cap / 32 + g->n_pad_cap + 2; /* tasks of >= 16 pairs */
    if (s == EG_OK) s = dalloc(g, &g->d_tasks, (size_t)g->task_cap);
    if (s == EG_OK) s = dalloc(g, (int64_t **)&g->d_hacc, (size_t)g->n_pad_cap);
    if (s == EG_OK) s = dalloc(g, &g->d_hrem, (size_t)g->n_pad_cap);
    if (s == EG_OK) s = dalloc(g, &g->d_toff, (size_t)g->n_pad_cap + 1);
    if (s == EG_OK) s = dalloc(g, &g->d_PM, (size_t)(g->m_pad_cap / 2 + 64));
    if (s == EG_OK) s = dalloc(g, &g->d_CB, (size_t)(g->m_pad_cap / 64 + 4));
    if (s == EG_OK) s = dalloc(g, &g->d_merr, 1);
    /* one bank of cut-vertex accumulators per sweep of a dense round */
    if (s == EG_OK) s = dalloc(g, &g->d_drem, (size_t)kMaxDenseSweeps * (size_t)g->n_pad_cap);
    if (s == EG_OK) s = dalloc(g, (int64_t **)&g->d_dacc, (size_t)kMaxDenseSweeps * (size_t)g->n_pad_cap);
    if (s == EG_OK) s = dalloc(g, &g->d_E8, (size_t)(g->m_pad_cap / 2 + 64));
    if (s != EG_OK) {
        eg_dgame_free(g);
        return s;
    }
    *out = g;
    return EG_OK;
}

extern "C" eg_status eg_dgame_upload(const eg_game *game, const eg_opts *opts, eg_dgame **out)
{
    if (!out) return eg_set_error(EG_ERR_INVALID, "out is NULL");
    EG_TRY(eg_validate(game));
    EG_TRY(check_lanes(opts));
    eg_dgame *g = nullptr;
    EG_TRY(dgame_alloc(game, opts, &g));
    cudaError_t e = cudaMemcpyAsync(g->d_rowptr, game->row_ptr, sizeof(long long) * ((size_t)g->n + 1),
                                    cudaMemcpyHostToDevice, g->st);
    if (e == cudaSuccess && g->m)
        e = cudaMemcpyAsync(g->d_succ, game->succ, sizeof(int) * (size_t)g->m, cudaMemcpyHostToDevice, g->st);
    if (e == cudaSuccess && g->m)
        e = cudaMemcpyAsync(g->d_w, game->weight, sizeof(int) * (size_t)g->m, cudaMemcpyHostToDevice, g->st);
    if (e == cudaSuccess && g->has_owner)
        e = cudaMemcpyAsync(g->d_owner, game->owner, (size_t)g->n, cudaMemcpyHostToDevice, g->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
    if (e != cudaSuccess) {
        eg_status s = eg_set_error(EG_ERR_CUDA, "upload failed: %s", cudaGetErrorString(e));
        eg_dgame_free(g);
        return s;
    }
    *out = g;
    return EG_OK;
}

extern "C" eg_status eg_dgame_from_device(const eg_game *dev_game, const eg_opts *opts, eg_dgame **out)
{
    if (!dev_game || !out) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    if (dev_game->num_nodes <= 0 || dev_game->num_edges < dev_game->num_nodes ||
        dev_game->num_edges > (int64_t)INT32_MAX - 64)
        return eg_set_error(EG_ERR_INVALID, "game sizes out of range (n=%d, m=%lld)", dev_game->num_nodes,
                            (long long)dev_game->num_edges);
    EG_TRY(check_lanes(opts));
    eg_dgame *g = nullptr;
    EG_TRY(dgame_alloc(dev_game, opts, &g));
    cudaError_t e = cudaMemcpyAsync(g->d_rowptr, dev_game->row_ptr, sizeof(long long) * ((size_t)g->n + 1),
                                    cudaMemcpyDeviceToDevice, g->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->d_succ, dev_game->succ, sizeof(int) * (size_t)g->m, cudaMemcpyDeviceToDevice, g->st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g->d_w, dev_game->weight, sizeof(int) * (size_t)g->m, cudaMemcpyDeviceToDevice, g->st);
    if (e == cudaSuccess && g->has_owner)
        e = cudaMemcpyAsync(g->d_owner, dev_game->owner, (size_t)g->n, cudaMemcpyDeviceToDevice, g->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
    if (e != cudaSuccess) {
        eg_status s = eg_set_error(EG_ERR_CUDA, "device copy failed: %s", cudaGetErrorString(e));
        eg_dgame_free(g);
        return s;
    }
    *out = g;
    return EG_OK;
}

extern "C" int64_t eg_dgame_device_bytes(const eg_dgame *g) { return g ? (int64_t)g->bytes : 0; }

/* Transpose + renumbering: classify, sort classes, renumber, pack edges,
 * counting-sort the CSC.  Leaves g->mg set (one device->host read of the
 * class counts and MG). */
static eg_status dgame_prepare(eg_dgame *g, const eg_opts *opts)
{
    cudaStream_t st = g->st;
    const int n = g->n;
    BucketBounds bb;
    int groups[EG_MAX_CLASSES / 2];
    choose_layout(opts, &bb, groups);
    g->bb = bb;
    memcpy(g->groups, groups, sizeof groups);
    EG_CUDA(cudaMemsetAsync(g->d_counts, 0, sizeof(int) * EG_MAX_CLASSES, st));
    EG_CUDA(cudaMemsetAsync(g->d_mg, 0, 2 * sizeof(unsigned long long), st));
    k_classify<<<grid_for(n, kPrepBlock), kPrepBlock, 0, st>>>(n, g->n0, g->d_rowptr, g->d_w, g->d_owner, bb, g->d_k0,
                                                                   g->d_v0, g->d_active0, g->d_mg, g->d_counts);
    g->launches++;
    int counts[EG_MAX_CLASSES];
    unsigned long long mgw[2] = {0, 0};
    EG_CUDA(cudaMemcpyAsync(counts, g->d_counts, sizeof counts, cudaMemcpyDeviceToHost, st));
    EG_CUDA(cudaMemcpyAsync(mgw, g->d_mg, sizeof mgw, cudaMemcpyDeviceToHost, st));
    int *sk, *sv;
    const int nc = 2 * bb.nb;
    radix_sort_pairs(g->d_k0, g->d_v0, g->d_k1, g->d_v1, n, bits_for(nc - 1), g->d_scratch, st, &sk, &sv);
    g->launches += 3 * ((bits_for(nc - 1) + 7) / 8) + 3;
    EG_CUDA(cudaStreamSynchronize(st));
    g->mg = (long long)mgw[0];
    g->wmax = (long long)mgw[1];
    ClassTable ct;
    memset(&ct, 0, sizeof ct);
    ct.nc = nc;
    long long pos = 0, sorted = 0;
    for (int c = 0; c < nc; c++) {
        ct.start[c] = (int)pos;
        ct.count[c] = counts[c];
        ct.sorted_begin[c] = sorted;
        sorted += counts[c];
        pos = align32(pos + counts[c]);
    }
    g->ct = ct;
    g->n_pad = (int)pos;
    g->words = g->n_pad / 32;
    const int n_pad = g->n_pad;
    EG_CUDA(cudaMemsetAsync(g->d_perm, 0xff, sizeof(int) * (size_t)n_pad, st));
    k_build_perm<<<grid_for(n, kPrepBlock), kPrepBlock, 0, st>>>(n, sk, sv, ct, g->d_perm, g->d_iperm);
    k_new_degree<<<grid_for(n_pad + 1, kPrepBlock), kPrepBlock, 0, st>>>(n_pad, g->d_perm, g->d_rowptr, g->d_P);
    excl_scan(g->d_P, (long long)n_pad + 1, g->d_scratch, st);
    EG_CUDA(cudaMemsetAsync(g->d_CP, 0, sizeof(int) * ((size_t)n_pad + 1), st));
    k_copy_edges<<<grid_for((long long)n_pad * 32, kPrepBlock), kPrepBlock, 0, st>>>(
        n_pad, g->d_perm, g->d_iperm, g->d_rowptr, g->d_succ, g->d_w, g->d_P, g->d_E, g->d_k0, g->d_v0, g->d_CP, ct,
        n_pad, n_pad + 1);
    /* padded predecessor offsets (d_hrem serves as temporary: n_pad + 1 ints) */
    k_round4<<<grid_for(n_pad + 1, kPrepBlock), kPrepBlock, 0, st>>>(n_pad + 1, g->d_CP, g->d_hrem);
    excl_scan(g->d_CP, (long long)n_pad + 1, g->d_scratch, st);
    excl_scan(g->d_hrem, (long long)n_pad + 1, g->d_scratch, st);
    radix_sort_pairs(g->d_k0, g->d_v0, g->d_k1, g->d_v1, g->m, bits_for(n_pad + 1), g->d_scratch, st, &sk, &sv);
    k_csc_pad<<<grid_for((long long)n_pad * 32, kPrepBlock), kPrepBlock, 0, st>>>(n_pad, g->d_CP, g->d_hrem, sv, g->d_CS);
    EG_CUDA(cudaMemcpyAsync(g->d_CP, g->d_hrem, sizeof(int) * ((size_t)n_pad + 1), cudaMemcpyDeviceToDevice, st));
    g->launches += 8 + 3 * ((bits_for(n_pad + 1) + 7) / 8) * 2;
    /* AUTO layout: vertices of the warp / CTA buckets become 256-edge tasks */
    g->num_tasks = 0;
    g->heavy_bucket = g->bb.nb;
    g->heavy_begin = n_pad;
    if (!opts || opts->variant == EG_VARIANT_AUTO || opts->variant == EG_VARIANT_SMEM) {
        for (int b = 0; b < g->bb.nb; b++)
            if (g->groups[b] == 32 || g->groups[b] == EG_GROUP_CTA) {
                g->heavy_bucket = b;
                break;
            }
        if (g->heavy_bucket < g->bb.nb) {
            g->heavy_begin = ct.start[2 * g->heavy_bucket];
            const int nh = n_pad - g->heavy_begin;
            if (nh > 0) {
                const int tp = opts && opts->task_edges > 0 ? std::min(kTaskPairs, std::max(16, opts->task_edges / 2)) : kTaskPairs;
                g->task_pairs = tp;
                k_task_count<<<grid_for(nh + 1, kPrepBlock), kPrepBlock, 0, st>>>(g->heavy_begin, n_pad, g->d_P, tp,
                                                                                   g->d_toff);
                excl_scan(g->d_toff, (long long)nh + 1, g->d_scratch, st);
                int total = 0;
                EG_CUDA(cudaMemcpyAsync(&total, g->d_toff + nh, sizeof total, cudaMemcpyDeviceToHost, st));
                EG_CUDA(cudaStreamSynchronize(st));
                if (total > g->task_cap) return eg_set_error(EG_ERR_INVALID, "task list overflow (%d tasks)", total);
                k_task_fill<<<grid_for(nh, kPrepBlock), kPrepBlock, 0, st>>>(g->heavy_begin, n_pad, g->d_P, tp,
                                                                               g->d_toff, ct, g->d_tasks);
                g->num_tasks = total;
                g->launches += 5;
            }
        }
    }
    /* AUTO layout: the pair stream of the dense rounds */
    g->meta_ok = false;
    g->npairs = 0;
    if (!opts || opts->variant == EG_VARIANT_AUTO || opts->variant == EG_VARIANT_SMEM) {
        int pend = 0, merr = 0;
        EG_CUDA(cudaMemsetAsync(g->d_merr, 0, sizeof(int), st));
        EG_CUDA(cudaMemcpyAsync(&pend, g->d_P + n_pad, sizeof pend, cudaMemcpyDeviceToHost, st));
        EG_CUDA(cudaStreamSynchronize(st));
        g->npairs = pend / 2;
        build_pair_meta(g->d_P, n_pad, g->npairs, g->ct, g->d_PM, g->d_CB, g->d_merr, st);
        EG_CUDA(cudaMemcpyAsync(&merr, g->d_merr, sizeof merr, cudaMemcpyDeviceToHost, st));
        EG_CUDA(cudaStreamSynchronize(st));
        g->meta_ok = merr == 0 && g->npairs > 0;
        g->launches += 2;
        /* 8-byte pairs when ids up to the sentinels and weights in
         * [-wmax, wmax] share 32 bits */
        g->wbits = 0;
        const int sbits = bits_for((long long)n_pad + 1);
        const int wbits = bits_for(2 * g->wmax);
        if (g->meta_ok && sbits + wbits <= 32 && !(opts && opts->wide_pairs)) {
            g->wbits = wbits;
            launch_pack_pairs((const int4 *)g->d_E, g->npairs, wbits, (int)g->wmax, g->d_E8, st);
            g->launches++;
        }
    }
    EG_CUDA(cudaGetLastError());
    g->prepared = true;
    return EG_OK;
}

extern "C" eg_status eg_dgame_solve(eg_dgame *g, const eg_opts *opts_in, eg_stats *stats)
{
    if (!g) return eg_set_error(EG_ERR_INVALID, "game handle is NULL");
    eg_opts dflt;
    eg_opts_default(&dflt);
    const eg_opts *opts = opts_in ? opts_in : &dflt;
    EG_TRY(check_lanes(opts));
    EG_CUDA(cudaSetDevice(g->device));
    cudaStream_t st = g->st;
    g->launches = 0;
    g->solved = false;
    EG_CUDA(cudaEventRecord(g->ev[0], st));
    if (!(opts->keep_layout && g->prepared)) EG_TRY(dgame_prepare(g, opts));
    /* with opts->narrow, a 64-bit request computes in 32 bits when every
     * finite credit (<= MG) and every difference credit - weight fit: the
     * same credits, half the bytes, 32-bit warp reductions in dense rounds */
    const bool fast32 = g->mg + g->wmax < (long long)INT32_MAX;
    const int bits = opts->credit_bits == 32 ? 32 : (fast32 && opts->narrow) ? 32 : 64;
    if (bits == 32 && g->mg > (long long)INT32_MAX)
        return eg_set_error(EG_ERR_OVERFLOW, "MG = %lld does not fit 32-bit credits", g->mg);
    const int n_pad = g->n_pad;
    const int topv = n_pad;
    launch_init_credits(bits, n_pad + 64, g->d_F, topv, st);
    const long long wds = g->words + 2;
    EG_CUDA(cudaMemsetAsync(g->d_B, 0, sizeof(uint32_t) * (size_t)(4 * wds), st));
    k_init_frontier<<<grid_for(n_pad, kPrepBlock), kPrepBlock, 0, st>>>(n_pad, g->d_perm, g->d_active0, g->d_B);
    EG_CUDA(cudaMemsetAsync(g->d_ctrl, 0, sizeof(Ctrl), st));
    g->launches += 2;

    LiftParams p;
    memset(&p, 0, sizeof p);
    p.P = g->d_P;
    p.E4 = (const int4 *)g->d_E;
    p.CP = g->d_CP;
    p.CS = g->d_CS;
    p.F = g->d_F;
    p.B0 = g->d_B;
    p.B1 = g->d_B + wds;
    p.CH0 = g->d_B + 2 * wds;
    p.CH1 = g->d_B + 3 * wds;
    p.ctrl = g->d_ctrl;
    p.mg = g->mg;
    p.max_rounds = opts->max_rounds;
    p.timeout_ns = opts->timeout_ms > 0 ? (unsigned long long)(opts->timeout_ms * 1e6) : 0ull;
    p.wait_limit_ns = kWaitLimitNs;
    p.cancel = nullptr;
    if (opts->cancel) {
        void *dp = nullptr;
        EG_CUDA(cudaHostGetDevicePointer(&dp, (void *)opts->cancel, 0));
        p.cancel = (const int *)dp;
    }
    p.n_pad = n_pad;
    p.profile = opts->profile != 0;
    const bool small = n_pad <= kSmallGameMaxPad &&
                       (opts->variant == EG_VARIANT_SMEM || (opts->variant == EG_VARIANT_AUTO && g->m <= kSmallGameEdges));
    /* the grid kernel lifts heavy buckets as tasks; the one-CTA kernel
     * lifts every class by words */
    const bool tasks = !small && g->num_tasks > 0;
    int nc = 0;
    for (int b = g->bb.nb - 1; b >= 0; b--) {
        if (tasks && b >= g->heavy_bucket) continue;
        for (int own = 0; own < 2; own++) {
            const int c = b * 2 + own;
            if (g->ct.count[c] == 0) continue;
            LiftClass &lc = p.cls[nc++];
            lc.word_begin = g->ct.start[c] / 32;
            lc.word_end = (g->ct.start[c] + g->ct.count[c] + 31) / 32;
            lc.owner = own;
            lc.group = g->groups[b];
            lc.grab = g->groups[b] == 1 ? (opts->schedule == 1 ? -4 : 2) : 1;
        }
    }
    p.nclasses = nc;
    /* the lean kernel knows only light words and tasks (a game without a
     * heavy vertex has no tasks and runs light words alone) */
    p.lean = !small && (opts->variant == EG_VARIANT_AUTO || opts->variant == EG_VARIANT_SMEM) && opts->ctas_per_sm != 2 &&
             opts->small_max_deg <= 0;
    /* round kinds: the lean layout alternates frontier rounds (k_lift) and
     * dense rounds (k_lift_dense) */
    const bool kinds = p.lean && g->meta_ok && opts->direction != EG_DIRECTION_SPARSE;
    p.direction = kinds ? opts->direction : EG_DIRECTION_SPARSE;
    {
        const long long dpm = opts->dense_permille > 0 ? opts->dense_permille : kDensePermille;
        const long long spm = opts->sparse_permille > 0 ? opts->sparse_permille : kSparsePermille;
        p.dense_min_changes = std::max(1LL, (dpm * g->n + 999) / 1000);
        p.sparse_max_changes = spm * g->n / 1000;
    }
    if (tasks) {
        launch_task_reset(bits, g->heavy_begin, n_pad, g->d_toff, g->ct, g->d_hacc, g->d_hrem, st);
        g->launches++;
        p.tasks = g->d_tasks;
        p.num_tasks = g->num_tasks;
        p.heavy_begin = g->heavy_begin;
        p.hacc = g->d_hacc;
        p.hrem = g->d_hrem;
    }
    int grid = 0, block = 0, dgrid = 0, dense_launches = 0;
    double dense_ms = 0.0;
    if (kinds) {
        /* one slice of the pair stream per warp of the dense grid */
        p.dense_depth = opts->dense_depth == 1 ? 1 : 2;
        p.dense_sweeps = opts->dense_sweeps ? opts->dense_sweeps : kMaxDenseSweeps;
        EG_TRY(dense_grid(bits, p.dense_depth, opts->grid_ctas, &dgrid));
        const long long warps = (long long)dgrid * 16;
        const long long per = (g->npairs + warps - 1) / warps;
        p.PM = g->d_PM;
        p.CB = g->d_CB;
        p.npairs = g->npairs;
        p.slice = (int)std::max(32LL, (per + 31) / 32 * 32);
        p.dacc = g->d_dacc;
        p.drem = g->d_drem;
        p.E8 = g->wbits ? (const int2 *)g->d_E8 : nullptr;
        p.wbits = g->wbits;
        p.wbias = (int)g->wmax;
        p.fast32 = bits == 32 && fast32;
        launch_dense_setup(p, bits, st);
        g->launches++;
    }
    EG_CUDA(cudaEventRecord(g->ev[1], st));
    if (small) {
        EG_TRY(launch_lift_cta(p, bits, st));
        grid = 1;
        block = 1024;
        g->launches++;
    } else if (!kinds) {
        EG_TRY(launch_lift(p, bits, st, &grid, &block, opts->grid_ctas));
        g->launches++;
    } else {
        /* frontier and dense kernels take turns; each returns when its last
         * round picks the other kind (or the solve ends) */
        int kind = opts->direction == EG_DIRECTION_DENSE ? ROUND_DENSE : ROUND_SPARSE;
        for (;;) {
            if (kind == ROUND_DENSE) {
                EG_CUDA(cudaEventRecord(g->ev[4], st));
                EG_TRY(launch_lift_dense(p, bits, st, dgrid));
                EG_CUDA(cudaEventRecord(g->ev[5], st));
                grid = dgrid;
                block = 512;
                dense_launches++;
            } else {
                EG_TRY(launch_lift(p, bits, st, &grid, &block, opts->grid_ctas));
            }
            g->launches++;
            int tail[2] = {0, 0}; /* stop, next_mode */
            EG_CUDA(cudaMemcpyAsync(&tail[0], &g->d_ctrl->stop, sizeof(int), cudaMemcpyDeviceToHost, st));
            EG_CUDA(cudaMemcpyAsync(&tail[1], &g->d_ctrl->next_mode, sizeof(int), cudaMemcpyDeviceToHost, st));
            EG_CUDA(cudaStreamSynchronize(st));
            if (kind == ROUND_DENSE) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, g->ev[4], g->ev[5]);
                dense_ms += ms;
            }
            if (tail[0] || tail[1] == ROUND_DONE) break;
            kind = (tail[1] == ROUND_DENSE || tail[1] == ROUND_RECORD) ? ROUND_DENSE : ROUND_SPARSE;
        }
    }
    EG_CUDA(cudaEventRecord(g->ev[2], st));
    launch_count_top(bits, n_pad, g->d_F, &g->d_ctrl->num_top, st);
    g->launches++;
    EG_CUDA(cudaEventRecord(g->ev[3], st));
    Ctrl ctrl;
    EG_CUDA(cudaMemcpyAsync(&ctrl, g->d_ctrl, sizeof ctrl, cudaMemcpyDeviceToHost, st));
    EG_CUDA(cudaStreamSynchronize(st));
    float solve_ms = 0.f, lift_ms = 0.f;
    cudaEventElapsedTime(&solve_ms, g->ev[0], g->ev[3]);
    cudaEventElapsedTime(&lift_ms, g->ev[1], g->ev[2]);
    g->solved_bits = bits;
    g->solved = true;
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->mg = g->mg;
        stats->rounds = ctrl.rounds;
        /* a dense round lifts every vertex and scans every edge once */
        stats->lifts = (int64_t)ctrl.lifts + (int64_t)ctrl.dense_rounds * g->n;
        stats->edges = (int64_t)ctrl.edges + (int64_t)ctrl.dense_rounds * g->m;
        stats->num_top = (int64_t)ctrl.num_top;
        stats->solve_ms = solve_ms;
        stats->lift_ms = lift_ms;
        stats->kernel_launches = g->launches;
        stats->credit_bits = bits;
        stats->small_max_deg = g->bb.nb > 1 ? g->bb.upper[0] : 0;
        stats->large_min_deg = g->bb.nb > 1 ? g->bb.upper[g->bb.nb - 2] + 1 : 0;
        stats->variant_small = g->groups[0];
        stats->variant_mid = g->bb.nb > 2 ? g->groups[1] : g->groups[0];
        stats->variant_large = g->groups[g->bb.nb - 1];
        stats->changes = (int64_t)ctrl.changes;
        stats->pushes = (int64_t)ctrl.pushes;
        stats->grid = grid;
        stats->block = block;
        stats->dense_rounds = (int32_t)ctrl.dense_rounds;
        stats->dense_launches = dense_launches;
        stats->dense_ms = dense_ms;
        stats->dense_changes = (int64_t)ctrl.dense_changes;
        if (p.profile && kinds) {
            /* dense rounds: mean slice time per warp, mean slowest slice per
             * round, mean round-to-round time */
            const double dr = (double)(ctrl.dense_rounds ? ctrl.dense_rounds : 1);
            stats->phase_light_ns = ctrl.t_light / ((double)dgrid * 16 * dr);
            stats->phase_heavy_ns = ctrl.t_heavy / dr;
            stats->phase_wait_ns = ctrl.t_wait / (dr > 1 ? dr - 1 : 1);
        } else if (p.profile) {
            /* average per warp and round, in nanoseconds */
            const double wr = (double)grid * (block / 32) * (double)(ctrl.rounds ? ctrl.rounds : 1);
            stats->phase_heavy_ns = ctrl.t_heavy / wr;
            stats->phase_light_ns = ctrl.t_light / wr;
            stats->phase_wait_ns = ctrl.t_wait / wr;
        }
    }
    if (ctrl.stop == EG_ERR_LOOPCAP)
        return eg_set_error(EG_ERR_LOOPCAP, "round cap %lld reached with work left", (long long)opts->max_rounds);
    if (ctrl.stop == EG_ERR_CANCELLED) return eg_set_error(EG_ERR_CANCELLED, "solve cancelled");
    if (ctrl.stop == EG_ERR_TIMEOUT) {
        if (ctrl.abort)
            return eg_set_error(EG_ERR_TIMEOUT, "a grid barrier wait ran out after round %llu", ctrl.wait_site);
        return eg_set_error(EG_ERR_TIMEOUT, "timeout of %.1f ms expired", opts->timeout_ms);
    }
    if (ctrl.stop) return eg_set_error((eg_status)ctrl.stop, "solve stopped with status %d", ctrl.stop);
    return EG_OK;
}

template <class O>
static eg_status dgame_credits(eg_dgame *g, O *host, int obits)
{
    if (!g || !host) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    if (!g->solved) return eg_set_error(EG_ERR_INVALID, "the game has no solved credits");
    EG_CUDA(cudaSetDevice(g->device));
    if (obits == 32 && g->solved_bits == 64 && g->mg > (long long)INT32_MAX)
        return eg_set_error(EG_ERR_OVERFLOW, "credits do not fit 32 bits (MG = %lld)", g->mg);
    launch_gather_out(g->solved_bits, obits, g->n, g->d_iperm, g->d_F, g->d_out, g->st);
    EG_CUDA(cudaMemcpyAsync(host, g->d_out, sizeof(O) * (size_t)g->n, cudaMemcpyDeviceToHost, g->st));
    EG_CUDA(cudaStreamSynchronize(g->st));
    return EG_OK;
}

extern "C" eg_status eg_dgame_credits_i32(eg_dgame *g, int32_t *credits) { return dgame_credits<int32_t>(g, credits, 32); }
extern "C" eg_status eg_dgame_credits_i64(eg_dgame *g, int64_t *credits) { return dgame_credits<int64_t>(g, credits, 64); }

extern "C" eg_status eg_dgame_credits_device(eg_dgame *g, void **dev_ptr, int32_t *credit_bits)
{
    if (!g || !dev_ptr) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    if (!g->solved) return eg_set_error(EG_ERR_INVALID, "the game has no solved credits");
    EG_CUDA(cudaSetDevice(g->device));
    launch_gather_out(g->solved_bits, g->solved_bits, g->n, g->d_iperm, g->d_F, g->d_out, g->st);
    EG_CUDA(cudaStreamSynchronize(g->st));
    *dev_ptr = g->d_out;
    if (credit_bits) *credit_bits = g->solved_bits;
    return EG_OK;
}

/* ------------------------------------------------------------------ */
/* One-call solve                                                       */
/* ------------------------------------------------------------------ */

template <class O>
static eg_status solve_once(const eg_game *game, const eg_opts *opts, O *credits, eg_stats *stats, int obits)
{
    if (!credits) return eg_set_error(EG_ERR_INVALID, "credits is NULL");
    eg_opts o;
    if (opts) o = *opts;
    else eg_opts_default(&o);
    if (o.credit_bits == 0) o.credit_bits = obits;
    if (obits == 32 && o.credit_bits == 64) o.credit_bits = 64; /* solve wide, narrow on output */
    eg_dgame *g = nullptr;
    EG_TRY(eg_dgame_upload(game, &o, &g));
    eg_status s = eg_dgame_solve(g, &o, stats);
    if (s == EG_OK || s == EG_ERR_LOOPCAP || s == EG_ERR_TIMEOUT || s == EG_ERR_CANCELLED) {
        char msg[512];
        snprintf(msg, sizeof msg, "%s", eg_last_error());
        eg_status s2 = dgame_credits<O>(g, credits, obits);
        if (s2 != EG_OK) s = s2;
        else if (s != EG_OK) eg_set_error(s, "%s", msg);
    }
    eg_dgame_free(g);
    return s;
}

extern "C" eg_status eg_solve_i32(const eg_game *game, const eg_opts *opts, int32_t *credits, eg_stats *stats)
{
    return solve_once<int32_t>(game, opts, credits, stats, 32);
}

extern "C" eg_status eg_solve_i64(const eg_game *game, const eg_opts *opts, int64_t *credits, eg_stats *stats)
{
    return solve_once<int64_t>(game, opts, credits, stats, 64);
}

/* ------------------------------------------------------------------ */
/* Standalone transpose                                                 */
/* ------------------------------------------------------------------ */

extern "C" eg_status eg_csr2csc_i32(int32_t num_rows, int32_t num_cols, int64_t nnz, const int64_t *row_ptr,
                                   const int32_t *col_idx, const int32_t *val, int64_t *csc_ptr, int32_t *csc_row,
                                   int32_t *csc_val)
{
    if (num_rows < 0 || num_cols < 0 || nnz < 0 || nnz > (int64_t)INT32_MAX - 64)
        return eg_set_error(EG_ERR_INVALID, "sizes out of range");
    if (!row_ptr || !csc_ptr || (nnz && (!col_idx || !val || !csc_row || !csc_val)))
        return eg_set_error(EG_ERR_INVALID, "NULL array");
    if (row_ptr[0] != 0 || row_ptr[num_rows] != nnz)
        return eg_set_error(EG_ERR_INVALID, "row_ptr must start at 0 and end at nnz");
    for (int32_t r = 0; r < num_rows; r++)
        if (row_ptr[r + 1] < row_ptr[r]) return eg_set_error(EG_ERR_INVALID, "row_ptr not monotone at row %d", r);
    for (int64_t j = 0; j < nnz; j++)
        if (col_idx[j] < 0 || col_idx[j] >= num_cols)
            return eg_set_error(EG_ERR_INVALID, "column %d of entry %lld out of range", col_idx[j], (long long)j);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return eg_set_error(EG_ERR_NO_DEVICE, "no CUDA device available");
    }
    cudaStream_t st;
    EG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const long long cap = std::max<long long>(nnz, 1);
    long long *d_rp = nullptr, *d_cp64 = nullptr;
    int *d_col = nullptr, *d_val = nullptr, *d_k0 = nullptr, *d_v0 = nullptr, *d_k1 = nullptr, *d_v1 = nullptr;
    int *d_rows = nullptr, *d_cnt = nullptr, *d_orow = nullptr, *d_oval = nullptr, *d_scr = nullptr;
    const long long scr = radix_scratch_ints(cap) + scan_scratch_ints((long long)num_cols + 1) + 64;
    cudaError_t e = cudaSuccess;
#define EG_MALLOC(p, n) \
    if (e == cudaSuccess) e = cudaMalloc((void **)&p, sizeof(*p) * (size_t)(n))
    EG_MALLOC(d_rp, (long long)num_rows + 1);
    EG_MALLOC(d_col, cap);
    EG_MALLOC(d_val, cap);
    EG_MALLOC(d_k0, cap);
    EG_MALLOC(d_v0, cap);
    EG_MALLOC(d_k1, cap);
    EG_MALLOC(d_v1, cap);
    EG_MALLOC(d_rows, cap);
    EG_MALLOC(d_orow, cap);
    EG_MALLOC(d_oval, cap);
    EG_MALLOC(d_cnt, (long long)num_cols + 1);
    EG_MALLOC(d_cp64, (long long)num_cols + 1);
    EG_MALLOC(d_scr, scr);
#undef EG_MALLOC
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rp, row_ptr, sizeof(long long) * ((size_t)num_rows + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(d_col, col_idx, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(d_val, val, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_cnt, 0, sizeof(int) * ((size_t)num_cols + 1), st);
    if (e == cudaSuccess) {
        const unsigned gw = grid_for((long long)num_rows * 32, 256);
        k_csr_expand<<<gw, 256, 0, st>>>(num_rows, d_rp, d_col, d_k0, d_v0, d_cnt);
        k_edge_rows<<<gw, 256, 0, st>>>(num_rows, d_rp, d_rows);
        excl_scan(d_cnt, (long long)num_cols + 1, d_scr, st);
        int *sk, *sv;
        radix_sort_pairs(d_k0, d_v0, d_k1, d_v1, nnz, bits_for(num_cols), d_scr, st, &sk, &sv);
        k_csc_gather<<<grid_for(nnz, 256), 256, 0, st>>>(nnz, sv, d_rows, d_val, d_orow, d_oval);
        k_widen<<<grid_for((long long)num_cols + 1, 256), 256, 0, st>>>((long long)num_cols + 1, d_cnt, d_cp64);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(csc_ptr, d_cp64, sizeof(long long) * ((size_t)num_cols + 1), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(csc_row, d_orow, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && nnz) e = cudaMemcpyAsync(csc_val, d_oval, sizeof(int) * (size_t)nnz, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    void *ptrs[] = {d_rp, d_cp64, d_col, d_val, d_k0, d_v0, d_k1, d_v1, d_rows, d_cnt, d_orow, d_oval, d_scr};
    for (void *ptr : ptrs)
        if (ptr) cudaFree(ptr);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return eg_set_error(e == cudaErrorMemoryAllocation ? EG_ERR_OOM : EG_ERR_CUDA, "transpose failed: %s",
                            cudaGetErrorString(e));
    }
    return EG_OK;
}

/* ------------------------------------------------------------------ */
/* Cancel flags                                                         */
/* ------------------------------------------------------------------ */

extern "C" eg_status eg_cancel_flag_alloc(volatile int32_t **flag)
{
    if (!flag) return eg_set_error(EG_ERR_INVALID, "flag is NULL");
    void *p = nullptr;
    EG_CUDA(cudaHostAlloc(&p, 64, cudaHostAllocMapped | cudaHostAllocPortable));
    memset(p, 0, 64);
    *flag = (volatile int32_t *)p;
    return EG_OK;
}

extern "C" void eg_cancel_flag_free(volatile int32_t *flag)
{
    if (flag) cudaFreeHost((void *)flag);
}

/* ------------------------------------------------------------------ */
/* Autotuner of the single-game layout                                  */
/* ------------------------------------------------------------------ */

namespace {

/* Shape of a game for the tuner's cache: log2 of n and of the mean
 * out-degree, and the share (in 1/16) of vertices in each log2 out-degree
 * bucket. */
std::string shape_key(const std::vector<long long> &rp, int n, long long m)
{
    int hist[32] = {0};
    for (int v = 0; v < n; v++) {
        const long long d = rp[(size_t)v + 1] - rp[(size_t)v];
        int b = 0;
        while (b < 31 && (1LL << (b + 1)) <= d) b++;
        hist[b]++;
    }
    std::string key = std::to_string(bits_for(n)) + "/" + std::to_string(bits_for(m / std::max(1, n))) + ":";
    for (int b = 0; b < 32; b++) key += std::to_string((hist[b] * 16 + n / 2) / std::max(1, n)) + ",";
    return key;
}

std::mutex g_tune_mu;
std::map<std::string, eg_opts> g_tune_cache;

}  // namespace

extern "C" eg_status eg_dgame_tune(eg_dgame *g, const eg_opts *base_in, int64_t rounds, eg_opts *tuned,
                                   eg_tune_report *rep)
{
    if (!g || !tuned) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    if (rounds < 1) return eg_set_error(EG_ERR_INVALID, "rounds must be >= 1");
    eg_opts base;
    if (base_in) base = *base_in;
    else eg_opts_default(&base);
    EG_TRY(check_lanes(&base));
    if (base.variant != EG_VARIANT_AUTO) return eg_set_error(EG_ERR_INVALID, "the tuner tunes the AUTO layout");
    EG_CUDA(cudaSetDevice(g->device));
    std::vector<long long> rp((size_t)g->n + 1);
    EG_CUDA(cudaMemcpy(rp.data(), g->d_rowptr, sizeof(long long) * rp.size(), cudaMemcpyDeviceToHost));
    const std::string key = shape_key(rp, g->n, g->m) + "|" + std::to_string(base.credit_bits) + "|" +
                            std::to_string(base.narrow);
    eg_tune_report r;
    memset(&r, 0, sizeof r);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            eg_opts t = base;
            const eg_opts &c = it->second;
            t.large_min_deg = c.large_min_deg;
            t.small_max_deg = c.small_max_deg;
            t.task_edges = c.task_edges;
            t.dense_sweeps = c.dense_sweeps;
            t.dense_depth = c.dense_depth;
            *tuned = t;
            r.from_cache = 1;
            if (rep) *rep = r;
            return EG_OK;
        }
    }
    /* coordinate descent: one knob at a time, each candidate a capped solve
     * from f = 0; the rate is edge relaxations per ms of the lifting loop */
    auto rate_of = [&](const eg_opts &o, double *rate) -> eg_status {
        eg_opts t = o;
        t.keep_layout = 0;
        t.max_rounds = rounds;
        t.profile = 0;
        eg_stats st;
        eg_status s = eg_dgame_solve(g, &t, &st);
        if (s != EG_OK && s != EG_ERR_LOOPCAP) return s;
        *rate = st.lift_ms > 0 ? (double)st.edges / st.lift_ms : 0.0;
        r.candidates++;
        return EG_OK;
    };
    eg_opts cur = base;
    /* the defaults spelled out, so that a knob's default is not timed twice */
    if (cur.large_min_deg <= 1) cur.large_min_deg = 17;
    if (cur.task_edges <= 0) cur.task_edges = 2 * kTaskPairs;
    if (cur.dense_sweeps <= 0) cur.dense_sweeps = kMaxDenseSweeps;
    if (cur.dense_depth <= 0) cur.dense_depth = 2;
    double best = 0.0;
    EG_TRY(rate_of(cur, &best));
    r.default_rate = best;
    struct Knob {
        int32_t eg_opts::*field;
        std::vector<int32_t> values;
    };
    const Knob knobs[] = {
        {&eg_opts::large_min_deg, {9, 17, 33, 65, 129}},   /* light / heavy bound        */
        {&eg_opts::task_edges, {64, 128, 256}},            /* edges per heavy task       */
        {&eg_opts::small_max_deg, {0, 2, 4}},              /* thread-per-vertex bucket   */
        {&eg_opts::dense_sweeps, {1, 2, 3, 4}},            /* sweeps per dense round     */
        {&eg_opts::dense_depth, {1, 2}},                   /* chunks in flight per warp  */
    };
    for (const Knob &k : knobs) {
        for (int32_t v : k.values) {
            if (cur.*(k.field) == v) continue;
            eg_opts cand = cur;
            cand.*(k.field) = v;
            double rate = 0.0;
            EG_TRY(rate_of(cand, &rate));
            if (rate > best * 1.02) { /* a clear win only: timings have noise */
                best = rate;
                cur = cand;
            }
        }
    }
    r.best_rate = best;
    cur.max_rounds = base.max_rounds;
    cur.keep_layout = 0;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = cur;
    }
    *tuned = cur;
    if (rep) *rep = r;
    return EG_OK;
}
