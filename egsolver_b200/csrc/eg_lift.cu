/*
 * eg_lift.cu -- the persistent lifting kernel.
 *
 * One cooperative launch runs the whole least-fixed-point iteration.  Each
 * round lifts every vertex of the current frontier bitmap and pushes the
 * predecessors of every vertex whose credit rose into the next bitmap; a
 * bounded grid barrier separates rounds, and the barrier's last arriver
 * decides termination on the device (frontier empty, round cap, timeout or
 * cancel), so there is no host round-trip per iteration.  This replaces the
 * reference's host loop of kernel launch + thrust::remove + cudaMemset per
 * half-iteration (reference src/dev_EG_alg.cu:307-381 and its K-lane
 * variants, src/thrust_wrapper.cu:30-42).
 *
 * The lift of one vertex u is the reference kernel body
 * (reference src/dev_EG_alg.cu:84-109): temp = min (player 0) or max
 * (player 1) over successors w of OMINUS(f(w), wt); if f(u) < temp then
 * f(u) = temp and every CSC predecessor is pushed.  The frontier bitmap
 * replaces the reference's atomicCAS(flags, 0, p+1) dedup.
 *
 * Variants (per class of the renumbered id space, all with 128-bit loads of
 * {succ, w, succ, w} edge pairs):
 *   group 1       thread-per-vertex            (reference --shuffling 1)
 *   group 2..32   G lanes per vertex, xor-shuffle min/max reduction
 *                 (reference --shuffling G, src/dev_EG_alg.cu:397-1480)
 *   CTA           all threads of the CTA per vertex, for high out-degree
 *
 * Credits are read with ld.global.cg: other SMs write them during the
 * kernel, and an L1 line kept across a barrier would be stale.  Reads that
 * race with a concurrent lift see the old or the new value; both are below
 * the least fixed point and a vertex whose successor rose is pushed again,
 * so the schedule stays a fair chaotic iteration and the result is exact.
 */
#include "eg_lift.cuh"

namespace eg {

constexpr int LIFT_BLOCK = 512;

template <int OWNER, class T>
__device__ __forceinline__ T combine(T a, T b)
{
    return OWNER ? (a > b ? a : b) : (a < b ? a : b);
}

template <int OWNER, class T>
__device__ __forceinline__ T identity()
{
    return OWNER ? (T)0 : credit_traits<T>::top;
}

template <class T>
__device__ __forceinline__ T shfl_xor(unsigned mask, T v, int off, int width)
{
    return __shfl_xor_sync(mask, v, off, width);
}
template <>
__device__ __forceinline__ int64_t shfl_xor<int64_t>(unsigned mask, int64_t v, int off, int width)
{
    return (int64_t)__shfl_xor_sync(mask, (long long)v, off, width);
}

template <class T>
__device__ __forceinline__ T shfl_idx(unsigned mask, T v, int src, int width)
{
    return __shfl_sync(mask, v, src, width);
}
template <>
__device__ __forceinline__ int64_t shfl_idx<int64_t>(unsigned mask, int64_t v, int src, int width)
{
    return (int64_t)__shfl_sync(mask, (long long)v, src, width);
}

/* Position of the k-th (0-based) set bit of w; requires popc(w) > k. */
__device__ __forceinline__ int nth_set_bit(uint32_t w, int k)
{
    int pos = 0;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const uint32_t low = w & ((1u << s) - 1u);
        const int c = __popc(low);
        if (k >= c) {
            k -= c;
            w >>= s;
            pos += s;
        } else {
            w = low;
        }
    }
    return pos;
}

/* Where pushes go and how credits are read: the persistent grid kernel
 * marks a global bitmap and reads credits from L2; the single-CTA kernel
 * owns its game, marks a shared-memory bitmap and may cache credits in L1. */
struct GridPolicy {
    uint32_t *bm;
    __device__ __forceinline__ void push(int32_t p) const { bitmap_mark(bm, p); }
    template <class T> __device__ __forceinline__ T load(const T *a) const { return ld_credit(a); }
    template <class T> __device__ __forceinline__ void store(T *a, T v) const { st_credit(a, v); }
};
struct CtaPolicy {
    uint32_t *bm; /* shared memory */
    __device__ __forceinline__ void push(int32_t p) const { atomicOr(bm + (p >> 5), 1u << (p & 31)); }
    template <class T> __device__ __forceinline__ T load(const T *a) const { return *a; }
    template <class T> __device__ __forceinline__ void store(T *a, T v) const { *a = v; }
};

struct LiftCounters {
    unsigned long long lifts, edges;
    unsigned changes, pushes;
    int any_new;
};

/* Lift vertex u with the G lanes of one group (gl = lane in group). */
template <class T, int G, int OWNER, class Pol>
__device__ __forceinline__ void lift_group(const LiftParams &p, T *F, const Pol &pol, int u, int gl, unsigned gmask,
                                           LiftCounters &cnt)
{
    const int b = __ldg(p.P + u) >> 1, e = __ldg(p.P + u + 1) >> 1;
    /* Only the group leader reads the old credit, before the reduction (a
     * group-wide synchronisation point) and so before its own write below:
     * a lane that read F[u] after the leader's write would see no change and
     * skip its share of the predecessor pushes. */
    T old = (gl == 0) ? pol.load(F + u) : (T)0;
    T acc = identity<OWNER, T>();
    int real = 0;
    for (int k = b + gl; k < e; k += G) {
        const int4 q = __ldg(p.E4 + k);
        const T v0 = ominus<T>(pol.load(F + q.x), q.y, p.mg);
        const T v1 = ominus<T>(pol.load(F + q.z), q.w, p.mg);
        acc = combine<OWNER>(acc, combine<OWNER>(v0, v1));
        real += 1 + (q.z < p.n_pad);
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) acc = combine<OWNER>(acc, shfl_xor<T>(gmask, acc, off, G));
    if (G > 1) old = shfl_idx<T>(gmask, old, 0, G);
    cnt.edges += (unsigned long long)real;
    if (old < acc) {
        if (gl == 0) {
            pol.store(F + u, acc);
            cnt.changes++;
        }
        const int cb = __ldg(p.CP + u), ce = __ldg(p.CP + u + 1);
        if (gl == 0) cnt.pushes += (unsigned)(ce - cb);
        cnt.any_new |= ce > cb;
#pragma unroll 4
        for (int k = cb + gl; k < ce; k += G) pol.push(__ldg(p.CS + k));
    }
    if (gl == 0) cnt.lifts++;
}

/* Warp-level processing of a class with G lanes per vertex: warps grab
 * frontier words dynamically; within a word, group g takes the g-th set bit. */
template <class T, int G, int OWNER>
__device__ __noinline__ void warp_class(const LiftParams &p, const LiftClass &lc, T *F, uint32_t *cur, uint32_t *nxt,
                                        int *ctr, LiftCounters &cnt)
{
    const int lane = threadIdx.x & 31;
    const int nwords = lc.word_end - lc.word_begin;
    constexpr int NG = 32 / G;
    const int grp = lane / G, gl = lane % G;
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (grp * G));
    const GridPolicy pol{nxt};
    for (;;) {
        int w0 = 0;
        if (lane == 0) w0 = atomicAdd(ctr, lc.grab);
        w0 = __shfl_sync(0xffffffffu, w0, 0);
        if (w0 >= nwords) break;
        const int w1 = min(w0 + lc.grab, nwords);
        for (int wi = w0; wi < w1; wi++) {
            const int gw = lc.word_begin + wi;
            uint32_t word = 0;
            if (lane == 0) {
                word = __ldcg(cur + gw);
                if (word) __stcg(cur + gw, 0u);
            }
            word = __shfl_sync(0xffffffffu, word, 0);
            const int base_u = gw << 5;
            if (G == 1) {
                if ((word >> lane) & 1u) lift_group<T, 1, OWNER>(p, F, pol, base_u + lane, 0, 0u, cnt);
            } else {
                while (word) {
                    const int c = __popc(word);
                    if (grp < c) lift_group<T, G, OWNER>(p, F, pol, base_u + nth_set_bit(word, grp), gl, gmask, cnt);
                    if (c <= NG) {
                        word = 0;
                    } else {
                        const int last = nth_set_bit(word, NG - 1);
                        word &= ~((2u << last) - 1u);
                    }
                }
            }
        }
    }
}

/* Thread-per-vertex processing with memory-level parallelism: a warp takes
 * U consecutive frontier words at a time (static assignment over the grid,
 * so no counter is touched) and every lane carries the U vertices it owns in
 * those words through each load phase together. */
template <class T, int OWNER>
__device__ __noinline__ void thread_class(const LiftParams &p, const LiftClass &lc, T *F, uint32_t *cur, uint32_t *nxt,
                                          LiftCounters &cnt)
{
    constexpr int U = 4;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    const int nwords = lc.word_end - lc.word_begin;
    /* every warp gets the same number of words (+-1) of this class */
    const int lo = (int)((long long)gwarp * nwords / nwarp), hi = (int)((long long)(gwarp + 1) * nwords / nwarp);
    for (int w0 = lo; w0 < hi; w0 += U) {
        uint32_t mine = 0;
        if (lane < U && w0 + lane < hi) {
            uint32_t *wp = cur + lc.word_begin + w0 + lane;
            mine = __ldcg(wp);
            if (mine) __stcg(wp, 0u);
        }
        int u[U], b[U], e[U];
        T old[U], acc[U];
#pragma unroll
        for (int j = 0; j < U; j++) {
            const uint32_t wj = __shfl_sync(0xffffffffu, mine, j);
            u[j] = ((lc.word_begin + w0 + j) << 5) + lane;
            acc[j] = identity<OWNER, T>();
            b[j] = e[j] = 0;
            old[j] = 0;
            if ((wj >> lane) & 1u) {
                b[j] = __ldg(p.P + u[j]) >> 1;
                e[j] = __ldg(p.P + u[j] + 1) >> 1;
                old[j] = ld_credit(F + u[j]);
            }
        }
        int real = 0;
        for (int k = 0;; k++) {
            bool more = false;
#pragma unroll
            for (int j = 0; j < U; j++) {
                if (b[j] + k < e[j]) {
                    const int4 q = __ldg(p.E4 + b[j] + k);
                    const T v0 = ominus<T>(ld_credit(F + q.x), q.y, p.mg);
                    const T v1 = ominus<T>(ld_credit(F + q.z), q.w, p.mg);
                    acc[j] = combine<OWNER>(acc[j], combine<OWNER>(v0, v1));
                    real += 1 + (q.z < p.n_pad);
                    more = true;
                }
            }
            if (!more) break;
        }
        cnt.edges += (unsigned long long)real;
#pragma unroll
        for (int j = 0; j < U; j++) {
            if (e[j] > b[j]) {
                cnt.lifts++;
                if (old[j] < acc[j]) {
                    st_credit(F + u[j], acc[j]);
                    cnt.changes++;
                    const int cb = __ldg(p.CP + u[j]), ce = __ldg(p.CP + u[j] + 1);
                    cnt.pushes += (unsigned)(ce - cb);
                    cnt.any_new |= ce > cb;
#pragma unroll 4
                    for (int k = cb; k < ce; k++) bitmap_mark(nxt, __ldg(p.CS + k));
                }
            }
        }
    }
}

template <int OWNER>
__device__ __forceinline__ void atomic_combine(int32_t *a, int32_t v)
{
    if (OWNER) atomicMax(a, v);
    else atomicMin(a, v);
}
template <int OWNER>
__device__ __forceinline__ void atomic_combine(int64_t *a, int64_t v)
{
    if (OWNER) atomicMax((long long *)a, (long long)v);
    else atomicMin((long long *)a, (long long)v);
}
__device__ __forceinline__ int32_t atomic_swap(int32_t *a, int32_t v) { return atomicExch(a, v); }
__device__ __forceinline__ int64_t atomic_swap(int64_t *a, int64_t v)
{
    return (int64_t)atomicExch((unsigned long long *)a, (unsigned long long)v);
}

/* The last step of a heavy vertex's lift (one warp): compare with the old
 * credit, raise it, clear the vertex's frontier bit, push predecessors. */
template <class T>
__device__ __forceinline__ void heavy_finalize(const LiftParams &p, T *F, uint32_t *cur, uint32_t *nxt, int u, T v,
                                               int lane, LiftCounters &cnt)
{
    int raise = 0;
    if (lane == 0) {
        const T old = ld_credit(F + u);
        raise = old < v;
        if (raise) {
            st_credit(F + u, v);
            cnt.changes++;
        }
        atomicAnd(cur + (u >> 5), ~(1u << (u & 31)));
        cnt.lifts++;
    }
    raise = __shfl_sync(0xffffffffu, raise, 0);
    if (raise) {
        const int cb = __ldg(p.CP + u), ce = __ldg(p.CP + u + 1);
        if (lane == 0) cnt.pushes += (unsigned)(ce - cb);
        cnt.any_new |= ce > cb;
        for (int k = cb + lane; k < ce; k += 32) bitmap_mark(nxt, __ldg(p.CS + k));
    }
}

/* One task of a heavy vertex: up to kTaskPairs edge pairs, a warp-wide
 * min/max; a vertex cut into several tasks combines the partial results
 * with an atomic min/max, and the task that reports last finalizes. */
template <class T, int OWNER>
__device__ __forceinline__ void heavy_task(const LiftParams &p, T *F, uint32_t *cur, uint32_t *nxt, const int4 tk,
                                           int lane, LiftCounters &cnt)
{
    T acc = identity<OWNER, T>();
    int real = 0;
#pragma unroll 4
    for (int k = tk.y + lane; k < tk.z; k += 32) {
        const int4 q = __ldg(p.E4 + k);
        const T v0 = ominus<T>(ld_credit(F + q.x), q.y, p.mg);
        const T v1 = ominus<T>(ld_credit(F + q.z), q.w, p.mg);
        acc = combine<OWNER>(acc, combine<OWNER>(v0, v1));
        real += 1 + (q.z < p.n_pad);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc = combine<OWNER>(acc, shfl_xor<T>(0xffffffffu, acc, off, 32));
    cnt.edges += (unsigned long long)real;
    const int u = tk.x, nt = tk.w >> 1;
    if (nt == 1) {
        heavy_finalize<T>(p, F, cur, nxt, u, acc, lane, cnt);
        return;
    }
    const int h = u - p.heavy_begin;
    T *hacc = (T *)p.hacc;
    int last = 0;
    if (lane == 0) {
        atomic_combine<OWNER>(hacc + h, acc);
        __threadfence();
        last = atomicSub(p.hrem + h, 1) == 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    T v = (T)0;
    if (lane == 0) {
        __threadfence();
        v = atomic_swap(hacc + h, identity<OWNER, T>());
        p.hrem[h] = nt; /* ready for the next round */
    }
    v = shfl_idx<T>(0xffffffffu, v, 0, 32);
    heavy_finalize<T>(p, F, cur, nxt, u, v, lane, cnt);
}

/* Heavy vertices: their edge tasks are dealt round-robin to all warps of
 * the grid (balanced without any counter); a task of an inactive vertex
 * costs one bitmap read. */
template <class T>
__device__ __noinline__ void heavy_tasks(const LiftParams &p, T *F, uint32_t *cur, uint32_t *nxt, LiftCounters &cnt)
{
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    for (int t = gwarp; t < p.num_tasks; t += nwarp) {
        const int4 tk = __ldg(p.tasks + t);
        const uint32_t w = __ldcg(cur + (tk.x >> 5));
        if (!((w >> (tk.x & 31)) & 1u)) continue;
        if (tk.w & 1) heavy_task<T, 1>(p, F, cur, nxt, tk, lane, cnt);
        else heavy_task<T, 0>(p, F, cur, nxt, tk, lane, cnt);
    }
}

/* CTA-level processing: the whole CTA lifts one vertex at a time. */
template <class T, int OWNER>
__device__ __noinline__ void cta_class(const LiftParams &p, const LiftClass &lc, T *F, uint32_t *cur, uint32_t *nxt,
                                       int *ctr, LiftCounters &cnt)
{
    __shared__ int s_w;
    __shared__ uint32_t s_word;
    __shared__ T s_red[LIFT_BLOCK / 32];
    __shared__ int s_raise;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nwords = lc.word_end - lc.word_begin;
    for (;;) {
        if (threadIdx.x == 0) {
            const int w = atomicAdd(ctr, 1);
            uint32_t word = 0;
            if (w < nwords) {
                word = __ldcg(cur + lc.word_begin + w);
                if (word) __stcg(cur + lc.word_begin + w, 0u);
            }
            s_w = w;
            s_word = word;
        }
        __syncthreads();
        const int w = s_w;
        uint32_t word = s_word;
        __syncthreads();
        if (w >= nwords) break;
        while (word) {
            const int bit = __ffs(word) - 1;
            word &= word - 1u;
            const int u = ((lc.word_begin + w) << 5) + bit;
            const int b = __ldg(p.P + u) >> 1, e = __ldg(p.P + u + 1) >> 1;
            T acc = identity<OWNER, T>();
            int real = 0;
            for (int k = b + threadIdx.x; k < e; k += LIFT_BLOCK) {
                const int4 q = __ldg(p.E4 + k);
                const T v0 = ominus<T>(ld_credit(F + q.x), q.y, p.mg);
                const T v1 = ominus<T>(ld_credit(F + q.z), q.w, p.mg);
                acc = combine<OWNER>(acc, combine<OWNER>(v0, v1));
                real += 1 + (q.z < p.n_pad);
            }
            cnt.edges += (unsigned long long)real;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc = combine<OWNER>(acc, shfl_xor<T>(0xffffffffu, acc, off, 32));
            if (lane == 0) s_red[wid] = acc;
            __syncthreads();
            if (wid == 0) {
                T x = lane < LIFT_BLOCK / 32 ? s_red[lane] : identity<OWNER, T>();
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) x = combine<OWNER>(x, shfl_xor<T>(0xffffffffu, x, off, 32));
                if (lane == 0) {
                    /* one thread reads, compares and writes, so that no thread
                     * can read the credit after it was raised */
                    const T old = ld_credit(F + u);
                    const int raise = old < x;
                    if (raise) st_credit(F + u, x);
                    s_raise = raise;
                }
            }
            __syncthreads();
            if (s_raise) {
                const int cb = __ldg(p.CP + u), ce = __ldg(p.CP + u + 1);
                if (threadIdx.x == 0) {
                    cnt.changes++;
                    cnt.pushes += (unsigned)(ce - cb);
                }
                cnt.any_new |= ce > cb;
                for (int k = cb + threadIdx.x; k < ce; k += LIFT_BLOCK) bitmap_mark(nxt, __ldg(p.CS + k));
            }
            if (threadIdx.x == 0) cnt.lifts++;
            __syncthreads();
        }
    }
}

template <class T, int OWNER>
__device__ __forceinline__ void run_class(const LiftParams &p, const LiftClass &lc, T *F, uint32_t *cur, uint32_t *nxt,
                                          int *ctr, LiftCounters &cnt)
{
    switch (lc.group) {
    case EG_GROUP_CTA: cta_class<T, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case 1: thread_class<T, OWNER>(p, lc, F, cur, nxt, cnt); break;
    case 2: warp_class<T, 2, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case 4: warp_class<T, 4, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case 8: warp_class<T, 8, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case 16: warp_class<T, 16, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    default: warp_class<T, 32, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    }
}

template <class T>
__global__ void __launch_bounds__(LIFT_BLOCK, 2) k_lift(const __grid_constant__ LiftParams p)
{
    Ctrl *c = p.ctrl;
    T *F = (T *)p.F;
    LiftCounters cnt = {0ull, 0ull, 0u, 0u, 0};
    if (blockIdx.x == 0 && threadIdx.x == 0) c->t_start = globaltimer_ns();
    for (long long round = 0;; round++) {
        uint32_t *cur = (round & 1) ? p.B1 : p.B0;
        uint32_t *nxt = (round & 1) ? p.B0 : p.B1;
        int *ctr = c->ctr[round & 1];
        cnt.any_new = 0;
        if (p.num_tasks) heavy_tasks<T>(p, F, cur, nxt, cnt);
        for (int ci = 0; ci < p.nclasses; ci++) {
            const LiftClass &lc = p.cls[ci];
            if (lc.owner) run_class<T, 1>(p, lc, F, cur, nxt, ctr + ci, cnt);
            else run_class<T, 0>(p, lc, F, cur, nxt, ctr + ci, cnt);
        }
        if (__syncthreads_or(cnt.any_new) && threadIdx.x == 0) c->flag[(round + 1) & 1] = 1;
        const bool ok = grid_barrier(c, p.wait_limit_ns, [&]() {
            /* last arriver of round `round`: clear this parity's counters
             * and flag, then decide whether the solve goes on */
            for (int ci = 0; ci < EG_MAX_CLASSES; ci++) c->ctr[round & 1][ci] = 0;
            c->flag[round & 1] = 0;
            c->rounds = round + 1;
            if (ld_volatile(&c->flag[(round + 1) & 1])) {
                if (p.max_rounds >= 0 && round + 1 >= p.max_rounds) {
                    c->stop = (int)EG_ERR_LOOPCAP;
                } else if (p.timeout_ns && globaltimer_ns() - c->t_start > p.timeout_ns) {
                    c->stop = (int)EG_ERR_TIMEOUT;
                } else if (p.cancel && (round & 63) == 0 && ld_volatile(p.cancel)) {
                    c->stop = (int)EG_ERR_CANCELLED;
                }
            }
        });
        if (!ok) break;
        if (ld_volatile(&c->stop)) break;
        if (!ld_volatile(&c->flag[(round + 1) & 1])) break;
    }
    /* statistics */
    unsigned long long l = cnt.lifts, e = cnt.edges, ch = cnt.changes, pu = cnt.pushes;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        l += __shfl_xor_sync(0xffffffffu, l, off);
        e += __shfl_xor_sync(0xffffffffu, e, off);
        ch += __shfl_xor_sync(0xffffffffu, ch, off);
        pu += __shfl_xor_sync(0xffffffffu, pu, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&c->lifts, l);
        atomicAdd(&c->edges, e);
        atomicAdd(&c->changes, ch);
        atomicAdd(&c->pushes, pu);
    }
}

/* One CTA of the shared-memory kernel: warps take words of a class from a
 * shared counter and serve them with G lanes per vertex (1, or 8 / 32 for
 * the larger buckets). */
template <class T, int G, int OWNER>
__device__ __forceinline__ void cta_warp_class(const LiftParams &p, const LiftClass &lc, T *F, uint32_t *cur,
                                               const CtaPolicy &pol, int *ctr, LiftCounters &cnt)
{
    const int lane = threadIdx.x & 31;
    constexpr int NG = 32 / G;
    const int grp = lane / G, gl = lane % G;
    const unsigned gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (grp * G));
    const int nwords = lc.word_end - lc.word_begin;
    for (;;) {
        int wi = 0;
        if (lane == 0) wi = atomicAdd(ctr, 1);
        wi = __shfl_sync(0xffffffffu, wi, 0);
        if (wi >= nwords) break;
        const int gw = lc.word_begin + wi;
        uint32_t word = cur[gw];
        __syncwarp();
        if (lane == 0 && word) cur[gw] = 0;
        const int base_u = gw << 5;
        if (G == 1) {
            if ((word >> lane) & 1u) lift_group<T, 1, OWNER>(p, F, pol, base_u + lane, 0, 0u, cnt);
            continue;
        }
        while (word) {
            const int c = __popc(word);
            if (grp < c) lift_group<T, G, OWNER>(p, F, pol, base_u + nth_set_bit(word, grp), gl, gmask, cnt);
            if (c <= NG) {
                word = 0;
            } else {
                const int last = nth_set_bit(word, NG - 1);
                word &= ~((2u << last) - 1u);
            }
        }
    }
}

/* A whole small game lifted by one CTA: both frontier bitmaps in shared
 * memory, rounds separated by __syncthreads, termination by
 * __syncthreads_or; no grid barrier and no spin-wait at all. */
template <class T>
__global__ void __launch_bounds__(1024, 1) k_lift_cta(const __grid_constant__ LiftParams p)
{
    extern __shared__ uint32_t sbits[];
    __shared__ int s_ctr[2][EG_MAX_CLASSES];
    const int words = p.n_pad >> 5;
    uint32_t *cur = sbits, *nxt = sbits + words;
    T *F = (T *)p.F;
    Ctrl *c = p.ctrl;
    LiftCounters cnt = {0ull, 0ull, 0u, 0u, 0};
    for (int w = threadIdx.x; w < words; w += blockDim.x) {
        cur[w] = p.B0[w];
        nxt[w] = 0;
    }
    if (threadIdx.x < 2 * EG_MAX_CLASSES) (&s_ctr[0][0])[threadIdx.x] = 0;
    const unsigned long long t0 = globaltimer_ns();
    __syncthreads();
    long long round = 0;
    int stop = 0;
    for (;;) {
        if (threadIdx.x < EG_MAX_CLASSES) s_ctr[(round + 1) & 1][threadIdx.x] = 0;
        cnt.any_new = 0;
        const CtaPolicy pol{nxt};
        for (int ci = 0; ci < p.nclasses; ci++) {
            const LiftClass &lc = p.cls[ci];
            int *ctr = &s_ctr[round & 1][ci];
            const int g = lc.group;
            if (lc.owner) {
                if (g == 1) cta_warp_class<T, 1, 1>(p, lc, F, cur, pol, ctr, cnt);
                else if (g == 8) cta_warp_class<T, 8, 1>(p, lc, F, cur, pol, ctr, cnt);
                else cta_warp_class<T, 32, 1>(p, lc, F, cur, pol, ctr, cnt);
            } else {
                if (g == 1) cta_warp_class<T, 1, 0>(p, lc, F, cur, pol, ctr, cnt);
                else if (g == 8) cta_warp_class<T, 8, 0>(p, lc, F, cur, pol, ctr, cnt);
                else cta_warp_class<T, 32, 0>(p, lc, F, cur, pol, ctr, cnt);
            }
        }
        round++;
        if (!__syncthreads_or(cnt.any_new)) break;
        if (p.max_rounds >= 0 && round >= p.max_rounds) {
            stop = EG_ERR_LOOPCAP;
            break;
        }
        const int late = __syncthreads_or(threadIdx.x == 0 && ((((round - 1) & 63) == 0 && p.cancel && ld_volatile(p.cancel)) ? 2 :
                                           (p.timeout_ns && globaltimer_ns() - t0 > p.timeout_ns) ? 1 : 0));
        if (late) {
            /* distinguish cancel from timeout with one more vote */
            const int was_cancel = __syncthreads_or(threadIdx.x == 0 && p.cancel && ld_volatile(p.cancel));
            stop = was_cancel ? EG_ERR_CANCELLED : EG_ERR_TIMEOUT;
            break;
        }
        uint32_t *t = cur;
        cur = nxt;
        nxt = t;
    }
    unsigned long long l = cnt.lifts, e = cnt.edges, ch = cnt.changes, pu = cnt.pushes;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        l += __shfl_xor_sync(0xffffffffu, l, off);
        e += __shfl_xor_sync(0xffffffffu, e, off);
        ch += __shfl_xor_sync(0xffffffffu, ch, off);
        pu += __shfl_xor_sync(0xffffffffu, pu, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&c->lifts, l);
        atomicAdd(&c->edges, e);
        atomicAdd(&c->changes, ch);
        atomicAdd(&c->pushes, pu);
    }
    if (threadIdx.x == 0) {
        c->rounds = round;
        c->stop = stop;
    }
}

eg_status launch_lift_cta(const LiftParams &p, int credit_bits, cudaStream_t st)
{
    const void *fn = credit_bits == 32 ? (const void *)k_lift_cta<int32_t> : (const void *)k_lift_cta<int64_t>;
    const size_t smem = (size_t)(p.n_pad / 32) * 2 * sizeof(uint32_t);
    cudaError_t err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess)
        return eg_set_error(EG_ERR_CUDA, "shared-memory kernel does not fit (%zu B): %s", smem, cudaGetErrorString(err));
    void *args[] = {(void *)&p};
    err = cudaLaunchKernel(fn, dim3(1), dim3(1024), args, smem, st);
    if (err != cudaSuccess)
        return eg_set_error(EG_ERR_CUDA, "launch of the shared-memory kernel failed: %s", cudaGetErrorString(err));
    return EG_OK;
}

eg_status launch_lift(const LiftParams &p, int credit_bits, cudaStream_t st, int *grid, int *block, int max_ctas)
{
    int dev = 0;
    cudaGetDevice(&dev);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void *fn = credit_bits == 32 ? (const void *)k_lift<int32_t> : (const void *)k_lift<int64_t>;
    int per_sm = 0;
    cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, LIFT_BLOCK, 0);
    if (err != cudaSuccess || per_sm < 1)
        return eg_set_error(EG_ERR_CUDA, "occupancy query for the lifting kernel failed: %s",
                            cudaGetErrorString(err));
    int g = sms * per_sm;
    if (max_ctas > 0 && max_ctas < g) g = max_ctas;
    void *args[] = {(void *)&p};
    err = cudaLaunchCooperativeKernel(fn, dim3(g), dim3(LIFT_BLOCK), args, 0, st);
    if (err != cudaSuccess)
        return eg_set_error(EG_ERR_CUDA, "cooperative launch of the lifting kernel failed: %s", cudaGetErrorString(err));
    *grid = g;
    *block = LIFT_BLOCK;
    return EG_OK;
}

}  // namespace eg
