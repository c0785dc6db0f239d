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
        const int cb = __ldg(p.CP + u) >> 2, ce = __ldg(p.CP + u + 1) >> 2;
        cnt.any_new |= ce > cb;
        for (int k = cb + gl; k < ce; k += G) cnt.pushes += push4(pol, __ldg((const int4 *)p.CS + k));
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
                                          int *ctr, LiftCounters &cnt)
{
    constexpr int U = 4;
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    const int nwords = lc.word_end - lc.word_begin;
    /* static: every warp gets the same number of words (+-1) of the class;
     * dynamic (grab < 0): warps take U words at a time in increasing order,
     * so later words see credits raised earlier in the same round */
    const bool dyn = lc.grab < 0;
    const int lo = dyn ? 0 : (int)((long long)gwarp * nwords / nwarp);
    const int hi = dyn ? nwords : (int)((long long)(gwarp + 1) * nwords / nwarp);
    for (int w0 = lo;; w0 += U) {
        if (dyn) {
            int t = 0;
            if (lane == 0) t = atomicAdd(ctr, U);
            w0 = __shfl_sync(0xffffffffu, t, 0);
        }
        if (w0 >= hi) break;
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
                    const int cb = __ldg(p.CP + u[j]) >> 2, ce = __ldg(p.CP + u[j] + 1) >> 2;
                    cnt.any_new |= ce > cb;
                    const GridPolicy pol{nxt};
                    for (int k = cb; k < ce; k++) cnt.pushes += push4(pol, __ldg((const int4 *)p.CS + k));
                }
            }
        }
    }
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
        const int cb = __ldg(p.CP + u) >> 2, ce = __ldg(p.CP + u + 1) >> 2;
        cnt.any_new |= ce > cb;
        const GridPolicy pol{nxt};
        for (int k = cb + lane; k < ce; k += 32) cnt.pushes += push4(pol, __ldg((const int4 *)p.CS + k));
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

/* Lane index of the last entry of a warp-wide exclusive scan `excl` whose
 * value is <= t (the owner of item t): binary search by shuffles.  Every
 * lane of the warp must call it. */
__device__ __forceinline__ int owner_of(int excl, int t)
{
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
        const int mid = lo + step;
        const int e = __shfl_sync(0xffffffffu, excl, mid & 31);
        if (mid < 32 && e <= t) lo = mid;
    }
    return lo;
}

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int *total)
{
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    *total = __shfl_sync(0xffffffffu, incl, 31);
    return incl - v;
}

/* The predecessor lists of the raised vertices of one word (lane j owns
 * vertex u of lane j), dealt to the 32 lanes and pushed four per 128-bit
 * load. */
template <class Pol>
__device__ __forceinline__ void push_raised(const LiftParams &p, const Pol &pol, int u, bool raise, int lane,
                                            LiftCounters &cnt)
{
    int cb = 0, nc = 0;
    if (raise) {
        cb = __ldg(p.CP + u) >> 2;
        nc = (__ldg(p.CP + u + 1) >> 2) - cb;
    }
    int ptotal;
    const int pexcl = warp_excl_scan(nc, lane, &ptotal);
    cnt.any_new |= ptotal > 0;
    for (int base = 0; base < ptotal; base += 32) {
        const int t = base + lane;
        const int own = owner_of(pexcl, t);
        const int ocb = __shfl_sync(0xffffffffu, cb, own);
        const int oex = __shfl_sync(0xffffffffu, pexcl, own);
        if (t < ptotal) cnt.pushes += push4(pol, __ldg((const int4 *)p.CS + ocb + (t - oex)));
    }
}

/* One frontier word of light vertices, warp-cooperative and edge-parallel:
 * lane j owns vertex j of the word; the word's edge pairs are dealt to the
 * 32 lanes, combined per vertex by a segmented shuffle reduction, and the
 * predecessor lists of the raised vertices are pushed the same way, four
 * per 128-bit load.  The dependent memory steps per word do not depend on
 * the vertices' degrees. */
template <class T, int OWNER, class Pol>
__device__ __forceinline__ void light_word(const LiftParams &p, T *F, const Pol &pol, int gw, uint32_t word, int lane,
                                           LiftCounters &cnt)
{
    const int u = (gw << 5) + lane;
    const bool act = (word >> lane) & 1u;
    int b = 0, np = 0;
    T old = (T)0;
    if (act) {
        b = __ldg(p.P + u) >> 1;
        np = (__ldg(p.P + u + 1) >> 1) - b;
        old = pol.load(F + u);
    }
    int total;
    const int excl = warp_excl_scan(np, lane, &total);
    T acc = identity<OWNER, T>();
    int real = 0;
    for (int base = 0; base < total; base += 32) {
        const int t = base + lane;
        const int own = owner_of(excl, t);
        const int ob = __shfl_sync(0xffffffffu, b, own);
        const int oe = __shfl_sync(0xffffffffu, excl, own);
        T val = identity<OWNER, T>();
        if (t < total) {
            const int4 q = __ldg(p.E4 + ob + (t - oe));
            const T v0 = ominus<T>(pol.load(F + q.x), q.y, p.mg);
            const T v1 = ominus<T>(pol.load(F + q.z), q.w, p.mg);
            val = combine<OWNER>(v0, v1);
            real += 1 + (q.z < p.n_pad);
        }
        /* segmented inclusive min / max over runs of equal owner */
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const T other = shfl_idx<T>(0xffffffffu, val, (lane - o) & 31, 32);
            const int oo = __shfl_sync(0xffffffffu, own, (lane - o) & 31);
            if (lane >= o && oo == own) val = combine<OWNER>(val, other);
        }
        /* vertex j takes the value of the last lane of its run in this chunk */
        const int s0 = excl > base ? excl : base;
        const int s1 = (excl + np < base + 32 ? excl + np : base + 32) - 1;
        const T mine = shfl_idx<T>(0xffffffffu, val, (s1 - base) & 31, 32);
        if (np > 0 && s0 <= s1) acc = combine<OWNER>(acc, mine);
    }
    cnt.edges += (unsigned long long)real;
    const bool raise = act && old < acc;
    if (act) {
        cnt.lifts++;
        if (raise) {
            pol.store(F + u, acc);
            cnt.changes++;
        }
    }
    push_raised(p, pol, u, raise, lane, cnt);
}

/* Two light words at once: the same steps as light_word, with the loads of
 * both words issued together so that twice as many are in flight. */
template <class T, int OWNER, class Pol>
__device__ __forceinline__ void light_word2(const LiftParams &p, T *F, const Pol &pol, const int gw[2],
                                            const uint32_t word[2], int lane, LiftCounters &cnt)
{
    int u[2], b[2], np[2], excl[2], total[2];
    bool act[2];
    T old[2], acc[2];
#pragma unroll
    for (int w = 0; w < 2; w++) {
        u[w] = (gw[w] << 5) + lane;
        act[w] = (word[w] >> lane) & 1u;
        b[w] = 0;
        np[w] = 0;
        old[w] = (T)0;
        acc[w] = identity<OWNER, T>();
        if (act[w]) {
            b[w] = __ldg(p.P + u[w]) >> 1;
            np[w] = (__ldg(p.P + u[w] + 1) >> 1) - b[w];
            old[w] = pol.load(F + u[w]);
        }
    }
#pragma unroll
    for (int w = 0; w < 2; w++) excl[w] = warp_excl_scan(np[w], lane, &total[w]);
    const int tmax = total[0] > total[1] ? total[0] : total[1];
    int real = 0;
    for (int base = 0; base < tmax; base += 32) {
        T val[2], f0[2], f1[2];
        int own[2];
        int4 q[2];
        bool has[2];
        /* phase 1: owners and edge pairs of both words */
#pragma unroll
        for (int w = 0; w < 2; w++) {
            const int t = base + lane;
            own[w] = owner_of(excl[w], t);
            const int ob = __shfl_sync(0xffffffffu, b[w], own[w]);
            const int oe = __shfl_sync(0xffffffffu, excl[w], own[w]);
            has[w] = t < total[w];
            q[w] = has[w] ? __ldg(p.E4 + ob + (t - oe)) : make_int4(0, 0, 0, 0);
        }
        /* phase 2: the successors' credits of both words */
#pragma unroll
        for (int w = 0; w < 2; w++) {
            f0[w] = has[w] ? pol.load(F + q[w].x) : (T)0;
            f1[w] = has[w] ? pol.load(F + q[w].z) : (T)0;
        }
#pragma unroll
        for (int w = 0; w < 2; w++) {
            val[w] = identity<OWNER, T>();
            if (has[w]) {
                val[w] = combine<OWNER>(ominus<T>(f0[w], q[w].y, p.mg), ominus<T>(f1[w], q[w].w, p.mg));
                real += 1 + (q[w].z < p.n_pad);
            }
        }
#pragma unroll
        for (int w = 0; w < 2; w++) {
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const T other = shfl_idx<T>(0xffffffffu, val[w], (lane - o) & 31, 32);
                const int oo = __shfl_sync(0xffffffffu, own[w], (lane - o) & 31);
                if (lane >= o && oo == own[w]) val[w] = combine<OWNER>(val[w], other);
            }
            const int s0 = excl[w] > base ? excl[w] : base;
            const int s1 = (excl[w] + np[w] < base + 32 ? excl[w] + np[w] : base + 32) - 1;
            const T mine = shfl_idx<T>(0xffffffffu, val[w], (s1 - base) & 31, 32);
            if (np[w] > 0 && s0 <= s1) acc[w] = combine<OWNER>(acc[w], mine);
        }
    }
    cnt.edges += (unsigned long long)real;
    int cb[2], nc[2], pexcl[2], ptotal[2];
#pragma unroll
    for (int w = 0; w < 2; w++) {
        cb[w] = 0;
        nc[w] = 0;
        if (act[w]) {
            cnt.lifts++;
            if (old[w] < acc[w]) {
                pol.store(F + u[w], acc[w]);
                cnt.changes++;
                cb[w] = __ldg(p.CP + u[w]) >> 2;
                nc[w] = (__ldg(p.CP + u[w] + 1) >> 2) - cb[w];
            }
        }
    }
#pragma unroll
    for (int w = 0; w < 2; w++) pexcl[w] = warp_excl_scan(nc[w], lane, &ptotal[w]);
    cnt.any_new |= (ptotal[0] + ptotal[1]) > 0;
    const int pmax = ptotal[0] > ptotal[1] ? ptotal[0] : ptotal[1];
    for (int base = 0; base < pmax; base += 32) {
#pragma unroll
        for (int w = 0; w < 2; w++) {
            const int t = base + lane;
            const int own = owner_of(pexcl[w], t);
            const int ocb = __shfl_sync(0xffffffffu, cb[w], own);
            const int oex = __shfl_sync(0xffffffffu, pexcl[w], own);
            if (t < ptotal[w]) cnt.pushes += push4(pol, __ldg((const int4 *)p.CS + ocb + (t - oex)));
        }
    }
}

/* Light words on the grid: dealt evenly to warps (static) or taken in
 * order (schedule 1), two at a time. */
template <class T, int OWNER>
__device__ __noinline__ void light_class(const LiftParams &p, const LiftClass &lc, T *F, uint32_t *cur, uint32_t *nxt,
                                         int *ctr, LiftCounters &cnt)
{
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    const int nwords = lc.word_end - lc.word_begin;
    const bool dyn = lc.grab < 0;
    const int lo = dyn ? 0 : (int)((long long)gwarp * nwords / nwarp);
    const int hi = dyn ? nwords : (int)((long long)(gwarp + 1) * nwords / nwarp);
    const GridPolicy pol{nxt};
    for (int w = lo;; w += 2) {
        if (dyn) {
            int t = 0;
            if (lane == 0) t = atomicAdd(ctr, 2);
            w = __shfl_sync(0xffffffffu, t, 0);
        }
        if (w >= hi) break;
        int gw[2];
        uint32_t word[2];
        uint32_t mine = 0;
        if (lane < 2 && w + lane < hi) {
            uint32_t *wp = cur + lc.word_begin + w + lane;
            mine = __ldcg(wp);
            if (mine) __stcg(wp, 0u);
        }
#pragma unroll
        for (int k = 0; k < 2; k++) {
            gw[k] = lc.word_begin + w + k;
            word[k] = __shfl_sync(0xffffffffu, mine, k);
        }
        if (word[0] | word[1]) light_word2<T, OWNER>(p, F, pol, gw, word, lane, cnt);
    }
}

/* The first step of the frontier rounds that follow dense ones: the
 * predecessors of the vertices raised by the last (recording) dense round,
 * marked in `ch`, join the frontier `bm`; the marks are consumed. */
__device__ __noinline__ void seed_words(const LiftParams &p, uint32_t *ch, uint32_t *bm, LiftCounters &cnt)
{
    const int lane = threadIdx.x & 31;
    const int gwarp = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
    const int nwarp = (int)((gridDim.x * (unsigned)blockDim.x) >> 5);
    const int nwords = p.n_pad >> 5;
    const GridPolicy pol{bm};
    for (int gw = gwarp; gw < nwords; gw += nwarp) {
        const uint32_t raised = __ldcg(ch + gw);
        if (!raised) continue;
        push_raised(p, pol, (gw << 5) + lane, (raised >> lane) & 1u, lane, cnt);
        if (lane == 0) __stcg(ch + gw, 0u);
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
                const int cb = __ldg(p.CP + u) >> 2, ce = __ldg(p.CP + u + 1) >> 2;
                if (threadIdx.x == 0) cnt.changes++;
                cnt.any_new |= ce > cb;
                const GridPolicy pol{nxt};
                for (int k = cb + threadIdx.x; k < ce; k += LIFT_BLOCK) cnt.pushes += push4(pol, __ldg((const int4 *)p.CS + k));
            }
            if (threadIdx.x == 0) cnt.lifts++;
            __syncthreads();
        }
    }
}

template <class T, int OWNER, bool LEAN>
__device__ __forceinline__ void run_class(const LiftParams &p, const LiftClass &lc, T *F, uint32_t *cur, uint32_t *nxt,
                                          int *ctr, LiftCounters &cnt)
{
    if (LEAN) { /* AUTO layout with heavy tasks: light classes only */
        light_class<T, OWNER>(p, lc, F, cur, nxt, ctr, cnt);
        return;
    }
    switch (lc.group) {
    case EG_GROUP_LIGHT: light_class<T, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case EG_GROUP_CTA: cta_class<T, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case 1: thread_class<T, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case 2: warp_class<T, 2, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case 4: warp_class<T, 4, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case 8: warp_class<T, 8, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    case 16: warp_class<T, 16, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    default: warp_class<T, 32, OWNER>(p, lc, F, cur, nxt, ctr, cnt); break;
    }
}

/* LEAN: the AUTO layout only (heavy tasks and light words), compiled for
 * three CTAs per SM; otherwise every variant, two CTAs per SM.
 *
 * Frontier rounds: round r lifts the vertices of B[r&1] and pushes into
 * B[(r+1)&1].  With round kinds on (LEAN, eg_opts.direction SWITCH) the
 * kernel hands over to the dense kernel: it starts at round Ctrl::rounds,
 * runs a seed step first when the dense kernel asked for one, and returns
 * as soon as the barrier's last arriver picks a dense round (raises of the
 * round >= dense_min_changes). */
template <class T, bool LEAN>
__global__ void __launch_bounds__(LIFT_BLOCK, LEAN ? 3 : 2) k_lift(const __grid_constant__ LiftParams p)
{
    __shared__ unsigned long long s_changes;
    Ctrl *c = p.ctrl;
    T *F = (T *)p.F;
    LiftCounters cnt = {0ull, 0ull, 0u, 0u, 0};
    const bool kinds = LEAN && p.direction == EG_DIRECTION_SWITCH;
    if (blockIdx.x == 0 && threadIdx.x == 0 && c->t_start == 0ull) c->t_start = globaltimer_ns();
    if (threadIdx.x == 0) s_changes = 0ull;
    __syncthreads();
    const long long round0 = ld_volatile(&c->rounds);
    for (long long round = round0;; round++) {
        uint32_t *cur = (round & 1) ? p.B1 : p.B0;
        uint32_t *nxt = (round & 1) ? p.B0 : p.B1;
        int *ctr = c->ctr[round & 1];
        const unsigned changes0 = cnt.changes;
        cnt.any_new = 0;
        unsigned long long t0 = 0, t1 = 0, t2 = 0;
        if (kinds && round == round0 && ld_volatile(&c->next_mode) == ROUND_SEED) {
            seed_words(p, (round & 1) ? p.CH0 : p.CH1, cur, cnt);
            if (!grid_barrier(c, p.wait_limit_ns, [] {})) break;
        }
        if (p.profile) t0 = globaltimer_ns();
        if (p.num_tasks) heavy_tasks<T>(p, F, cur, nxt, cnt);
        if (p.profile) t1 = globaltimer_ns();
        for (int ci = 0; ci < p.nclasses; ci++) {
            const LiftClass &lc = p.cls[ci];
            if (lc.owner) run_class<T, 1, LEAN>(p, lc, F, cur, nxt, ctr + ci, cnt);
            else run_class<T, 0, LEAN>(p, lc, F, cur, nxt, ctr + ci, cnt);
        }
        if (p.profile) t2 = globaltimer_ns();
        if (kinds) {
            /* this round's raises: warp sums into shared memory, then one
             * global add per CTA below */
            unsigned d = cnt.changes - changes0;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) d += __shfl_xor_sync(0xffffffffu, d, off);
            if ((threadIdx.x & 31) == 0 && d) atomicAdd(&s_changes, (unsigned long long)d);
        }
        if (__syncthreads_or(cnt.any_new) && threadIdx.x == 0) c->flag[(round + 1) & 1] = 1;
        if (kinds && threadIdx.x == 0) {
            if (s_changes) atomicAdd(&c->round_changes[round & 1], s_changes);
            s_changes = 0ull;
        }
        const bool ok = grid_barrier(c, p.wait_limit_ns, [&]() {
            /* last arriver of round `round`: clear this parity's counters
             * and flag, pick the next round's kind, then decide whether the
             * solve goes on */
            for (int ci = 0; ci < EG_MAX_CLASSES; ci++) c->ctr[round & 1][ci] = 0;
            c->flag[round & 1] = 0;
            c->rounds = round + 1;
            const bool more = ld_volatile(&c->flag[(round + 1) & 1]) != 0;
            if (kinds) {
                const unsigned long long raised = c->round_changes[round & 1];
                c->round_changes[(round + 1) & 1] = 0ull;
                c->next_mode = !more ? ROUND_DONE
                               : (long long)raised >= p.dense_min_changes ? ROUND_DENSE : ROUND_SPARSE;
            } else if (!more) {
                c->next_mode = ROUND_DONE;
            }
            if (more) check_stop(p, c, round);
        });
        if (p.profile && !kinds && (threadIdx.x & 31) == 0) {
            const unsigned long long t3 = globaltimer_ns();
            atomicAdd(&c->t_heavy, t1 - t0);
            atomicAdd(&c->t_light, t2 - t1);
            atomicAdd(&c->t_wait, t3 - t2);
        }
        if (!ok) break;
        if (ld_volatile(&c->stop)) break;
        if (!ld_volatile(&c->flag[(round + 1) & 1])) break;
        if (kinds && ld_volatile(&c->next_mode) == ROUND_DENSE) break; /* the dense kernel takes over */
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
    constexpr int NG = G >= 32 ? 1 : 32 / G;
    const int grp = lane / G, gl = lane % G;
    const unsigned gmask = (G >= 32) ? 0xffffffffu : (((1u << (G & 31)) - 1u) << (grp * G));
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
        if (G == EG_GROUP_LIGHT) {
            if (word) light_word<T, OWNER>(p, F, pol, gw, word, lane, cnt);
            continue;
        }
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
                if (g == EG_GROUP_LIGHT) cta_warp_class<T, EG_GROUP_LIGHT, 1>(p, lc, F, cur, pol, ctr, cnt);
                else if (g == 1) cta_warp_class<T, 1, 1>(p, lc, F, cur, pol, ctr, cnt);
                else if (g == 8) cta_warp_class<T, 8, 1>(p, lc, F, cur, pol, ctr, cnt);
                else cta_warp_class<T, 32, 1>(p, lc, F, cur, pol, ctr, cnt);
            } else {
                if (g == EG_GROUP_LIGHT) cta_warp_class<T, EG_GROUP_LIGHT, 0>(p, lc, F, cur, pol, ctr, cnt);
                else if (g == 1) cta_warp_class<T, 1, 0>(p, lc, F, cur, pol, ctr, cnt);
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
    const void *fn = credit_bits == 32 ? (p.lean ? (const void *)k_lift<int32_t, true> : (const void *)k_lift<int32_t, false>)
                                       : (p.lean ? (const void *)k_lift<int64_t, true> : (const void *)k_lift<int64_t, false>);
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
