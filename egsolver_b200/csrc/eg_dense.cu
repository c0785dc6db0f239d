/*
 * eg_dense.cu -- dense rounds: every vertex lifted, no frontier.
 *
 * When a large share of the credits rise in each round (the usual case on
 * large random games, where most vertices have a raised successor every
 * round), a frontier round spends most of its time pushing predecessors
 * into a bitmap that ends up nearly full.  A dense round lifts every vertex
 * against the current credits instead and pushes nothing: it reads the
 * edge pairs once, in order, and gathers the successors' credits.
 *
 * The padded edge-pair array E4 (pairs of one vertex are contiguous, see
 * k_copy_edges) is one stream of `npairs` pairs.  It is cut into equal
 * slices of `slice` pairs (a multiple of 32), one per warp of the grid, so
 * the work is balanced by construction whatever the degree distribution.
 * A warp walks its slice 32 pairs (one chunk) at a time: lane j gathers the
 * two successor credits of pair j and applies OMINUS, and a segmented
 * shuffle scan over runs of equal vertex gives every vertex's min (player 0)
 * or max (player 1) -- the max is taken as a min of negated values so one
 * scan serves both owners.  A vertex that runs on into the next chunk
 * carries its partial value in registers; a vertex cut by a slice edge
 * combines the partial values of all its slices with an atomic min / max,
 * and the slice that reports last finalizes it (reporter counts from
 * k_dense_setup).  Per pair, 16 bits of metadata (PM) give the owner, "last
 * pair of its vertex" and the vertex as an offset from the chunk's first
 * vertex (CB).
 *
 * Exactness: each dense round lifts every vertex once against credits that
 * are the round's start values or values raised during the round, all
 * below the least fixed point; a round without a raise has lifted every
 * vertex against the final credits, so they are the least fixed point.  This
 * is the same fair chaotic iteration as the reference's worklist loop
 * (reference src/dev_EG_alg.cu:307-381), so the credits are bit-identical.
 *
 * Hand-over to frontier rounds (k_lift): when a dense round raises fewer
 * than sparse_max_changes credits, the next round records its raised
 * vertices in the bitmap CH[r&1] (a "recording" round); if it too stays
 * below the bound, the kernel returns with Ctrl::next_mode = ROUND_SEED and
 * k_lift starts by pushing the predecessors of the recorded vertices.  Every
 * dense round clears CH[(r+1)&1], so a recording round always starts from a
 * clear map.
 */
#include "eg_lift.cuh"
#include "eg_prep.cuh"

namespace eg {

constexpr int DENSE_BLOCK = 512;
constexpr int kMetaBlock = 256;
constexpr uint32_t PM_OWNER = 0x8000u, PM_END = 0x4000u, PM_OFF = 0x3fffu;

template <class T>
__device__ __forceinline__ T shfl_up_t(T v, int off)
{
    return __shfl_up_sync(0xffffffffu, v, off);
}
template <>
__device__ __forceinline__ int64_t shfl_up_t<int64_t>(int64_t v, int off)
{
    return (int64_t)__shfl_up_sync(0xffffffffu, (long long)v, off);
}
template <class T>
__device__ __forceinline__ T shfl_t(T v, int src)
{
    return __shfl_sync(0xffffffffu, v, src);
}
template <>
__device__ __forceinline__ int64_t shfl_t<int64_t>(int64_t v, int src)
{
    return (int64_t)__shfl_sync(0xffffffffu, (long long)v, src);
}

/* ------------------------------------------------------------------ */
/* Pair-stream metadata (once per layout)                               */
/* ------------------------------------------------------------------ */

/* The vertex whose pairs hold pair t: the largest u with P[u] / 2 <= t.
 * Padding slots own no pairs and share the next vertex's offset, so they
 * are never the largest such u. */
__device__ __forceinline__ int pair_vertex(const int *P, int n_pad, int t)
{
    int lo = 0, hi = n_pad; /* P[lo] / 2 <= t < P[hi] / 2 */
    while (hi - lo > 1) {
        const int mid = lo + ((hi - lo) >> 1);
        if ((__ldg(P + mid) >> 1) <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void k_chunk_base(const int *P, int n_pad, int npairs, int *CB)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if ((long long)c * 32 >= npairs) return;
    CB[c] = pair_vertex(P, n_pad, c * 32);
}

__global__ void k_pair_meta(const int *P, int n_pad, int npairs, const ClassTable ct, const int *CB, uint16_t *PM,
                            int *err)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs) return;
    const int u = pair_vertex(P, n_pad, t);
    int off = u - CB[t >> 5];
    if (off < 0 || off > (int)PM_OFF) {
        atomicExch(err, 1);
        off = 0;
    }
    const bool end = t == (__ldg(P + u + 1) >> 1) - 1;
    PM[t] = (uint16_t)((ct.owner_of_new(u) ? PM_OWNER : 0u) | (end ? PM_END : 0u) | (uint32_t)off);
}

void build_pair_meta(const int *P, int n_pad, int npairs, const ClassTable &ct, uint16_t *PM, int *CB, int *err,
                     cudaStream_t st)
{
    if (npairs <= 0) return;
    const int nchunks = (npairs + 31) / 32;
    k_chunk_base<<<(nchunks + kMetaBlock - 1) / kMetaBlock, kMetaBlock, 0, st>>>(P, n_pad, npairs, CB);
    k_pair_meta<<<(npairs + kMetaBlock - 1) / kMetaBlock, kMetaBlock, 0, st>>>(P, n_pad, npairs, ct, CB, PM, err);
}

/* ------------------------------------------------------------------ */
/* Per solve: reporter counts of the vertices cut by slice edges         */
/* ------------------------------------------------------------------ */

template <class T>
__global__ void k_dense_setup(const int *P, int n_pad, const uint16_t *PM, int slice, int banks, T *dacc, int *drem)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_pad) return;
    const int b = P[u] >> 1, e = P[u + 1] >> 1;
    if (e <= b) return;
    const int nrep = (e - 1) / slice - b / slice + 1;
    if (nrep > 1) {
        for (int k = 0; k < banks; k++) {
            drem[(size_t)k * n_pad + u] = nrep;
            dacc[(size_t)k * n_pad + u] = (PM[b] & PM_OWNER) ? (T)0 : credit_traits<T>::top;
        }
    }
}

void launch_dense_setup(const LiftParams &p, int credit_bits, cudaStream_t st)
{
    const int grid = (p.n_pad + kMetaBlock - 1) / kMetaBlock;
    if (credit_bits == 32)
        k_dense_setup<int32_t><<<grid, kMetaBlock, 0, st>>>(p.P, p.n_pad, p.PM, p.slice, p.dense_sweeps,
                                                            (int32_t *)p.dacc, p.drem);
    else
        k_dense_setup<int64_t><<<grid, kMetaBlock, 0, st>>>(p.P, p.n_pad, p.PM, p.slice, p.dense_sweeps,
                                                            (int64_t *)p.dacc, p.drem);
}

/* ------------------------------------------------------------------ */
/* The dense-round kernel                                               */
/* ------------------------------------------------------------------ */

/* Packs E4's pairs into 8 bytes: per out-edge (succ << wbits) | (w + wbias). */
__global__ void k_pack_pairs(const int4 *E4, int npairs, int wbits, int wbias, int2 *E8)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= npairs) return;
    const int4 q = E4[t];
    E8[t] = make_int2((int)(((unsigned)q.x << wbits) | (unsigned)(q.y + wbias)),
                      (int)(((unsigned)q.z << wbits) | (unsigned)(q.w + wbias)));
}

void launch_pack_pairs(const int4 *E4, int npairs, int wbits, int wbias, int2 *E8, cudaStream_t st)
{
    if (npairs <= 0) return;
    k_pack_pairs<<<(npairs + kMetaBlock - 1) / kMetaBlock, kMetaBlock, 0, st>>>(E4, npairs, wbits, wbias, E8);
}

/* OMINUS in 32-bit arithmetic, for games where MG + max |w| < 2^31 - 1:
 * a finite credit minus a weight cannot overflow there, and the wrapped
 * difference of a = TOP is discarded. */
__device__ __forceinline__ int32_t ominus_fast(int32_t a, int32_t w, int32_t mg)
{
    const int32_t d = (int32_t)((uint32_t)a - (uint32_t)w);
    return (a < INT32_MAX && d <= mg) ? (d > 0 ? d : 0) : INT32_MAX;
}

/* A slice's partial value v (actual, not negated) of cut vertex u; the
 * slice that reports last raises the credit.  Returns whether it rose.
 * Each sweep of a round has its own accumulator bank: a warp may start its
 * next sweep before a slower warp has reported the same vertex for this
 * one, and mixing their reports would combine part of the edges only. */
template <class T>
__device__ __forceinline__ bool dense_report(const LiftParams &p, T *F, int u, bool own, T v, unsigned &changes,
                                             int bank)
{
    T *acc = (T *)p.dacc + (size_t)bank * p.n_pad;
    int *rem = p.drem + (size_t)bank * p.n_pad;
    if (own) atomic_combine<1>(acc + u, v);
    else atomic_combine<0>(acc + u, v);
    __threadfence();
    if (atomicSub(rem + u, 1) != 1) return false;
    __threadfence();
    const T r = atomic_swap(acc + u, own ? (T)0 : credit_traits<T>::top);
    const int b = __ldg(p.P + u) >> 1, e = __ldg(p.P + u + 1) >> 1;
    rem[u] = (e - 1) / p.slice - b / p.slice + 1; /* ready for the next round */
    const T old = ld_credit(F + u);
    if (old < r) {
        st_credit(F + u, r);
        changes++;
        return true;
    }
    return false;
}

/* Recording round: OR the raised vertices of this chunk into `ch`, one
 * atomic per distinct word (the raised vertices' ids rise with the lane). */
__device__ __forceinline__ void mark_raised(uint32_t *ch, int u, bool raise, int lane)
{
    unsigned rm = __ballot_sync(0xffffffffu, raise);
    while (rm) {
        const int l = __ffs(rm) - 1;
        const int wd = __shfl_sync(0xffffffffu, u >> 5, l);
        const bool mine = raise && (u >> 5) == wd;
        const unsigned same = __ballot_sync(0xffffffffu, mine);
        const uint32_t bits = __reduce_or_sync(0xffffffffu, mine ? (1u << (u & 31)) : 0u);
        if (lane == l) atomicOr(ch + wd, bits);
        rm &= ~same;
    }
}

/* The two out-edges of pair t: successors and weights. */
template <bool PACKED>
__device__ __forceinline__ void load_pair(const LiftParams &p, int t, int4 &q)
{
    if (PACKED) {
        const int2 e = __ldg(p.E8 + t);
        q = make_int4(e.x, e.y, 0, 0);
    } else {
        q = __ldg(p.E4 + t);
    }
}
template <bool PACKED>
__device__ __forceinline__ void decode_pair(const LiftParams &p, const int4 &q, int &s0, int &w0, int &s1, int &w1)
{
    if (PACKED) {
        const unsigned mask = (1u << p.wbits) - 1u;
        s0 = (int)((unsigned)q.x >> p.wbits);
        w0 = (int)((unsigned)q.x & mask) - p.wbias;
        s1 = (int)((unsigned)q.y >> p.wbits);
        w1 = (int)((unsigned)q.y & mask) - p.wbias;
    } else {
        s0 = q.x;
        w0 = q.y;
        s1 = q.z;
        w1 = q.w;
    }
}

/* One 32-pair chunk of a slice as its lanes hold it: the pair, its
 * metadata and the chunk's first vertex. */
struct Chunk {
    int4 q;
    uint32_t md;
    int base;
    bool in;
};

template <bool PACKED>
__device__ __forceinline__ void load_chunk(const LiftParams &p, int c0, int s1, int lane, Chunk &k)
{
    const int t = c0 + lane;
    k.in = t < s1;
    k.q = make_int4(0, 0, 0, 0);
    k.md = PM_END; /* lanes past the slice end count as ends */
    k.base = 0;
    if (k.in) {
        load_pair<PACKED>(p, t, k.q);
        k.md = __ldg(p.PM + t);
    }
    if (c0 < s1) k.base = __ldg(p.CB + (c0 >> 5));
}

/* The credits a chunk needs: both successors of the lane's pair and, on the
 * last pair of a vertex, the vertex's own. */
template <class T, bool PACKED>
__device__ __forceinline__ void gather_chunk(const LiftParams &p, const T *F, const Chunk &k, T &fa, T &fb, T &old)
{
    fa = fb = old = (T)0;
    if (k.in) {
        int sa, wa, sb, wb;
        decode_pair<PACKED>(p, k.q, sa, wa, sb, wb);
        fa = ld_credit(F + sa);
        fb = ld_credit(F + sb);
        if (k.md & PM_END) old = ld_credit(F + k.base + (int)(k.md & PM_OFF));
    }
}

/* Carry of a slice walk: the partial (min-space) value of the vertex that
 * runs on from the previous chunk. */
template <class T>
struct Carry {
    T val;
    bool on;   /* the chunk's lane-0 vertex continues from before      */
    bool cut;  /* that vertex began before this slice: report it       */
    int u_last;
    bool own_last;
};

/* Lifts the vertices of one chunk whose credits have arrived. */
template <class T, bool FAST, bool PACKED>
__device__ __forceinline__ void compute_chunk(const LiftParams &p, T *F, uint32_t *ch, bool rec, const Chunk &k, T fa,
                                              T fb, T old, int lane, uint32_t le_mask, Carry<T> &cr,
                                              unsigned &changes, int bank)
{
    constexpr T top = credit_traits<T>::top;
    const int u = k.base + (int)(k.md & PM_OFF);
    const bool own = (k.md & PM_OWNER) != 0;
    const bool end = (k.md & PM_END) != 0;
    T x = top;
    if (k.in) {
        int sa, wa, sb, wb;
        decode_pair<PACKED>(p, k.q, sa, wa, sb, wb);
        T va, vb;
        if (FAST) {
            va = (T)ominus_fast((int32_t)fa, wa, (int32_t)p.mg);
            vb = (T)ominus_fast((int32_t)fb, wb, (int32_t)p.mg);
        } else {
            va = ominus<T>(fa, wa, p.mg);
            vb = ominus<T>(fb, wb, p.mg);
        }
        x = own ? -(va > vb ? va : vb) : (va < vb ? va : vb);
    }
    /* inclusive min over each run of one vertex (a max for player 1,
     * negated), by a shuffle scan */
    const uint32_t ends = __ballot_sync(0xffffffffu, end);
    const int head = 31 - __clz(((ends << 1) | 1u) & le_mask);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = shfl_up_t<T>(x, o);
        if (lane - o >= head && y < x) x = y;
    }
    if (cr.on && head == 0 && cr.val < x) x = cr.val;
    /* vertices whose last pair is here */
    bool raise = false;
    if (k.in && end) {
        const T v = own ? -x : x;
        if (head == 0 && cr.cut) {
            raise = dense_report<T>(p, F, u, own, v, changes, bank);
        } else if (old < v) {
            st_credit(F + u, v);
            changes++;
            raise = true;
        }
    }
    if (rec) mark_raised(ch, u, raise, lane);
    /* the last lane's vertex runs on into the next chunk? */
    const bool open = !(ends >> 31);
    cr.cut = open && cr.cut && (ends & 0x7fffffffu) == 0u;
    cr.on = open;
    cr.val = shfl_t<T>(x, 31);
    cr.u_last = u;
    cr.own_last = own;
}

/* One warp's slice [s0, s1) of the pair stream.  FAST (32-bit credits
 * whose differences fit 32 bits): 32-bit OMINUS.  PACKED: 8-byte pairs.
 * DEPTH 1: the next chunk's pairs load while a chunk's credits are
 * gathered and reduced; DEPTH 2: also the next chunk's credits are in
 * flight while a chunk is reduced (more registers: two CTAs per SM). */
template <class T, bool FAST, bool PACKED, int DEPTH>
__device__ __forceinline__ void dense_slice(const LiftParams &p, T *F, uint32_t *ch, bool rec, int s0, int s1,
                                            int lane, unsigned &changes, int bank)
{
    if (s0 >= s1) return;
    const uint32_t le_mask = 0xffffffffu >> (31 - lane);
    Carry<T> cr;
    /* the vertex of the slice's first pair began in an earlier slice? */
    cr.on = s0 > 0 && !(__ldg(p.PM + s0 - 1) & PM_END);
    cr.cut = cr.on;
    cr.val = credit_traits<T>::top;
    cr.u_last = 0;
    cr.own_last = false;
    Chunk k0, k1;
    load_chunk<PACKED>(p, s0, s1, lane, k0);
    if (DEPTH == 1) {
        for (int c0 = s0; c0 < s1; c0 += 32) {
            load_chunk<PACKED>(p, c0 + 32, s1, lane, k1);
            T fa, fb, old;
            gather_chunk<T, PACKED>(p, F, k0, fa, fb, old);
            compute_chunk<T, FAST, PACKED>(p, F, ch, rec, k0, fa, fb, old, lane, le_mask, cr, changes, bank);
            k0 = k1;
        }
    } else {
        load_chunk<PACKED>(p, s0 + 32, s1, lane, k1);
        T fa0, fb0, old0;
        gather_chunk<T, PACKED>(p, F, k0, fa0, fb0, old0);
        for (int c0 = s0; c0 < s1; c0 += 32) {
            Chunk k2;
            load_chunk<PACKED>(p, c0 + 64, s1, lane, k2);
            T fa1, fb1, old1;
            gather_chunk<T, PACKED>(p, F, k1, fa1, fb1, old1);
            compute_chunk<T, FAST, PACKED>(p, F, ch, rec, k0, fa0, fb0, old0, lane, le_mask, cr, changes, bank);
            k0 = k1;
            k1 = k2;
            fa0 = fa1;
            fb0 = fb1;
            old0 = old1;
        }
    }
    /* the last vertex goes on in the next slice: report its part */
    const int cu = __shfl_sync(0xffffffffu, cr.u_last, 31);
    const bool cown = __shfl_sync(0xffffffffu, (int)cr.own_last, 31) != 0;
    if (cr.on && lane == 0) {
        const bool r = dense_report<T>(p, F, cu, cown, cown ? -cr.val : cr.val, changes, bank);
        if (rec && r) atomicOr(ch + (cu >> 5), 1u << (cu & 31));
    }
}

/* Persistent dense rounds from round Ctrl::rounds until the last arriver
 * picks another kind: ROUND_DONE (no raise: solved), or ROUND_SEED after a
 * recording round below sparse_max_changes.  Lifts and scanned edges are
 * not counted here: a dense round lifts every vertex and scans every edge. */
template <class T, bool FAST, bool PACKED, int DEPTH>
__global__ void __launch_bounds__(DENSE_BLOCK, DEPTH == 1 ? 3 : 2) k_lift_dense(const __grid_constant__ LiftParams p)
{
    __shared__ unsigned long long s_changes, s_busy, s_busy_max;
    Ctrl *c = p.ctrl;
    T *F = (T *)p.F;
    unsigned changes = 0u;
    const int lane = threadIdx.x & 31;
    const int gthr = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int nthr = (int)(gridDim.x * blockDim.x);
    const long long sl = (long long)(gthr >> 5) * p.slice;
    const int s0 = (int)(sl < p.npairs ? sl : p.npairs);
    const int s1 = (int)(sl + p.slice < p.npairs ? sl + p.slice : p.npairs);
    const int words = p.n_pad >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0 && c->t_start == 0ull) c->t_start = globaltimer_ns();
    if (threadIdx.x == 0) s_changes = s_busy = s_busy_max = 0ull;
    __syncthreads();
    const long long round0 = ld_volatile(&c->rounds);
    for (long long round = round0;; round++) {
        const int kind = round == round0 ? ROUND_DENSE : ld_volatile(&c->next_mode);
        uint32_t *cur = (round & 1) ? p.B1 : p.B0;
        uint32_t *ch = (round & 1) ? p.CH1 : p.CH0;
        uint32_t *chn = (round & 1) ? p.CH0 : p.CH1;
        /* the frontier left by frontier rounds is not used; the other
         * raised-map must be clear for a recording round next */
        for (int w = gthr; w < words; w += nthr) {
            if (round == round0) __stcg(cur + w, 0u);
            __stcg(chn + w, 0u);
        }
        const unsigned changes0 = changes;
        const unsigned long long t0 = p.profile ? globaltimer_ns() : 0ull;
        /* dense_sweeps sweeps of the slice per grid barrier; a round
         * without a raise in any of them ends the solve */
        for (int sw = 0; sw < p.dense_sweeps; sw++)
            dense_slice<T, FAST, PACKED, DEPTH>(p, F, ch, kind == ROUND_RECORD, s0, s1, lane, changes, sw);
        if (p.profile && lane == 0) {
            const unsigned long long dt = globaltimer_ns() - t0;
            atomicAdd(&s_busy, dt);
            atomicMax(&s_busy_max, dt);
        }
        unsigned d = changes - changes0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) d += __shfl_xor_sync(0xffffffffu, d, off);
        if (lane == 0 && d) atomicAdd(&s_changes, (unsigned long long)d);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (s_changes) atomicAdd(&c->round_changes[round & 1], s_changes);
            s_changes = 0ull;
            if (p.profile) {
                atomicAdd(&c->t_light, s_busy);
                atomicMax(&c->round_max[round & 1], s_busy_max);
                s_busy = s_busy_max = 0ull;
            }
        }
        const bool ok = grid_barrier(c, p.wait_limit_ns, [&]() {
            c->flag[round & 1] = 0;
            c->rounds = round + 1;
            c->dense_rounds += p.dense_sweeps; /* sweeps over every vertex */
            if (p.profile) {
                c->t_heavy += c->round_max[round & 1]; /* the slowest slice of the round */
                c->round_max[round & 1] = 0ull;
                const unsigned long long now = globaltimer_ns();
                if (c->t_round_prev) c->t_wait += now - c->t_round_prev; /* round to round */
                c->t_round_prev = now;
            }
            const unsigned long long raised = c->round_changes[round & 1];
            c->round_changes[(round + 1) & 1] = 0ull;
            c->changes += raised;
            c->dense_changes += raised;
            int next;
            if (raised == 0ull) {
                next = ROUND_DONE;
            } else if (p.direction == EG_DIRECTION_DENSE || (long long)raised >= p.sparse_max_changes) {
                next = ROUND_DENSE;
            } else if (kind == ROUND_RECORD) {
                next = ROUND_SEED;
                c->flag[(round + 1) & 1] = 1;
            } else {
                next = ROUND_RECORD;
            }
            c->next_mode = next;
            if (raised) check_stop(p, c, round);
        });
        if (!ok) break;
        if (ld_volatile(&c->stop)) break;
        const int nk = ld_volatile(&c->next_mode);
        if (nk != ROUND_DENSE && nk != ROUND_RECORD) break;
    }
}

template <class T, bool FAST, bool PACKED>
static const void *dense_fn_depth(int depth)
{
    return depth == 2 ? (const void *)k_lift_dense<T, FAST, PACKED, 2> : (const void *)k_lift_dense<T, FAST, PACKED, 1>;
}

template <class T, bool FAST>
static const void *dense_fn_packed(bool packed, int depth)
{
    return packed ? dense_fn_depth<T, FAST, true>(depth) : dense_fn_depth<T, FAST, false>(depth);
}

static const void *dense_fn(const LiftParams &p, int credit_bits)
{
    const bool packed = p.E8 != nullptr;
    if (credit_bits == 64) return dense_fn_packed<int64_t, false>(packed, p.dense_depth);
    return p.fast32 ? dense_fn_packed<int32_t, true>(packed, p.dense_depth)
                    : dense_fn_packed<int32_t, false>(packed, p.dense_depth);
}

eg_status dense_grid(int credit_bits, int depth, int max_ctas, int *grid)
{
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    /* the instantiations of one depth share their launch bounds */
    const void *fn = credit_bits == 32 ? dense_fn_depth<int32_t, true, true>(depth)
                                       : dense_fn_depth<int64_t, false, false>(depth);
    cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, DENSE_BLOCK, 0);
    if (err != cudaSuccess || per_sm < 1)
        return eg_set_error(EG_ERR_CUDA, "occupancy query for the dense kernel failed: %s", cudaGetErrorString(err));
    int g = sms * per_sm;
    if (max_ctas > 0 && max_ctas < g) g = max_ctas;
    *grid = g;
    return EG_OK;
}

eg_status launch_lift_dense(const LiftParams &p, int credit_bits, cudaStream_t st, int grid)
{
    const void *fn = dense_fn(p, credit_bits);
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, DENSE_BLOCK, 0);
    if (err != cudaSuccess || per_sm * sms < grid)
        return eg_set_error(EG_ERR_CUDA, "the dense kernel cannot hold %d co-resident CTAs", grid);
    void *args[] = {(void *)&p};
    err = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(DENSE_BLOCK), args, 0, st);
    if (err != cudaSuccess)
        return eg_set_error(EG_ERR_CUDA, "cooperative launch of the dense kernel failed: %s", cudaGetErrorString(err));
    return EG_OK;
}

}  // namespace eg
