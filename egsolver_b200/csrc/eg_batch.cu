/*
 * eg_batch.cu -- batched solving of many games at K mean-payoff thresholds
 * in one persistent launch.
 *
 * Work is cut into units: a game at a group of 1, 2, 4 or 8 of its
 * thresholds (weights w * d - p_k).  One CTA solves one unit at a time,
 * taking units from a device queue, heaviest first.  The unit's credits live
 * in the CTA's shared memory (rows x group x 4 or 8 bytes, up to the 227 KB
 * opt-in), so every credit gather of the lift is a shared-memory load; only
 * games too large for that keep their credits in a global scratch block.
 * The edges stream from L2 in the sliced layout of eg_batch.cuh, one
 * coalesced 128-byte column per warp step.
 *
 * A unit runs in-place sweeps over its vertices (a warp lifts the 32
 * vertices of a slice for all thresholds of the group at once) until a
 * sweep raises nothing.  A threshold whose credits did not rise in a sweep
 * is at its fixed point and is dropped from the following sweeps.  Every
 * lift reads credits that are initial values or values raised since, all
 * below the least fixed point, so each threshold's iteration is a fair
 * chaotic iteration of the reference's lifting operator (reference
 * src/dev_EG_alg.cu:84-109 on the weights w * d - p, OMINUS of
 * src/common.h:270-272) and its credits equal the worklist solver's.
 *
 * Arithmetic.  For a successor credit a and weight b = w * d - p, OMINUS is
 * g(a - b) with g(x) = x > MG ? TOP : max(x, 0), TOP stored as 2^30 (32-bit
 * credits) or 2^62 (64-bit): with MG + wpad * d + |p| below it, a TOP
 * successor gives a - b > MG, so g maps it to TOP exactly as OMINUS does.
 * g is monotone, so min_e g(a_e - b_e) = g(p + min_e (a_e - w_e d)) and
 * likewise for max: per edge and threshold one subtraction and one min (or
 * max), and g once per vertex.
 *
 * No wait in this kernel spins: sweeps end at __syncthreads and units come
 * from an atomic counter.
 */
#include "eg_batch.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <thread>
#include <type_traits>
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

template <typename CT> struct Lim;
template <> struct Lim<int> {
    static constexpr int top = 1 << 30;
    static constexpr int low = -(1 << 30);
    static constexpr int lo_acc = INT32_MIN;
    static constexpr int hi_acc = INT32_MAX;
};
template <> struct Lim<long long> {
    static constexpr long long top = 1LL << 62;
    static constexpr long long low = -(1LL << 62);
    static constexpr long long lo_acc = INT64_MIN;
    static constexpr long long hi_acc = INT64_MAX;
};

/* The KG credits of one vertex, loaded as one vector. */
template <int KG, typename CT>
struct alignas(sizeof(CT) * KG >= 16 ? 16 : sizeof(CT) * KG) Row {
    CT v[KG];
};

template <bool WIDE> struct Slot;
template <> struct Slot<false> {
    using T = uint32_t;
    static __device__ __forceinline__ T load(const void *E, int i) { return __ldg((const uint32_t *)E + i); }
    static __device__ __forceinline__ void dec(T e, int &s, int &w)
    {
        s = (int)(e & 0xffffu);
        w = (int)e >> 16;
    }
};
template <> struct Slot<true> {
    using T = int2;
    static __device__ __forceinline__ T load(const void *E, int i) { return __ldg((const int2 *)E + i); }
    static __device__ __forceinline__ void dec(T e, int &s, int &w)
    {
        s = e.x;
        w = e.y;
    }
};

/* Internal status of a unit handed to the tail (never returned). */
constexpr int kParked = -1;

struct Shared {
    unsigned raise[3];    /* per-sweep OR of raised thresholds (rotating)     */
    int unit;
    long long p[8], mg[8];
};

template <int KG> struct Log2 {
    static constexpr int v = KG == 1 ? 0 : KG == 2 ? 1 : KG == 4 ? 2 : 3;
};

/* Where a unit's credits live: all rows in shared memory, or (HYB, a
 * hybrid unit) rows below S there and the rest in the unit's global
 * scratch, which only the owning CTA touches. */
template <int KG, typename CT, bool HYB>
struct Cred {
    CT *Fs;
    CT *Fg;
    int S;
    __device__ __forceinline__ CT *at(int row) const
    {
        if (!HYB || row < S) return Fs + ((long long)row << Log2<KG>::v);
        return Fg + ((long long)(row - S) << Log2<KG>::v);
    }
};

/* min (player 0) or max (player 1, MAXV) over the W columns of a slice of
 * credit - w * d, for the KG thresholds at once; lane's first slot at i0. */
template <int KG, typename CT, bool WIDE, bool MAXV, int UNR, bool HYB>
__device__ __forceinline__ void column_walk(const void *E, int i0, int W, const Cred<KG, CT, HYB> &F, CT d,
                                            CT (&acc)[KG])
{
    using S = Slot<WIDE>;
    using ST = typename S::T;
    using R = Row<KG, CT>;
#pragma unroll
    for (int k = 0; k < KG; k++) acc[k] = MAXV ? Lim<CT>::lo_acc : Lim<CT>::hi_acc;
    for (int c = 0; c < W; c += UNR) {
        ST q[UNR];
#pragma unroll
        for (int x = 0; x < UNR; x++)
            if (c + x < W) q[x] = S::load(E, i0 + 32 * (c + x));
        R fr[UNR];
        int wt[UNR];
#pragma unroll
        for (int x = 0; x < UNR; x++) {
            if (c + x < W) {
                int sc;
                S::dec(q[x], sc, wt[x]);
                fr[x] = *(const R *)F.at(sc);
            }
        }
#pragma unroll
        for (int x = 0; x < UNR; x++) {
            if (c + x < W) {
                const CT t = (CT)wt[x] * d;
#pragma unroll
                for (int k = 0; k < KG; k++) {
                    const CT y = fr[x].v[k] - t;
                    acc[k] = MAXV ? (y > acc[k] ? y : acc[k]) : (y < acc[k] ? y : acc[k]);
                }
            }
        }
    }
}

/* Solves one unit (KG thresholds, credit type CT, slot width WIDE, credits
 * in shared memory or, with GF (a hybrid unit, KG = 1), rows from u.srows on
 * in the unit's global scratch). */
template <int KG, typename CT, bool WIDE, bool GF>
__device__ __forceinline__ void run_unit(const UnitDesc &u, int uglobal, unsigned char *smem, Shared &sh,
                                         const UnitParams &P, unsigned long long t0, unsigned long long &lifts,
                                         unsigned long long &edges, unsigned long long &ntop)
{
    using R = Row<KG, CT>;
    constexpr CT TOPI = Lim<CT>::top, LOWI = Lim<CT>::low;
    constexpr int LK = Log2<KG>::v;
    /* columns whose loads are issued together: about 16 bytes of credits */
    constexpr int UNR = (KG * (int)sizeof(CT) <= 4) ? 8 : (KG * (int)sizeof(CT) <= 8) ? 4
                        : (KG * (int)sizeof(CT) <= 16) ? 2 : 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    Cred<KG, CT, GF> F;
    F.Fs = (CT *)smem;
    F.Fg = (CT *)u.gscratch;
    F.S = GF ? u.srows : 0;
    const int ns = u.ns, s0 = u.s0, npad = 32 * ns;
    const int rows = npad + 2;
    for (int i = tid; i < rows * KG; i += blockDim.x) {
        const int r = i >> LK;
        F.at(r)[i & (KG - 1)] = r < npad ? (CT)0 : (r == npad ? TOPI : LOWI);
    }
    if (tid < KG) {
        sh.p[tid] = u.p[u.k0 + tid];
        sh.mg[tid] = u.mg[u.k0 + tid];
    }
    if (tid == 0) sh.raise[0] = sh.raise[1] = sh.raise[2] = 0;
    __syncthreads();
    const CT d = (CT)u.d;
    const unsigned full = (1u << KG) - 1u;
    unsigned amask = full;
    long long r = 0;
    int st = EG_OK;
    for (;;) {
        unsigned raised = 0;
        for (int s = warp; s < ns; s += nwarps) {
            const int b = __ldg(u.slice_off + s);
            const int W = (__ldg(u.slice_off + s + 1) - b) >> 5;
            const bool own1 = s >= s0;
            CT acc[KG];
            if (own1) column_walk<KG, CT, WIDE, true, UNR, GF>(u.E, b + lane, W, F, d, acc);
            else column_walk<KG, CT, WIDE, false, UNR, GF>(u.E, b + lane, W, F, d, acc);
            const int v = 32 * s + lane;
            const bool real = own1 ? (v - 32 * s0 < u.n1) : (v < u.n0);
            if (real) {
                CT *mine = F.at(v);
                R old = *(const R *)mine;
#pragma unroll
                for (int k = 0; k < KG; k++) {
                    if (amask >> k & 1u) {
                        /* threshold and MG from shared memory: used once per vertex */
                        const CT val = acc[k] + (CT)sh.p[k];
                        const CT nv = val > (CT)sh.mg[k] ? TOPI : (val > 0 ? val : (CT)0);
                        if (nv > old.v[k]) {
                            mine[k] = nv;
                            raised |= 1u << k;
                        }
                    }
                }
            }
        }
        raised = __reduce_or_sync(0xffffffffu, raised);
        const int slot = (int)(r % 3);
        if (lane == 0 && raised) atomicOr(&sh.raise[slot], raised);
        if (tid == 0) {
            if (P.timeout_ns && globaltimer_ns() - t0 > P.timeout_ns) atomicOr(&sh.raise[slot], 1u << 16);
            /* park: this variant's queue is empty and half of all phase-1
             * CTAs have nothing left, so the GPU is running the tail; the
             * unit's open thresholds continue on clusters */
            if (P.tails && (r & 15) == 15 && ld_volatile(&P.ctrl->next) >= P.num_units &&
                100 * ld_volatile(P.idle) >= P.park_percent * P.park_total)
                atomicOr(&sh.raise[slot], 1u << 17);
        }
        __syncthreads();
        const unsigned word = sh.raise[slot];
        if (tid == 0) {
            sh.raise[(r + 2) % 3] = 0;
            lifts += (unsigned long long)(u.n0 + u.n1) * (unsigned)__popc(amask);
            edges += (unsigned long long)u.m * (unsigned)__popc(amask);
        }
        r++;
        amask &= word & full;
        if (amask == 0) break;
        if (word & (1u << 16)) {
            st = EG_ERR_TIMEOUT;
            break;
        }
        if (word & (1u << 17)) {
            st = kParked;
            break;
        }
        if (P.max_rounds >= 0 && r >= P.max_rounds) {
            st = EG_ERR_LOOPCAP;
            break;
        }
    }
    __syncthreads();
    /* credits out, threshold-major in original vertex ids */
    unsigned long long top = 0;
    for (int i = tid; i < npad * KG; i += blockDim.x) {
        const int k = i / npad, v = i - k * npad;
        const int o = __ldg(u.orig + v);
        if (o >= 0) {
            const CT c = F.at(v)[k];
            u.F[(long long)(u.k0 + k) * u.n + o] = c >= TOPI ? (long long)INT64_MAX : (long long)c;
            /* the TOPs of a parked unit's open thresholds are counted by the tail */
            top += c >= TOPI && !(st == kParked && (amask >> k & 1u));
        }
    }
    ntop += top;
    if (tid == 0) sh.unit = 0; /* reused below as the overflow flag */
    __syncthreads();
    if (st == kParked && tid < KG && (amask >> tid & 1u)) {
        TailList *tl = P.tails + tail_class(u.variant);
        const int at = atomicAdd(&tl->count, 1);
        if (at < tl->cap) {
            TailEntry e;
            e.unit = uglobal;
            e.k = u.k0 + tid;
            e.sweeps = r;
            e.resume = 1;
            e.pad = 0;
            tl->e[at] = e;
        } else {
            atomicExch(&sh.unit, 1); /* cannot happen: lists hold every threshold */
        }
    }
    __syncthreads();
    if (tid == 0) {
        *u.rounds = r;
        *u.status = sh.unit ? EG_ERR_OOM : (st == kParked ? EG_OK : st);
    }
    __syncthreads();
}

/* One persistent kernel per unit variant: CTAs take units of that variant
 * from its queue (heaviest first) until it is empty. */
template <int KG, typename CT, bool WIDE, bool GF>
__global__ void __launch_bounds__(1024, 1) k_units(const __grid_constant__ UnitParams P)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Shared sh;
    if (threadIdx.x == 0) {
        const unsigned long long now = globaltimer_ns();
        atomicCAS(&P.ctrl->t_begin, 0ull, now);
        atomicCAS(P.t_start, 0ull, now);
    }
    __syncthreads();
    /* timeouts count from the launch's first CTA (phase 1 or tail) */
    const unsigned long long t0 = ld_volatile_u64(P.t_start);
    unsigned long long lifts = 0, edges = 0, ntop = 0;
    for (;;) {
        if (threadIdx.x == 0) sh.unit = atomicAdd(&P.ctrl->next, 1);
        __syncthreads();
        const int ui = sh.unit;
        __syncthreads();
        if (ui >= P.num_units) break;
        const UnitDesc u = P.units[ui];
        run_unit<KG, CT, WIDE, GF>(u, P.unit_base + ui, smem, sh, P, t0, lifts, edges, ntop);
    }
    if (threadIdx.x == 0 && P.idle) atomicAdd(P.idle, 1);
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ntop += __shfl_xor_sync(0xffffffffu, ntop, off);
    if (lane == 0 && ntop) atomicAdd(&P.ctrl->num_top, ntop);
    if (threadIdx.x == 0) {
        atomicAdd(&P.ctrl->lifts, lifts);
        atomicAdd(&P.ctrl->edges, edges);
        atomicMax(&P.ctrl->t_end, globaltimer_ns());
    }
}

typedef void (*unit_kernel_t)(UnitParams);

/* The kernel of a variant (NULL for combinations that do not exist). */
unit_kernel_t kernel_of(int v)
{
#define EG_K(KG, CT, WD, GF) (unit_kernel_t)k_units<KG, CT, WD, GF>
    switch (v) {
    case 0: return EG_K(1, int, false, false);
    case 1: return EG_K(2, int, false, false);
    case 2: return EG_K(4, int, false, false);
    case 3: return EG_K(8, int, false, false);
    case kUnitCredit64 | 0: return EG_K(1, long long, false, false);
    case kUnitCredit64 | 1: return EG_K(2, long long, false, false);
    case kUnitCredit64 | 2: return EG_K(4, long long, false, false);
    case kUnitCredit64 | 3: return EG_K(8, long long, false, false);
    case kUnitWide | 0: return EG_K(1, int, true, false);
    case kUnitWide | 1: return EG_K(2, int, true, false);
    case kUnitWide | 2: return EG_K(4, int, true, false);
    case kUnitWide | 3: return EG_K(8, int, true, false);
    case kUnitWide | kUnitCredit64 | 0: return EG_K(1, long long, true, false);
    case kUnitWide | kUnitCredit64 | 1: return EG_K(2, long long, true, false);
    case kUnitWide | kUnitCredit64 | 2: return EG_K(4, long long, true, false);
    case kUnitWide | kUnitCredit64 | 3: return EG_K(8, long long, true, false);
    case kUnitGlobal: return EG_K(1, int, false, true);
    case kUnitGlobal | kUnitCredit64: return EG_K(1, long long, false, true);
    case kUnitGlobal | kUnitWide: return EG_K(1, int, true, true);
    case kUnitGlobal | kUnitWide | kUnitCredit64: return EG_K(1, long long, true, true);
    default: return nullptr;
    }
#undef EG_K
}


/* ------------------------------------------------------------------ */
/* The tail: one (unit, threshold) per thread-block cluster             */
/* ------------------------------------------------------------------ */

namespace cg = cooperative_groups;

/* Every CTA of the cluster holds a full replica of the unit's credits in
 * its shared memory and lifts the slices of its own row range [rank * R,
 * (rank + 1) * R) (R = ceil(rows / cluster size) rounded up to 32, so a
 * slice never straddles two ranges), gathering successor credits from its
 * local replica.  The range's slots are copied into shared memory behind
 * the replica when they fit, so a sweep touches no global memory.  A warp
 * that raised a credit of its slice writes the slice's 32 credits into
 * every peer's replica right away (one coalesced store per peer through
 * the cluster's distributed shared memory).
 *
 * A CTA runs T.sweeps sweeps between two cluster barriers (fewer at a
 * sweep cap), its
 * warps without waiting for one another, and reads whatever its replica
 * holds: every value there is a credit some CTA computed, hence below the
 * least fixed point, so the iteration stays a fair chaotic one.  The
 * barrier makes every write before it visible after it.  If no CTA raised
 * anything between two barriers, nothing was written there either, so each
 * vertex was lifted against the state of the first barrier without rising:
 * that state is the least fixed point.  The OR of the CTAs' raise flags is
 * gathered in rank 0's shared memory (three rotating words, as in phase 1).
 * Random 4-byte gathers through distributed shared memory are about ten
 * times slower than local ones, hence the replicas. */
template <typename CT, bool WIDE, bool HYB>
struct TailSweep {
    using S = Slot<WIDE>;
    using ST = typename S::T;
    static constexpr int UNR = sizeof(CT) == 4 ? 4 : 2;
    CT *F;             /* the replica (shared memory)                          */
    CT *G;             /* hybrid: rows >= SR of this CTA's replica (global)    */
    const ST *Es;      /* the range's slots in shared memory (staged) or null  */
    const ST *Eg;      /* the unit's slots in global memory                    */
    const int *slice_off;
    char *gpeer0;      /* hybrid: the cluster's first global region            */
    long long gstride;
    int SR, s_lo, s_hi, s0, n0, n1, b0, rank, C;
    CT pk, mgk, d;

    __device__ __forceinline__ CT ld(int row) const
    {
        return (!HYB || row < SR) ? F[row] : (CT)__ldcg(G + (row - SR));
    }

    /* One sweep of the warp's slices; true if a credit rose.  Slots are
     * read through a generic pointer: shared memory when staged, else
     * global memory. */
    __device__ __forceinline__ bool sweep(cg::cluster_group &cl, int lane, int warp, int nwarps) const
    {
        bool raised = false;
        for (int s = s_lo + warp; s < s_hi; s += nwarps) {
            const int b = __ldg(slice_off + s);
            const int W = (__ldg(slice_off + s + 1) - b) >> 5;
            const bool own1 = s >= s0;
            CT acc = own1 ? Lim<CT>::lo_acc : Lim<CT>::hi_acc;
            const ST *E = Es ? Es + (b - b0) : Eg + b;
            for (int c = 0; c < W; c += UNR) {
                ST q[UNR];
#pragma unroll
                for (int x = 0; x < UNR; x++)
                    if (c + x < W) q[x] = E[lane + 32 * (c + x)];
                CT f[UNR];
                int wt[UNR];
#pragma unroll
                for (int x = 0; x < UNR; x++) {
                    if (c + x < W) {
                        int sc;
                        S::dec(q[x], sc, wt[x]);
                        f[x] = ld(sc);
                    }
                }
#pragma unroll
                for (int x = 0; x < UNR; x++) {
                    if (c + x < W) {
                        const CT y = f[x] - (CT)wt[x] * d;
                        acc = own1 ? (y > acc ? y : acc) : (y < acc ? y : acc);
                    }
                }
            }
            const int v = 32 * s + lane;
            const bool real = own1 ? (v - 32 * s0 < n1) : (v < n0);
            bool up = false;
            if (real) {
                const CT val = acc + pk;
                const CT nv = val > mgk ? Lim<CT>::top : (val > 0 ? val : (CT)0);
                if (nv > ld(v)) {
                    if (!HYB || v < SR) F[v] = nv;
                    else __stcg(G + (v - SR), nv);
                    up = true;
                }
            }
            /* the slice's raised credits go to every peer's replica at once
             * (32 consecutive rows: one coalesced store per peer) */
            if (__any_sync(0xffffffffu, up)) {
                raised = true;
                const CT x = ld(v);
                for (int q = 1; q < C; q++) {
                    const int peer = rank + q < C ? rank + q : rank + q - C;
                    if (!HYB || v < SR) *cl.map_shared_rank(F + v, peer) = x;
                    else __stcg((CT *)(gpeer0 + (long long)peer * gstride) + (v - SR), x);
                }
            }
        }
        return raised;
    }
};

template <typename CT, bool WIDE, bool HYB>
__global__ void __launch_bounds__(1024, 1) k_tail(const __grid_constant__ TailParams T)
{
    using TS = TailSweep<CT, WIDE, HYB>;
    using ST = typename TS::ST;
    constexpr CT TOPI = Lim<CT>::top, LOWI = Lim<CT>::low;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    CT *F = (CT *)smem_raw;
    __shared__ int s_entry;
    __shared__ unsigned s_word[3];
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int C = (int)cl.num_blocks();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    /* hybrid: rows >= srows of this CTA's replica live in its own global
     * region, which its peers write (read through L2) */
    CT *G = HYB ? (CT *)(T.gscratch + (long long)blockIdx.x * T.gstride) : nullptr;
    if (tid == 0) {
        const unsigned long long now = globaltimer_ns();
        atomicCAS(&T.ctrl->t_begin, 0ull, now);
        atomicCAS(T.t_start, 0ull, now);
    }
    __syncthreads();
    const unsigned long long t0 = ld_volatile_u64(T.t_start);
    unsigned long long lifts = 0, edges = 0, ntop = 0;
    for (;;) {
        if (rank == 0 && tid == 0) s_entry = atomicAdd(&T.list->next, 1);
        cl.sync();
        const int ei = *cl.map_shared_rank(&s_entry, 0);
        cl.sync();
        if (ei >= T.list->count || ei >= T.list->cap) break;
        const TailEntry en = T.list->e[ei];
        const UnitDesc &u = T.units[en.unit];
        const int k = en.k;
        const int npad = 32 * u.ns, rows = npad + 2;
        const int R = (((rows + C - 1) / C) + 31) & ~31;
        const int lo = min(rows, rank * R);
        const int hi = min(npad, lo + R); /* own rows */
        TS w;
        w.F = F;
        w.G = G;
        w.Eg = (const ST *)u.E;
        w.slice_off = u.slice_off;
        w.gpeer0 = HYB ? T.gscratch + (long long)(blockIdx.x - rank) * T.gstride : nullptr;
        w.gstride = T.gstride;
        w.SR = HYB ? u.srows : rows; /* rows in shared memory */
        w.s_lo = lo >> 5;
        w.s_hi = hi >> 5;
        w.s0 = u.s0;
        w.n0 = u.n0;
        w.n1 = u.n1;
        w.rank = rank;
        w.C = C;
        w.pk = (CT)u.p[k];
        w.mgk = (CT)u.mg[k];
        w.d = (CT)u.d;
        /* the full replica */
        for (int v = tid; v < rows; v += blockDim.x) {
            CT x;
            if (v == npad) x = TOPI;
            else if (v == npad + 1) x = LOWI;
            else {
                x = 0;
                const int o = __ldg(u.orig + v);
                if (en.resume && o >= 0) {
                    const long long c = u.F[(long long)k * u.n + o];
                    x = c == (long long)INT64_MAX ? TOPI : (CT)c;
                }
            }
            if (!HYB || v < w.SR) F[v] = x;
            else __stcg(G + (v - w.SR), x);
        }
        /* the range's slots behind the replica, when they fit (whole
         * slices: a multiple of 32 slots, 16-byte aligned in both places) */
        w.b0 = __ldg(u.slice_off + w.s_lo);
        const int b1 = __ldg(u.slice_off + w.s_hi);
        const long long rep_bytes = ((long long)w.SR * (long long)sizeof(CT) + 15) & ~15LL;
        const long long slot_bytes = (long long)(b1 - w.b0) * (long long)sizeof(ST);
        const bool stage = !HYB && rep_bytes + slot_bytes <= (long long)T.smem_bytes &&
                           ((uintptr_t)(w.Eg + w.b0) & 15) == 0;
        w.Es = stage ? (const ST *)(smem_raw + rep_bytes) : nullptr;
        if (stage) {
            const uint4 *src = (const uint4 *)(w.Eg + w.b0);
            uint4 *dst = (uint4 *)(smem_raw + rep_bytes);
            const int n16 = (int)(slot_bytes >> 4);
            for (int i = tid; i < n16; i += blockDim.x) dst[i] = __ldg(src + i);
        }
        if (tid == 0) s_word[0] = s_word[1] = s_word[2] = 0u;
        cl.sync();
        long long r = 0;
        int st = EG_OK;
        for (int iv = 0;; iv++) {
            long long ns = T.sweeps;
            if (T.max_rounds >= 0) ns = max(1LL, min(ns, T.max_rounds - en.sweeps - r));
            bool raised = false;
            for (int it = 0; it < (int)ns; it++) {
                raised |= w.sweep(cl, lane, warp, nwarps);
                __syncwarp();
            }
            const int slot = iv % 3;
            if (__syncthreads_or((int)raised) && tid == 0) atomicOr(cl.map_shared_rank(&s_word[slot], 0), 1u);
            if (rank == 0 && tid == 0 && T.timeout_ns && globaltimer_ns() - t0 > T.timeout_ns)
                atomicOr(&s_word[slot], 1u << 16);
            cl.sync();
            const unsigned word = *cl.map_shared_rank(&s_word[slot], 0);
            if (rank == 0 && tid == 0) {
                s_word[(slot + 2) % 3] = 0u;
                lifts += (unsigned long long)(u.n0 + u.n1) * (unsigned long long)ns;
                edges += (unsigned long long)u.m * (unsigned long long)ns;
            }
            r += ns;
            if (!(word & 1u)) break;
            if (word & (1u << 16)) {
                st = EG_ERR_TIMEOUT;
                break;
            }
            if (T.max_rounds >= 0 && en.sweeps + r >= T.max_rounds) {
                st = EG_ERR_LOOPCAP;
                break;
            }
        }
        /* credits out (own rows), TOP count, the unit's sweeps and status */
        unsigned long long top = 0;
        for (int v = lo + tid; v < hi; v += blockDim.x) {
            const int o = __ldg(u.orig + v);
            if (o >= 0) {
                const CT c = w.ld(v);
                u.F[(long long)k * u.n + o] = c >= TOPI ? (long long)INT64_MAX : (long long)c;
                top += c >= TOPI;
            }
        }
        ntop += top;
        if (rank == 0 && tid == 0) {
            atomicMax((unsigned long long *)u.rounds, (unsigned long long)(en.sweeps + r));
            if (st != EG_OK) atomicExch(u.status, st);
        }
        cl.sync(); /* no CTA writes into another's replica of this entry any more */
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ntop += __shfl_xor_sync(0xffffffffu, ntop, off);
    if (lane == 0 && ntop) atomicAdd(&T.ctrl->num_top, ntop);
    if (tid == 0) {
        atomicAdd(&T.ctrl->lifts, lifts);
        atomicAdd(&T.ctrl->edges, edges);
        atomicMax(&T.ctrl->t_end, globaltimer_ns());
    }
}

/* Heaviest first: sorts each tail list by the work its entry has shown so
 * far (sweeps x edges; an entry listed by the host counts n / 4 sweeps), one
 * CTA per class, bitonic over the list padded to a power of two with
 * entries of key -1 (unit -1) that sort last. */
__device__ __forceinline__ double tail_key(const TailEntry &e, const UnitDesc *units)
{
    if (e.unit < 0) return -1.0;
    const UnitDesc &u = units[e.unit];
    const double sw = e.resume ? (double)e.sweeps : (double)u.n * 0.25;
    return sw * (double)u.m;
}

__global__ void k_tail_order(TailList *lists, const UnitDesc *units)
{
    TailList &l = lists[blockIdx.x];
    const int n = min(l.count, l.cap);
    if (n < 2) return;
    int N = 1;
    while (N < n) N <<= 1;
    for (int i = n + threadIdx.x; i < N; i += blockDim.x) {
        TailEntry pad;
        pad.unit = -1;
        pad.k = 0;
        pad.sweeps = 0;
        pad.resume = 0;
        pad.pad = 0;
        l.e[i] = pad;
    }
    __syncthreads();
    for (int k = 2; k <= N; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < N; i += blockDim.x) {
                const int m = i ^ j;
                if (m <= i) continue;
                const TailEntry a = l.e[i], b = l.e[m];
                const double ka = tail_key(a, units), kb = tail_key(b, units);
                const bool desc = (i & k) == 0; /* descending runs first */
                if (desc ? (ka < kb) : (ka > kb)) {
                    l.e[i] = b;
                    l.e[m] = a;
                }
            }
            __syncthreads();
        }
    }
}

typedef void (*tail_kernel_t)(TailParams);

tail_kernel_t tail_kernel_of(int cls)
{
    switch (cls) {
    case 0: return (tail_kernel_t)k_tail<int, false, false>;
    case 1: return (tail_kernel_t)k_tail<long long, false, false>;
    case 2: return (tail_kernel_t)k_tail<int, true, false>;
    case 3: return (tail_kernel_t)k_tail<long long, true, false>;
    case 4: return (tail_kernel_t)k_tail<int, false, true>;
    case 5: return (tail_kernel_t)k_tail<long long, false, true>;
    case 6: return (tail_kernel_t)k_tail<int, true, true>;
    default: return (tail_kernel_t)k_tail<long long, true, true>;
    }
}

/* Before a solve: rewinds the tail lists to their host-listed entries and
 * clears the sweeps and status of the units those entries belong to (no
 * phase-1 kernel writes them). */
__global__ void k_tail_rewind(TailList *lists, const UnitDesc *units)
{
    for (int c = 0; c < kTailClasses; c++) {
        const TailList &l = lists[c];
        for (int i = threadIdx.x; i < l.init; i += blockDim.x) {
            const TailEntry en = l.ie[i];
            l.e[i] = en; /* the previous solve's sort moved them */
            const UnitDesc &u = units[en.unit];
            *u.rounds = 0;
            *u.status = EG_OK;
        }
    }
    __syncthreads();
    if (threadIdx.x < kTailClasses) {
        lists[threadIdx.x].count = lists[threadIdx.x].init;
        lists[threadIdx.x].next = 0;
    }
}

int align32i(int x) { return (x + 31) & ~31; }

}  // namespace

/* ------------------------------------------------------------------ */
/* Packing, planning and launch (shared with the serving loop)          */
/* ------------------------------------------------------------------ */

namespace eg {

eg_status pack_game(const eg_game &G, HostPacked *out)
{
    HostPacked h;
    const int n = G.num_nodes;
    h.n = n;
    h.m = G.num_edges;
    auto owner = [&](int v) { return G.owner ? (int)G.owner[v] : (v >= G.num_nodes0 ? 1 : 0); };
    std::vector<int> deg((size_t)n);
    long long maxabs = 0;
    h.minw.assign((size_t)n, 0);
    for (int v = 0; v < n; v++) {
        deg[(size_t)v] = (int)(G.row_ptr[v + 1] - G.row_ptr[v]);
        h.maxdeg = std::max(h.maxdeg, deg[(size_t)v]);
        int mn = INT32_MAX;
        for (long long j = G.row_ptr[v]; j < G.row_ptr[v + 1]; j++) {
            const int w = G.weight[j];
            mn = std::min(mn, w);
            maxabs = std::max(maxabs, w < 0 ? -(long long)w : (long long)w);
        }
        h.minw[(size_t)v] = mn;
        if (owner(v)) h.n1++;
        else h.n0++;
    }
    if (maxabs + 1 > (long long)INT32_MAX) return eg_set_error(EG_ERR_INVALID, "weights out of range for the batch path");
    h.wpad = (int)(maxabs + 1);
    /* stable counting sort by (owner, degree) */
    std::vector<int> order((size_t)n);
    {
        const int nb = 2 * (h.maxdeg + 1);
        std::vector<int> cnt((size_t)nb + 1, 0);
        for (int v = 0; v < n; v++) cnt[(size_t)(owner(v) * (h.maxdeg + 1) + deg[(size_t)v]) + 1]++;
        for (int i = 0; i < nb; i++) cnt[(size_t)i + 1] += cnt[(size_t)i];
        for (int v = 0; v < n; v++) order[(size_t)cnt[(size_t)(owner(v) * (h.maxdeg + 1) + deg[(size_t)v])]++] = v;
    }
    const int a0 = align32i(h.n0), a1 = align32i(h.n1);
    const int npad = a0 + a1;
    h.ns = npad / 32;
    h.s0 = a0 / 32;
    h.wide = (npad + 2 > 65536 || h.wpad > 32767) ? 1 : 0;
    h.orig.assign((size_t)npad, -1);
    std::vector<int> newid((size_t)n);
    for (int i = 0; i < n; i++) {
        const int v = order[(size_t)i];
        const int u = i < h.n0 ? i : a0 + (i - h.n0);
        newid[(size_t)v] = u;
        h.orig[(size_t)u] = v;
    }
    h.slice_off.assign((size_t)h.ns + 1, 0);
    long long slots = 0;
    for (int s = 0; s < h.ns; s++) {
        int W = 0;
        for (int l = 0; l < 32; l++) {
            const int v = h.orig[(size_t)(32 * s + l)];
            if (v >= 0) W = std::max(W, deg[(size_t)v]);
        }
        slots += 32LL * W;
        if (slots > (long long)INT32_MAX - 64) return eg_set_error(EG_ERR_INVALID, "game too large for the batch path");
        h.slice_off[(size_t)s + 1] = (int)slots;
    }
    h.slots = slots;
    const int toprow = npad, lowrow = npad + 1;
    if (h.wide) h.e64.resize((size_t)slots);
    else h.e32.resize((size_t)slots);
    for (int s = 0; s < h.ns; s++) {
        const int W = (h.slice_off[(size_t)s + 1] - h.slice_off[(size_t)s]) / 32;
        const bool own1 = s >= h.s0;
        for (int l = 0; l < 32; l++) {
            const int v = h.orig[(size_t)(32 * s + l)];
            for (int j = 0; j < W; j++) {
                int sc, w;
                if (v >= 0 && j < deg[(size_t)v]) {
                    const long long e = G.row_ptr[v] + j;
                    sc = newid[(size_t)G.succ[e]];
                    w = G.weight[e];
                } else {
                    sc = own1 ? lowrow : toprow;
                    w = own1 ? h.wpad : -h.wpad;
                }
                const size_t at = (size_t)h.slice_off[(size_t)s] + (size_t)j * 32 + (size_t)l;
                if (h.wide) h.e64[at] = make_int2(sc, w);
                else h.e32[at] = (uint32_t)(sc & 0xffff) | ((uint32_t)(uint16_t)(int16_t)w << 16);
            }
        }
    }
    *out = std::move(h);
    return EG_OK;
}

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t packed_dev_bytes(const HostPacked &h)
{
    const size_t eb = (size_t)h.slots * (h.wide ? sizeof(int2) : sizeof(uint32_t));
    return al256(std::max<size_t>(eb, 16)) + al256(sizeof(int) * ((size_t)h.ns + 1)) + al256(sizeof(int) * (size_t)(32 * h.ns + 1));
}

eg_status packed_upload(const HostPacked &h, void *block, cudaStream_t st, PackedDev *out)
{
    char *p = (char *)block;
    const size_t eb = (size_t)h.slots * (h.wide ? sizeof(int2) : sizeof(uint32_t));
    PackedDev d;
    d.block = block;
    d.E = p;
    d.slice_off = (int *)(p + al256(std::max<size_t>(eb, 16)));
    d.orig = (int *)((char *)d.slice_off + al256(sizeof(int) * ((size_t)h.ns + 1)));
    d.bytes = packed_dev_bytes(h);
    cudaError_t e = cudaSuccess;
    if (eb) e = cudaMemcpyAsync(d.E, h.wide ? (const void *)h.e64.data() : (const void *)h.e32.data(), eb,
                                cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d.slice_off, h.slice_off.data(), sizeof(int) * ((size_t)h.ns + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && h.ns)
        e = cudaMemcpyAsync(d.orig, h.orig.data(), sizeof(int) * (size_t)(32 * h.ns), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "packed game upload failed: %s", cudaGetErrorString(e));
    *out = d;
    return EG_OK;
}

long long threshold_mg(const HostPacked &h, int p, int d)
{
    long long s = 0;
    for (int v = 0; v < h.n; v++) {
        const long long x = (long long)p - (long long)d * h.minw[(size_t)v];
        if (x > 0) s += x;
    }
    return s;
}

bool credits32_ok(const HostPacked &h, const int *p, int K, int d, const long long *mg)
{
    for (int k = 0; k < K; k++) {
        const long long ap = p[k] < 0 ? -(long long)p[k] : (long long)p[k];
        if (mg[k] + (long long)h.wpad * d + ap >= (1LL << 30)) return false;
    }
    return true;
}

int tail_rows_per_cta(int rows) { return (rows + 31) & ~31; }

UnitPlan plan_game(const HostPacked &h, bool credit64, int smem_budget, int kg_cap, int tail_rows)
{
    UnitPlan pl;
    pl.credit64 = credit64 ? 1 : 0;
    pl.kg_max = 0;
    pl.tail = 0;
    const long long cb = credit64 ? 8 : 4;
    for (int kg = 8; kg >= 1; kg >>= 1) {
        if (tail_rows > 0 && h.n >= tail_rows) break;
        if (kg > kg_cap) continue;
        if ((long long)h.rows() * kg * cb <= smem_budget) {
            pl.kg_max = kg;
            return pl;
        }
    }
    /* too large for one CTA: a cluster holds it, else global scratch */
    pl.tail = (long long)tail_rows_per_cta(h.rows()) * cb <= smem_budget ? 1 : 0;
    return pl;
}

void split_thresholds(int K, int kg_max, std::vector<std::pair<int, int>> *groups)
{
    const int cap = kg_max < 1 ? 1 : kg_max;
    int k0 = 0;
    while (k0 < K) {
        int g = 1;
        while (g * 2 <= cap && g * 2 <= K - k0) g *= 2;
        groups->push_back({k0, g == 1 ? 0 : g == 2 ? 1 : g == 4 ? 2 : 3});
        k0 += g;
    }
}

eg_status make_units(const HostPacked &h, const PackedDev &pd, int K, int d, const int *p, const long long *mg,
                     const int *p_dev, const long long *mg_dev, long long *F_dev, int smem_budget, int kg_cap,
                     std::vector<UnitDesc> *units, std::vector<size_t> *gneed, std::vector<long long> *cost,
                     int *smem, int tail_rows)
{
    if ((long long)h.wpad * d >= (1LL << 31))
        return eg_set_error(EG_ERR_OVERFLOW, "weight * scale does not fit 32 bits");
    for (int k = 0; k < K; k++)
        if (mg[k] >= (1LL << 61)) return eg_set_error(EG_ERR_OVERFLOW, "threshold %d: MG %lld too large", k, mg[k]);
    const bool c64 = !credits32_ok(h, p, K, d, mg);
    const UnitPlan pl = plan_game(h, c64, smem_budget, kg_cap, tail_rows);
    std::vector<std::pair<int, int>> groups;
    split_thresholds(K, pl.kg_max, &groups);
    if (pl.tail) {
        /* one unit for all thresholds: the host lists (unit, k) for every k */
        UnitDesc u;
        memset(&u, 0, sizeof u);
        u.E = pd.E;
        u.slice_off = pd.slice_off;
        u.orig = pd.orig;
        u.p = p_dev;
        u.mg = mg_dev;
        u.F = F_dev;
        u.m = h.m;
        u.n = h.n;
        u.n0 = h.n0;
        u.n1 = h.n1;
        u.ns = h.ns;
        u.s0 = h.s0;
        u.d = d;
        u.k0 = 0;
        u.pad = K; /* thresholds to list */
        u.variant = kUnitTail | (c64 ? kUnitCredit64 : 0) | (h.wide ? kUnitWide : 0);
        units->push_back(u);
        gneed->push_back(0);
        cost->push_back(h.m * (long long)h.n * K);
        return EG_OK;
    }
    for (auto &gr : groups) {
        UnitDesc u;
        memset(&u, 0, sizeof u);
        u.E = pd.E;
        u.slice_off = pd.slice_off;
        u.orig = pd.orig;
        u.p = p_dev;
        u.mg = mg_dev;
        u.F = F_dev;
        u.m = h.m;
        u.n = h.n;
        u.n0 = h.n0;
        u.n1 = h.n1;
        u.ns = h.ns;
        u.s0 = h.s0;
        u.d = d;
        u.k0 = gr.first;
        const int kg = 1 << gr.second;
        const size_t need = (size_t)h.rows() * kg * (c64 ? 8 : 4);
        if (pl.kg_max == 0) {
            /* hybrid: as many rows as fit in shared memory, the rest in the
             * unit's global scratch */
            const int cb = c64 ? 8 : 4;
            u.variant = (c64 ? kUnitCredit64 : 0) | (h.wide ? kUnitWide : 0) | kUnitGlobal;
            u.srows = std::max(32, (smem_budget / cb) & ~31);
            gneed->push_back(((size_t)(h.rows() - u.srows) * cb + 255) & ~(size_t)255);
            *smem = std::max(*smem, u.srows * cb);
        } else {
            u.variant = gr.second | (c64 ? kUnitCredit64 : 0) | (h.wide ? kUnitWide : 0);
            gneed->push_back(0);
            *smem = std::max(*smem, (int)need);
        }
        units->push_back(u);
        cost->push_back(h.m * (long long)h.n * kg);
    }
    return EG_OK;
}

int unit_smem_budget(int device)
{
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess) {
        cudaGetLastError();
        optin = 48 * 1024;
    }
    int stat = 0;
    for (int v = 0; v < kNumVariants; v++) {
        unit_kernel_t k = kernel_of(v);
        if (!k) continue;
        cudaFuncAttributes fa;
        memset(&fa, 0, sizeof fa);
        if (cudaFuncGetAttributes(&fa, (const void *)k) != cudaSuccess) cudaGetLastError();
        stat = std::max(stat, (int)fa.sharedSizeBytes);
    }
    for (int c = 0; c < kTailClasses; c++) {
        cudaFuncAttributes fa;
        memset(&fa, 0, sizeof fa);
        if (cudaFuncGetAttributes(&fa, (const void *)tail_kernel_of(c)) != cudaSuccess) cudaGetLastError();
        stat = std::max(stat, (int)fa.sharedSizeBytes);
    }
    return optin - stat - 64;
}

eg_status unit_kernel_setup(int device)
{
    const int budget = unit_smem_budget(device);
    for (int v = 0; v < kNumVariants; v++) {
        unit_kernel_t k = kernel_of(v);
        if (!k) continue;
        cudaError_t e = cudaFuncSetAttribute((const void *)k, cudaFuncAttributeMaxDynamicSharedMemorySize, budget);
        if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "cudaFuncSetAttribute failed: %s", cudaGetErrorString(e));
    }
    for (int c = 0; c < kTailClasses; c++) {
        cudaError_t e = cudaFuncSetAttribute((const void *)tail_kernel_of(c), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             budget);
        if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "cudaFuncSetAttribute failed: %s", cudaGetErrorString(e));
        /* 16-CTA clusters are beyond the portable 8 */
        if (cudaFuncSetAttribute((const void *)tail_kernel_of(c), cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess)
            cudaGetLastError();
    }
    return EG_OK;
}

void group_units(const std::vector<UnitDesc> &units, const std::vector<long long> &cost,
                 const std::vector<size_t> &gneed, UnitSet *out, std::vector<int> *perm)
{
    const int nu = (int)units.size();
    std::vector<int> order((size_t)nu);
    std::iota(order.begin(), order.end(), 0);
    /* phase-1 units by variant, heaviest first; tail units last */
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        if (units[(size_t)a].variant != units[(size_t)c].variant)
            return units[(size_t)a].variant < units[(size_t)c].variant;
        return cost[(size_t)a] > cost[(size_t)c];
    });
    UnitSet S;
    for (int v = 0; v <= kNumVariants; v++) S.off[v] = 0;
    for (int v = 0; v < kNumVariants; v++) {
        S.smem[v] = 16;
        S.top_cost[v] = -1;
    }
    for (int c = 0; c < kTailClasses; c++) {
        S.tail_cap[c] = 0;
        S.tail_smem[c] = 16;
        S.tail_gbytes[c] = 0;
    }
    for (int i : order) {
        const UnitDesc &u = units[(size_t)i];
        const int v = u.variant;
        const int j = (int)S.units.size();
        S.units.push_back(u);
        S.gneed.push_back(gneed[(size_t)i]);
        const int cls = tail_class(v);
        const int rows = 32 * u.ns + 2;
        const int cb = (v & kUnitCredit64) ? 8 : 4;
        if (v & kUnitTail) {
            for (int k = 0; k < u.pad; k++) {
                TailEntry e;
                memset(&e, 0, sizeof e);
                e.unit = j;
                e.k = k;
                S.tail_init[cls].push_back(e);
            }
            S.tail_cap[cls] += u.pad;
            S.tail_smem[cls] = std::max(S.tail_smem[cls], tail_rows_per_cta(rows) * cb);
            continue;
        }
        S.off[v + 1]++;
        S.top_cost[v] = std::max(S.top_cost[v], cost[(size_t)i]);
        /* a parked unit lists its open thresholds for the tail */
        if (!(v & kUnitGlobal)) {
            const int kg = 1 << (v & kUnitKgMask);
            S.smem[v] = std::max(S.smem[v], rows * kg * cb);
            S.tail_cap[cls] += kg;
            S.tail_smem[cls] = std::max(S.tail_smem[cls], tail_rows_per_cta(rows) * cb);
        } else {
            S.smem[v] = std::max(S.smem[v], u.srows * cb);
            S.tail_cap[cls] += 1;
            S.tail_smem[cls] = std::max(S.tail_smem[cls], u.srows * cb);
            S.tail_gbytes[cls] = std::max(S.tail_gbytes[cls], ((long long)(rows - u.srows) * cb + 255) & ~255LL);
        }
    }
    for (int v = 0; v < kNumVariants; v++) S.off[v + 1] += S.off[v];
    if (perm) *perm = order;
    *out = std::move(S);
}

static size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

/* Cluster CTAs a hybrid tail class may launch: its scratch holds one
 * region per CTA. */
static int tail_hyb_ctas(int num_sms) { return num_sms + kTailCluster; }

size_t tail_scratch_bytes(const UnitSet &S, int num_sms)
{
    size_t b = 0;
    for (int c = 0; c < kTailClasses; c++)
        if (S.tail_cap[c] > 0 && S.tail_gbytes[c] > 0) b += (size_t)tail_hyb_ctas(num_sms) * (size_t)S.tail_gbytes[c];
    return b;
}

static int pow2_ceil(int x)
{
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

size_t tail_bytes(const UnitSet &S)
{
    size_t b = al16(sizeof(TailList) * kTailClasses);
    for (int c = 0; c < kTailClasses; c++)
        b += al16(sizeof(TailEntry) * (size_t)pow2_ceil(std::max(S.tail_cap[c], 1))) +
             al16(sizeof(TailEntry) * std::max<size_t>(S.tail_init[c].size(), 1));
    return b;
}

eg_status tail_upload(const UnitSet &S, void *block, cudaStream_t st, TailList **lists)
{
    TailList hl[kTailClasses];
    char *p = (char *)block;
    char *q = p + al16(sizeof(TailList) * kTailClasses);
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < kTailClasses; c++) {
        hl[c].count = hl[c].init = (int)S.tail_init[c].size();
        hl[c].next = 0;
        hl[c].cap = S.tail_cap[c];
        hl[c].cap2 = pow2_ceil(std::max(S.tail_cap[c], 1));
        hl[c].pad = 0;
        hl[c].e = (TailEntry *)q;
        q += al16(sizeof(TailEntry) * (size_t)hl[c].cap2);
        hl[c].ie = (const TailEntry *)q;
        if (e == cudaSuccess && !S.tail_init[c].empty())
            e = cudaMemcpyAsync(q, S.tail_init[c].data(), sizeof(TailEntry) * S.tail_init[c].size(),
                                cudaMemcpyHostToDevice, st);
        q += al16(sizeof(TailEntry) * std::max<size_t>(S.tail_init[c].size(), 1));
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(p, hl, sizeof hl, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "tail list upload failed: %s", cudaGetErrorString(e));
    *lists = (TailList *)p;
    return EG_OK;
}

eg_status UnitLauncher::init()
{
    if (cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&fork2, cudaEventDisableTiming) != cudaSuccess)
        return eg_set_error(EG_ERR_CUDA, "event creation failed");
    for (int v = 0; v < kNumCtrl; v++) {
        if (v < kNumVariants && !kernel_of(v)) continue;
        if (cudaStreamCreateWithFlags(&aux[v], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&join[v], cudaEventDisableTiming) != cudaSuccess)
            return eg_set_error(EG_ERR_CUDA, "stream creation failed");
    }
    return EG_OK;
}

void UnitLauncher::destroy()
{
    for (int v = 0; v < kNumCtrl; v++) {
        if (aux[v]) cudaStreamDestroy(aux[v]);
        if (join[v]) cudaEventDestroy(join[v]);
        aux[v] = nullptr;
        join[v] = nullptr;
    }
    if (fork) cudaEventDestroy(fork);
    if (fork2) cudaEventDestroy(fork2);
    fork = fork2 = nullptr;
}

/* Clusters of `csize` CTAs of the tail kernel of class cls that fit the
 * GPU at once (0 when none). */
static int tail_clusters(int cls, int csize, int block, int smem)
{
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof cfg);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(csize);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, (const void *)tail_kernel_of(cls), &cfg) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

eg_status launch_unit_set(UnitLauncher &L, cudaStream_t main, const UnitSet &S, const UnitDesc *units_dev,
                          TailList *tails, void *tail_scratch, LaunchCtrl *ctrl, int block, int num_sms,
                          long long max_rounds, unsigned long long timeout_ns, int *grid_total, int park_percent,
                          int tail_sweeps, int tail_cluster)
{
    cudaError_t e = cudaMemsetAsync(ctrl, 0, sizeof(LaunchCtrl), main);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "launch set-up failed: %s", cudaGetErrorString(e));
    k_tail_rewind<<<1, 256, 0, main>>>(tails, units_dev);
    e = cudaEventRecord(L.fork, main);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "launch set-up failed: %s", cudaGetErrorString(e));
    /* phase 1: the variant holding the heaviest unit is launched first */
    std::vector<int> vs;
    for (int v = 0; v < kNumVariants; v++)
        if (S.off[v + 1] > S.off[v]) vs.push_back(v);
    std::stable_sort(vs.begin(), vs.end(), [&](int a, int c) { return S.top_cost[a] > S.top_cost[c]; });
    std::vector<int> grids(vs.size());
    int total = 0;
    for (size_t i = 0; i < vs.size(); i++) {
        const int v = vs[i];
        unit_kernel_t k = kernel_of(v);
        if (!k) return eg_set_error(EG_ERR_INVALID, "no kernel for unit variant %d", v);
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k, block, (size_t)S.smem[v]);
        if (e != cudaSuccess || per_sm < 1)
            return eg_set_error(EG_ERR_CUDA, "unit kernel does not fit (block %d, %d B shared)", block, S.smem[v]);
        grids[i] = std::max(1, std::min(num_sms * per_sm, S.off[v + 1] - S.off[v]));
        total += grids[i];
    }
    for (size_t i = 0; i < vs.size(); i++) {
        const int v = vs[i];
        UnitParams p;
        memset(&p, 0, sizeof p);
        p.units = units_dev + S.off[v];
        p.ctrl = &ctrl->c[v];
        p.tails = tails;
        p.idle = &ctrl->idle;
        p.num_units = S.off[v + 1] - S.off[v];
        p.unit_base = S.off[v];
        p.park_total = total;
        p.park_percent = park_percent;
        if (park_percent > 100) p.tails = nullptr; /* no parking */
        p.t_start = &ctrl->t_start;
        p.max_rounds = max_rounds;
        p.timeout_ns = timeout_ns;
        void *args[] = {(void *)&p};
        e = cudaStreamWaitEvent(L.aux[v], L.fork, 0);
        if (e == cudaSuccess)
            e = cudaLaunchKernel((const void *)kernel_of(v), dim3(grids[i]), dim3(block), args, (size_t)S.smem[v], L.aux[v]);
        if (e == cudaSuccess) e = cudaEventRecord(L.join[v], L.aux[v]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(main, L.join[v], 0);
        if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "unit kernel launch failed: %s", cudaGetErrorString(e));
    }
    /* phase 2: the tail lists on clusters, heaviest entries first, one
     * kernel per class that can hold entries (those with no entries at run
     * time exit at once) */
    k_tail_order<<<kTailClasses, 1024, 0, main>>>(tails, units_dev);
    e = cudaEventRecord(L.fork2, main);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "launch set-up failed: %s", cudaGetErrorString(e));
    char *gs = (char *)tail_scratch;
    int dev = 0;
    cudaGetDevice(&dev);
    /* the class kernels share the GPU, and whichever's clusters start first
     * hold their SMs until its list is empty; hybrid classes (rows in
     * global memory, the slowest sweeps, so the likeliest to bound the
     * tail) launch first and at the greatest priority */
    int prio_least = 0, prio_greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest) != cudaSuccess) {
        cudaGetLastError();
        prio_least = prio_greatest = 0;
    }
    for (int c = kTailClasses - 1; c >= 0; c--) {
        if (S.tail_cap[c] == 0) continue;
        const int slot = kNumVariants + c;
        /* a tail CTA owns its SM: all the shared memory a CTA may have
         * keeps a second CTA (of this or another cluster) off it, which
         * would halve a heavy entry's sweep rate, and leaves room behind the
         * replica for the CTA's slots */
        const int tsmem = std::max(S.tail_smem[c], unit_smem_budget(dev));
        /* clusters of tail_cluster CTAs where they can be scheduled, else
         * half as many, down to 8 */
        int csize = tail_cluster > 0 ? tail_cluster : kTailCluster;
        int ncl = tail_clusters(c, csize, 1024, tsmem);
        while (ncl < 1 && csize > 8) {
            csize >>= 1;
            ncl = tail_clusters(c, csize, 1024, tsmem);
        }
        if (ncl < 1) return eg_set_error(EG_ERR_CUDA, "tail kernel clusters do not fit (%d B shared)", tsmem);
        TailParams tp;
        memset(&tp, 0, sizeof tp);
        tp.units = units_dev;
        tp.list = tails + c;
        tp.ctrl = &ctrl->c[slot];
        tp.t_start = &ctrl->t_start;
        tp.max_rounds = max_rounds;
        tp.timeout_ns = timeout_ns;
        tp.smem_bytes = tsmem;
        tp.sweeps = std::max(1, tail_sweeps);
        if (S.tail_gbytes[c] > 0) {
            if (!gs) return eg_set_error(EG_ERR_INVALID, "hybrid tail without scratch");
            ncl = std::min(ncl, tail_hyb_ctas(num_sms) / csize);
            tp.gscratch = gs;
            tp.gstride = S.tail_gbytes[c];
            gs += (size_t)tail_hyb_ctas(num_sms) * (size_t)S.tail_gbytes[c];
        }
        cudaLaunchConfig_t cfg;
        memset(&cfg, 0, sizeof cfg);
        cudaLaunchAttribute attr[2];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = csize;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        attr[1].id = cudaLaunchAttributePriority;
        attr[1].val.priority = (c & 4) ? prio_greatest : prio_least;
        const int ent = S.tail_cap[c];
        cfg.gridDim = dim3(csize * std::max(1, std::min(ncl, ent)));
        cfg.blockDim = dim3(1024);
        cfg.dynamicSmemBytes = (size_t)tsmem;
        cfg.stream = L.aux[slot];
        cfg.attrs = attr;
        cfg.numAttrs = 2;
        e = cudaStreamWaitEvent(L.aux[slot], L.fork2, 0);
        if (e == cudaSuccess) {
            e = cudaLaunchKernelEx(&cfg, tail_kernel_of(c), tp);
            if (e != cudaSuccess) { /* without the priority, where it is refused */
                cudaGetLastError();
                cfg.numAttrs = 1;
                e = cudaLaunchKernelEx(&cfg, tail_kernel_of(c), tp);
            }
        }
        if (e == cudaSuccess) e = cudaEventRecord(L.join[slot], L.aux[slot]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(main, L.join[slot], 0);
        if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "tail kernel launch failed: %s", cudaGetErrorString(e));
    }
    if (grid_total) *grid_total = total;
    return EG_OK;
}

void sum_ctrl(const LaunchCtrl &lc, UnitCtrl *out)
{
    memset(out, 0, sizeof *out);
    for (int v = 0; v < kNumCtrl; v++) {
        const UnitCtrl &c = lc.c[v];
        out->lifts += c.lifts;
        out->edges += c.edges;
        out->num_top += c.num_top;
        if (c.t_begin && (!out->t_begin || c.t_begin < out->t_begin)) out->t_begin = c.t_begin;
        out->t_end = std::max(out->t_end, c.t_end);
    }
}

}  // namespace eg

/* ------------------------------------------------------------------ */
/* Batch API                                                            */
/* ------------------------------------------------------------------ */

struct eg_batch {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int num_games = 0, K = 0, d = 1;
    long long total_nodes = 0, total_edges = 0;
    int block = 1024, kg_cap = 8, smem_budget = 0, sms = 148, tail_rows = 0, park_percent = 10;
    int tail_sweeps = kTailSweeps;
    int tail_cluster = kTailCluster;
    long long max_rounds = -1;
    double timeout_ms = 0;
    std::vector<HostPacked> hp;      /* host images (slots dropped after upload) */
    std::vector<PackedDev> pd;
    std::vector<long long> f_off;    /* credits of game g start at F + f_off[g]  */
    void *dblock = nullptr;          /* packed games                             */
    long long *F = nullptr;          /* sum_g n_g * K credits                    */
    int *p_dev = nullptr;            /* num_games * K thresholds                 */
    long long *mg_dev = nullptr;     /* num_games * K MG values                  */
    std::vector<int> p_host;
    std::vector<long long> mg_host;
    UnitSet set;                     /* units grouped by variant                 */
    std::vector<int> unit_game;      /* game of each grouped unit                */
    UnitDesc *units_dev = nullptr;
    long long *u_rounds = nullptr;
    int *u_status = nullptr;
    int units_cap = 0;
    void *gscratch = nullptr;
    size_t gscratch_bytes = 0;
    LaunchCtrl *ctrl = nullptr;      /* counters of a solve                      */
    void *tails = nullptr;           /* tail lists (tail_bytes of the plan)      */
    size_t tails_bytes = 0;
    void *tscratch = nullptr;        /* hybrid tail regions                      */
    size_t tscratch_bytes = 0;
    UnitLauncher launcher;
    size_t bytes = 0, unit_bytes = 0;
    bool thresholds_set = false, solved = false, use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_block = 0, graph_grid = 0;
    std::vector<long long> last_rounds;
    std::vector<int> last_status;
};

static void batch_drop_graph(eg_batch *b)
{
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
}

static void batch_free_units(eg_batch *b)
{
    void *ptrs[] = {b->units_dev, b->u_rounds, b->u_status, b->gscratch};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    b->units_dev = nullptr;
    b->u_rounds = nullptr;
    b->u_status = nullptr;
    b->gscratch = nullptr;
    b->gscratch_bytes = 0;
    b->units_cap = 0;
    b->bytes -= b->unit_bytes;
    b->unit_bytes = 0;
}

extern "C" void eg_batch_free(eg_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->st) cudaStreamSynchronize(b->st);
    batch_drop_graph(b);
    batch_free_units(b);
    void *ptrs[] = {b->dblock, b->F, b->p_dev, b->mg_dev, b->ctrl, b->tails, b->tscratch};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    b->launcher.destroy();
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

extern "C" int64_t eg_batch_device_bytes(const eg_batch *b) { return b ? (int64_t)b->bytes : 0; }

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

/* Runs fn(i) for i in [0, count) on the host's cores. */
template <class Fn>
static void parallel_for(int count, Fn fn)
{
    int nt = (int)std::thread::hardware_concurrency();
    nt = std::max(1, std::min(nt, 32));
    if (count < 4 || nt == 1) {
        for (int i = 0; i < count; i++) fn(i);
        return;
    }
    std::vector<std::thread> th;
    std::atomic<int> next(0);
    for (int t = 0; t < nt; t++)
        th.emplace_back([&]() {
            for (int i = next.fetch_add(1); i < count; i = next.fetch_add(1)) fn(i);
        });
    for (auto &x : th) x.join();
}

extern "C" eg_status eg_batch_create(const eg_game *games, int32_t num_games, const eg_batch_opts *opts, eg_batch **out)
{
    if (!games || num_games <= 0 || !opts || !out) return eg_set_error(EG_ERR_INVALID, "bad batch arguments");
    if (opts->thresholds < 1 || opts->thresholds > EG_BATCH_MAX_K)
        return eg_set_error(EG_ERR_INVALID, "thresholds must be in [1, %d]", EG_BATCH_MAX_K);
    if (opts->scale < 1) return eg_set_error(EG_ERR_INVALID, "scale d must be >= 1");
    if (opts->block && (opts->block < 64 || opts->block > 1024 || (opts->block & 31)))
        return eg_set_error(EG_ERR_INVALID, "block must be a multiple of 32 in [64, 1024]");
    if (opts->group_max && opts->group_max != 1 && opts->group_max != 2 && opts->group_max != 4 && opts->group_max != 8)
        return eg_set_error(EG_ERR_INVALID, "group_max must be 1, 2, 4 or 8");
    if (opts->tail_sweeps < 0 || opts->tail_sweeps > 16)
        return eg_set_error(EG_ERR_INVALID, "tail_sweeps must be in [0, 16]");
    if (opts->tail_cluster != 0 && opts->tail_cluster != 1 && opts->tail_cluster != 2 && opts->tail_cluster != 4 &&
        opts->tail_cluster != 8 && opts->tail_cluster != 16)
        return eg_set_error(EG_ERR_INVALID, "tail_cluster must be 0, 1, 2, 4, 8 or 16");
    long long tn = 0, tm = 0;
    for (int g = 0; g < num_games; g++) {
        eg_status s = eg_validate(&games[g]);
        if (s != EG_OK) return eg_set_error(s, "game %d: %s", g, eg_last_error());
        if (games[g].num_nodes > kBatchMaxGameNodes)
            return eg_set_error(EG_ERR_INVALID, "game %d has %d vertices; the batch path holds at most %d per game",
                                g, games[g].num_nodes, kBatchMaxGameNodes);
        tn += games[g].num_nodes;
        tm += games[g].num_edges;
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return eg_set_error(EG_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (opts->device < 0 || opts->device >= count) return eg_set_error(EG_ERR_INVALID, "device %d not available", opts->device);
    EG_CUDA(cudaSetDevice(opts->device));
    eg_batch *b = new eg_batch();
    b->device = opts->device;
    b->num_games = num_games;
    b->K = opts->thresholds;
    b->d = opts->scale;
    b->total_nodes = tn;
    b->total_edges = tm;
    b->block = opts->block ? opts->block : 1024;
    b->kg_cap = opts->group_max ? opts->group_max : 8;
    b->tail_rows = opts->tail_rows > 0 ? opts->tail_rows : 0;
    b->park_percent = opts->park_percent > 0 ? opts->park_percent : 10;
    b->tail_sweeps = opts->tail_sweeps > 0 ? opts->tail_sweeps : kTailSweeps;
    b->tail_cluster = opts->tail_cluster > 0 ? opts->tail_cluster : kTailCluster;
    b->max_rounds = opts->max_rounds;
    b->timeout_ms = opts->timeout_ms;
    b->use_graph = opts->use_graph != 0;
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
    eg_status s = unit_kernel_setup(b->device);
    if (s == EG_OK) s = b->launcher.init();
    if (s != EG_OK) {
        eg_batch_free(b);
        return s;
    }
    b->smem_budget = unit_smem_budget(b->device);
    /* pack every game on the host cores */
    b->hp.resize((size_t)num_games);
    std::vector<eg_status> ps((size_t)num_games, EG_OK);
    parallel_for(num_games, [&](int g) { ps[(size_t)g] = pack_game(games[g], &b->hp[(size_t)g]); });
    for (int g = 0; g < num_games; g++)
        if (ps[(size_t)g] != EG_OK) {
            eg_batch_free(b);
            return eg_set_error(ps[(size_t)g], "game %d could not be packed", g);
        }
    size_t pbytes = 0;
    std::vector<size_t> poff((size_t)num_games);
    b->f_off.assign((size_t)num_games + 1, 0);
    for (int g = 0; g < num_games; g++) {
        poff[(size_t)g] = pbytes;
        pbytes += packed_dev_bytes(b->hp[(size_t)g]);
        b->f_off[(size_t)g + 1] = b->f_off[(size_t)g] + (long long)b->hp[(size_t)g].n * b->K;
    }
    cudaError_t e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
    if (e != cudaSuccess) s = eg_set_error(EG_ERR_CUDA, "stream/event creation failed: %s", cudaGetErrorString(e));
    if (s == EG_OK) s = balloc(b, (char **)&b->dblock, pbytes);
    if (s == EG_OK) s = balloc(b, &b->F, (size_t)b->f_off[(size_t)num_games]);
    if (s == EG_OK) s = balloc(b, &b->p_dev, (size_t)num_games * b->K);
    if (s == EG_OK) s = balloc(b, &b->mg_dev, (size_t)num_games * b->K);
    if (s == EG_OK) s = balloc(b, &b->ctrl, 1);
    b->pd.resize((size_t)num_games);
    for (int g = 0; g < num_games && s == EG_OK; g++)
        s = packed_upload(b->hp[(size_t)g], (char *)b->dblock + poff[(size_t)g], b->st, &b->pd[(size_t)g]);
    if (s == EG_OK) {
        e = cudaStreamSynchronize(b->st);
        if (e != cudaSuccess) s = eg_set_error(EG_ERR_CUDA, "batch upload failed: %s", cudaGetErrorString(e));
    }
    if (s != EG_OK) {
        eg_batch_free(b);
        return s;
    }
    /* the device holds the slots now; the host keeps sizes and min weights */
    for (HostPacked &h : b->hp) {
        std::vector<uint32_t>().swap(h.e32);
        std::vector<int2>().swap(h.e64);
        std::vector<int>().swap(h.orig);
        std::vector<int>().swap(h.slice_off);
    }
    *out = b;
    return EG_OK;
}

/* Units of every game for the current thresholds, grouped by variant. */
static eg_status batch_plan(eg_batch *b)
{
    const int K = b->K;
    std::vector<UnitDesc> units;
    std::vector<int> ugame;
    std::vector<long long> cost;
    std::vector<size_t> gneed; /* global scratch bytes per unit (0: shared memory) */
    int smem = 16;
    for (int g = 0; g < b->num_games; g++) {
        const size_t before = units.size();
        EG_TRY(make_units(b->hp[(size_t)g], b->pd[(size_t)g], K, b->d, b->p_host.data() + (size_t)g * K,
                          b->mg_host.data() + (size_t)g * K, b->p_dev + (size_t)g * K, b->mg_dev + (size_t)g * K,
                          b->F + b->f_off[(size_t)g], b->smem_budget, b->kg_cap, &units, &gneed, &cost, &smem,
                          b->tail_rows));
        for (size_t i = before; i < units.size(); i++) ugame.push_back(g);
    }
    std::vector<int> perm;
    UnitSet S;
    group_units(units, cost, gneed, &S, &perm);
    const int nu = (int)S.units.size();
    size_t gbytes = 0;
    for (size_t x : S.gneed) gbytes += x;
    bool reallocated = false;
    if (nu > b->units_cap || gbytes > b->gscratch_bytes) {
        reallocated = true;
        batch_free_units(b);
        const size_t before = b->bytes;
        eg_status s = balloc(b, &b->units_dev, (size_t)nu);
        if (s == EG_OK) s = balloc(b, &b->u_rounds, (size_t)nu);
        if (s == EG_OK) s = balloc(b, &b->u_status, (size_t)nu);
        if (s == EG_OK && gbytes) s = balloc(b, (char **)&b->gscratch, gbytes);
        b->unit_bytes = b->bytes - before;
        if (s != EG_OK) {
            batch_free_units(b);
            return s;
        }
        b->units_cap = nu;
        b->gscratch_bytes = gbytes;
    }
    size_t goff = 0;
    b->unit_game.assign((size_t)nu, 0);
    for (int j = 0; j < nu; j++) {
        UnitDesc &u = S.units[(size_t)j];
        if (S.gneed[(size_t)j]) {
            u.gscratch = (char *)b->gscratch + goff;
            goff += S.gneed[(size_t)j];
        }
        u.rounds = b->u_rounds + j;
        u.status = b->u_status + j;
        b->unit_game[(size_t)j] = ugame[(size_t)perm[(size_t)j]];
    }
    const size_t tb = tail_bytes(S);
    if (tb > b->tails_bytes) {
        reallocated = true;
        if (b->tails) {
            cudaFree(b->tails);
            b->bytes -= b->tails_bytes;
            b->tails = nullptr;
            b->tails_bytes = 0;
        }
        EG_TRY(balloc(b, (char **)&b->tails, tb));
        b->tails_bytes = tb;
    }
    const size_t tsb = tail_scratch_bytes(S, b->sms);
    if (tsb > b->tscratch_bytes) {
        reallocated = true;
        if (b->tscratch) {
            cudaFree(b->tscratch);
            b->bytes -= b->tscratch_bytes;
            b->tscratch = nullptr;
            b->tscratch_bytes = 0;
        }
        EG_TRY(balloc(b, (char **)&b->tscratch, tsb));
        b->tscratch_bytes = tsb;
    }
    /* a captured graph stays valid when the plan is the same (the units read
     * their thresholds and MG from device memory at run time) */
    bool same = !reallocated && b->set.units.size() == S.units.size() &&
                memcmp(b->set.off, S.off, sizeof S.off) == 0 && memcmp(b->set.smem, S.smem, sizeof S.smem) == 0 &&
                memcmp(b->set.tail_cap, S.tail_cap, sizeof S.tail_cap) == 0 &&
                memcmp(b->set.tail_smem, S.tail_smem, sizeof S.tail_smem) == 0 &&
                memcmp(b->set.units.data(), S.units.data(), sizeof(UnitDesc) * S.units.size()) == 0;
    for (int c = 0; c < kTailClasses && same; c++)
        same = b->set.tail_init[c].size() == S.tail_init[c].size() &&
               memcmp(b->set.tail_init[c].data(), S.tail_init[c].data(), sizeof(TailEntry) * S.tail_init[c].size()) == 0;
    b->set = std::move(S);
    EG_CUDA(cudaMemcpyAsync(b->units_dev, b->set.units.data(), sizeof(UnitDesc) * (size_t)nu, cudaMemcpyHostToDevice,
                            b->st));
    TailList *tl = nullptr;
    EG_TRY(tail_upload(b->set, b->tails, b->st, &tl));
    EG_CUDA(cudaStreamSynchronize(b->st));
    if (!same) batch_drop_graph(b);
    return EG_OK;
}

extern "C" eg_status eg_batch_set_thresholds(eg_batch *b, const int32_t *p)
{
    if (!b || !p) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    EG_CUDA(cudaSetDevice(b->device));
    const int K = b->K;
    b->p_host.assign(p, p + (size_t)b->num_games * K);
    b->mg_host.assign((size_t)b->num_games * K, 0);
    parallel_for(b->num_games, [&](int g) {
        for (int k = 0; k < K; k++)
            b->mg_host[(size_t)g * K + k] = threshold_mg(b->hp[(size_t)g], p[(size_t)g * K + k], b->d);
    });
    EG_CUDA(cudaMemcpyAsync(b->p_dev, b->p_host.data(), sizeof(int) * b->p_host.size(), cudaMemcpyHostToDevice, b->st));
    EG_CUDA(cudaMemcpyAsync(b->mg_dev, b->mg_host.data(), sizeof(long long) * b->mg_host.size(), cudaMemcpyHostToDevice,
                            b->st));
    EG_TRY(batch_plan(b));
    b->thresholds_set = true;
    b->solved = false;
    return EG_OK;
}

static eg_status batch_enqueue(eg_batch *b, cudaStream_t st, int *grid)
{
    const unsigned long long tns = b->timeout_ms > 0 ? (unsigned long long)(b->timeout_ms * 1e6) : 0ull;
    return launch_unit_set(b->launcher, st, b->set, b->units_dev, (TailList *)b->tails, b->tscratch, b->ctrl, b->block,
                           b->sms, b->max_rounds, tns, grid, b->park_percent, b->tail_sweeps, b->tail_cluster);
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
            batch_drop_graph(b);
            /* capture on a side stream so that the timing events stay outside the graph */
            cudaStream_t cs;
            EG_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            EG_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
            eg_status s = batch_enqueue(b, cs, &grid);
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
            b->graph_grid = grid;
        } else {
            replay = true;
            grid = b->graph_grid;
        }
        EG_CUDA(cudaGraphLaunch(b->graph_exec, b->st));
    } else {
        EG_TRY(batch_enqueue(b, b->st, &grid));
    }
    EG_CUDA(cudaEventRecord(b->ev1, b->st));
    LaunchCtrl cv;
    const size_t nu = b->set.units.size();
    b->last_rounds.assign(nu, 0);
    b->last_status.assign(nu, 0);
    EG_CUDA(cudaMemcpyAsync(&cv, b->ctrl, sizeof cv, cudaMemcpyDeviceToHost, b->st));
    EG_CUDA(cudaMemcpyAsync(b->last_rounds.data(), b->u_rounds, sizeof(long long) * nu, cudaMemcpyDeviceToHost, b->st));
    EG_CUDA(cudaMemcpyAsync(b->last_status.data(), b->u_status, sizeof(int) * nu, cudaMemcpyDeviceToHost, b->st));
    EG_CUDA(cudaStreamSynchronize(b->st));
    UnitCtrl c;
    sum_ctrl(cv, &c);
    /* the two phases on the device clock */
    unsigned long long p1b = 0, p1e = 0, tb = 0, te = 0;
    for (int v = 0; v < kNumCtrl; v++) {
        const UnitCtrl &x = cv.c[v];
        if (!x.t_begin) continue;
        unsigned long long &b0 = v < kNumVariants ? p1b : tb, &e0 = v < kNumVariants ? p1e : te;
        if (!b0 || x.t_begin < b0) b0 = x.t_begin;
        e0 = std::max(e0, x.t_end);
    }
    TailList tls[kTailClasses];
    EG_CUDA(cudaMemcpy(tls, b->tails, sizeof tls, cudaMemcpyDeviceToHost));
    int tail_entries = 0;
    for (int t = 0; t < kTailClasses; t++) tail_entries += std::min(tls[t].count, tls[t].cap);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    b->solved = true;
    std::vector<char> gfail((size_t)b->num_games, 0);
    long long rmax = 0, rsum = 0;
    eg_status first = EG_OK;
    for (size_t i = 0; i < nu; i++) {
        rmax = std::max(rmax, b->last_rounds[i]);
        rsum += b->last_rounds[i];
        if (b->last_status[i] != EG_OK) {
            gfail[(size_t)b->unit_game[i]] = 1;
            if (first == EG_OK) first = (eg_status)b->last_status[i];
        }
    }
    int failed = 0;
    for (char f : gfail) failed += f;
    int smem = 0;
    for (int v = 0; v < kNumVariants; v++)
        if (b->set.off[v + 1] > b->set.off[v]) smem = std::max(smem, b->set.smem[v]);
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
        stats->num_units = (int32_t)nu;
        stats->smem_bytes = smem;
        stats->tail_entries = tail_entries;
        stats->phase1_ms = p1e > p1b ? (double)(p1e - p1b) * 1e-6 : 0.0;
        stats->tail_ms = te > tb ? (double)(te - tb) * 1e-6 : 0.0;
    }
    if (first != EG_OK) return eg_set_error(first, "%d game(s) stopped early (status %d)", failed, (int)first);
    return EG_OK;
}

extern "C" eg_status eg_batch_credits(eg_batch *b, int32_t game, int64_t *credits)
{
    if (!b || !credits || game < 0 || game >= b->num_games) return eg_set_error(EG_ERR_INVALID, "bad arguments");
    if (!b->solved) return eg_set_error(EG_ERR_INVALID, "batch not solved");
    EG_CUDA(cudaSetDevice(b->device));
    const long long cnt = b->f_off[(size_t)game + 1] - b->f_off[(size_t)game];
    EG_CUDA(cudaMemcpyAsync(credits, b->F + b->f_off[(size_t)game], sizeof(long long) * (size_t)cnt,
                            cudaMemcpyDeviceToHost, b->st));
    EG_CUDA(cudaStreamSynchronize(b->st));
    return EG_OK;
}

extern "C" eg_status eg_batch_game_result(eg_batch *b, int32_t game, int64_t *rounds, int32_t *status)
{
    if (!b || game < 0 || game >= b->num_games) return eg_set_error(EG_ERR_INVALID, "bad arguments");
    if (!b->solved) return eg_set_error(EG_ERR_INVALID, "batch not solved");
    long long r = 0;
    int s = EG_OK;
    for (size_t i = 0; i < b->set.units.size(); i++) {
        if (b->unit_game[i] != game) continue;
        r = std::max(r, b->last_rounds[i]);
        if (s == EG_OK && b->last_status[i] != EG_OK) s = b->last_status[i];
    }
    if (rounds) *rounds = r;
    if (status) *status = s;
    return EG_OK;
}

/* Autotuner: every candidate CTA size solves the planned batch under a
 * sweep cap (enough sweeps to reach the steady state, few enough to be
 * quick); the candidate with the most edge relaxations per second is kept.
 * The threshold group size stays as configured: a capped solve favours one
 * threshold per unit (more CTAs busy early), while the whole solve is faster
 * with groups of eight (each sweep of a unit relaxes eight thresholds, and
 * the long-running thresholds reach the cluster tail together). */
extern "C" eg_status eg_batch_tune(eg_batch *b, int32_t *block_out)
{
    if (!b) return eg_set_error(EG_ERR_INVALID, "batch is NULL");
    if (!b->thresholds_set) return eg_set_error(EG_ERR_INVALID, "thresholds not set");
    const int blocks[] = {512, 1024};
    const long long keep_cap = b->max_rounds;
    const bool keep_graph = b->use_graph;
    b->use_graph = false;
    b->max_rounds = 48;
    double best = -1.0;
    int best_block = b->block;
    for (int c : blocks) {
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
    EG_TRY(batch_plan(b));
    if (block_out) *block_out = best_block;
    if (best < 0) return eg_set_error(EG_ERR_CUDA, "no candidate ran");
    return EG_OK;
}
