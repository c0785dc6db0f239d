/*
 * eg_device.cuh -- device-side building blocks shared by the solver's CUDA
 * sources: the OMINUS operator, cache-controlled loads, the frontier bitmap,
 * and a bounded grid barrier for persistent cooperative kernels.
 */
#ifndef EG_DEVICE_CUH
#define EG_DEVICE_CUH

#include <cstdint>
#include <cuda_runtime.h>

#include "eg_internal.h"

#define EG_MAX_CLASSES 16

namespace eg {

template <class T> struct credit_traits;
template <> struct credit_traits<int32_t> { static constexpr int32_t top = INT32_MAX; };
template <> struct credit_traits<int64_t> { static constexpr int64_t top = INT64_MAX; };

/* OMINUS of reference src/common.h:270-272 / src/dev_EG_alg.cu:35-37:
 * a < TOP and a - b <= MG give max(0, a - b), anything else TOP.  The
 * difference is formed in 64 bits (identical to the reference's int
 * arithmetic whenever that does not overflow). */
template <class T>
__device__ __forceinline__ T ominus(T a, int32_t b, long long mg)
{
    const long long d = (long long)a - (long long)b;
    return (a < credit_traits<T>::top && d <= mg) ? (T)(d > 0 ? d : 0) : credit_traits<T>::top;
}

/* Credits are written by other SMs during a persistent solve: read them from
 * L2 (ld.global.cg) so that no stale L1 line survives a grid barrier. */
__device__ __forceinline__ int32_t ld_credit(const int32_t *p) { return __ldcg(p); }
__device__ __forceinline__ int64_t ld_credit(const int64_t *p) { return (int64_t)__ldcg((const long long *)p); }
__device__ __forceinline__ void st_credit(int32_t *p, int32_t v) { __stcg(p, v); }
__device__ __forceinline__ void st_credit(int64_t *p, int64_t v) { __stcg((long long *)p, (long long)v); }

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_volatile(const int *p) { return *(volatile const int *)p; }
__device__ __forceinline__ long long ld_volatile(const long long *p) { return *(volatile const long long *)p; }
__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p)
{
    return *(volatile const unsigned long long *)p;
}

/* Sets bit p of a frontier bitmap; returns true when this call set it.
 * The plain L2 read first filters the common case of an already-set bit. */
__device__ __forceinline__ bool bitmap_push(uint32_t *bm, int32_t p)
{
    const uint32_t mask = 1u << (p & 31);
    uint32_t *w = bm + (p >> 5);
    if (__ldcg(w) & mask) return false;
    return !(atomicOr(w, mask) & mask);
}

/* Sets bit p of a frontier bitmap.  Most pushes in a dense round find the
 * bit already set, so an L2 read filters them before the atomic: frontier
 * words are hot and atomics on one word serialise.  The atomic's result is
 * not needed (the caller decides "the next round has work" from the raise
 * itself), so it is issued as a reduction. */
__device__ __forceinline__ void bitmap_mark(uint32_t *bm, int32_t p)
{
    const uint32_t mask = 1u << (p & 31);
    uint32_t *w = bm + (p >> 5);
    if (!(__ldcg(w) & mask)) atomicOr(w, mask);
}

/* Pushes the four predecessors of one 128-bit load of a padded list;
 * returns how many were real (not padding). */
template <class Pol>
__device__ __forceinline__ unsigned push4(const Pol &pol, const int4 c)
{
    if (c.x >= 0) pol.push(c.x);
    if (c.y >= 0) pol.push(c.y);
    if (c.z >= 0) pol.push(c.z);
    if (c.w >= 0) pol.push(c.w);
    return (unsigned)(c.x >= 0) + (c.y >= 0) + (c.z >= 0) + (c.w >= 0);
}

/* Atomic min (OWNER 0) / max (OWNER 1) and exchange on credits. */
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

/* Control block of a persistent solve.  Counters that a round uses are
 * double-buffered by round parity and cleared by the barrier's last
 * arriver, so that no extra pass over them is needed. */
struct Ctrl {
    unsigned bar_count;                /* arrivals at the current barrier            */
    unsigned bar_gen;                  /* barrier generation                         */
    int ctr[2][EG_MAX_CLASSES];        /* per-round work-grab counters per class     */
    int flag[2];                       /* "round r has work", set during round r-1  */
    int stop;                          /* 0 running; else an eg_status               */
    int abort;                         /* a CTA gave up waiting                      */
    long long rounds;                  /* rounds completed                           */
    unsigned long long lifts;          /* vertices lifted                            */
    unsigned long long edges;          /* real out-edges scanned                     */
    unsigned long long t_start;        /* globaltimer at kernel start                */
    unsigned long long wait_site;      /* diagnostic: round at which a wait gave up  */
    unsigned long long num_top;        /* vertices at TOP after the solve            */
    unsigned long long changes;        /* lifts that raised a credit                 */
    unsigned long long pushes;         /* predecessor entries scanned                */
    /* phase timers (diagnostic mode): warp-nanoseconds summed over warps and
     * rounds in heavy tasks, in word classes, and waiting at the barrier */
    unsigned long long t_heavy, t_light, t_wait;
    /* round kinds (lean kernel): raises of round r by parity, the kind the
     * last arriver picked for the next round, and dense rounds run */
    unsigned long long round_changes[2];
    int next_mode;
    int pad2;
    long long dense_rounds;
    unsigned long long dense_changes;
    unsigned long long round_max[2];   /* diagnostic: slowest slice of a dense round */
    unsigned long long t_round_prev;   /* diagnostic: globaltimer at the last round end */
};

/* Grid barrier for a cooperative launch.  Every wait is bounded by
 * wait_limit_ns of globaltimer time; a CTA that gives up records
 * EG_ERR_TIMEOUT and raises abort so the other CTAs stop waiting too.  The
 * last arriver runs `last()` (single thread) before releasing the grid.
 * Returns false when the solve must stop (abort raised). */
template <class F>
__device__ __forceinline__ bool grid_barrier(Ctrl *c, unsigned long long wait_limit_ns, F last)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned gen = ld_acquire_gpu(&c->bar_gen);
        __threadfence();
        const unsigned prev = atomicAdd(&c->bar_count, 1u);
        if (prev == gridDim.x - 1) {
            c->bar_count = 0;
            __threadfence(); /* order the other CTAs' round writes before last() reads them */
            last();
            __threadfence();
            st_release_gpu(&c->bar_gen, gen + 1);
        } else {
            const unsigned long long t0 = globaltimer_ns();
            unsigned spins = 0;
            while (ld_acquire_gpu(&c->bar_gen) == gen) {
                if (++spins > 64) __nanosleep(64);
                if ((spins & 255) == 0) {
                    if (ld_volatile(&c->abort)) { ok = 0; break; }
                    if (globaltimer_ns() - t0 > wait_limit_ns) {
                        atomicCAS(&c->stop, 0, (int)EG_ERR_TIMEOUT);
                        atomicExch(&c->abort, 1);
                        c->wait_site = (unsigned long long)c->rounds;
                        ok = 0;
                        break;
                    }
                }
            }
        }
        __threadfence();
        if (ld_volatile(&c->abort)) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace eg

#endif
