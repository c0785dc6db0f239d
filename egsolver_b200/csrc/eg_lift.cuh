/*
 * eg_lift.cuh -- parameters of the persistent lifting kernel.
 */
#ifndef EG_LIFT_CUH
#define EG_LIFT_CUH

#include "eg_device.cuh"

namespace eg {

/* Most sweeps of the edge stream per grid barrier in dense rounds (one bank
 * of cut-vertex accumulators each). */
constexpr int kMaxDenseSweeps = 4;

/* Lane-group sizes of the lifting variants; EG_GROUP_CTA lifts one vertex
 * with the whole CTA. */
enum { EG_GROUP_CTA = 0, EG_GROUP_LIGHT = 64 };

struct LiftClass {
    int word_begin, word_end;  /* frontier words of the class              */
    int owner;                 /* 0: min (player 0), 1: max (player 1)      */
    int group;                 /* lanes per vertex: 1..32, or EG_GROUP_CTA  */
    int grab;                  /* frontier words taken per work grab        */
};

struct LiftParams {
    const int *P;              /* padded row offsets, n_pad + 1             */
    const int4 *E4;            /* edge pairs {succ, w, succ, w}             */
    const int *CP;             /* predecessor offsets, n_pad + 1            */
    const int *CS;             /* predecessor ids                           */
    void *F;                   /* credits (int32 or int64), n_pad + 64      */
    uint32_t *B0, *B1;         /* frontier bitmaps                          */
    Ctrl *ctrl;
    long long mg;
    long long max_rounds;      /* < 0: no cap                               */
    unsigned long long timeout_ns;     /* 0: none                           */
    unsigned long long wait_limit_ns;  /* bound of every barrier wait       */
    const int *cancel;         /* device view of a mapped host flag, or 0   */
    int n_pad;                 /* ids >= n_pad are the padding sentinels    */
    int nclasses;
    LiftClass cls[EG_MAX_CLASSES];
    /* heavy vertices (ids >= heavy_begin) cut into edge tasks */
    const int4 *tasks;         /* {vertex, first pair, end pair, (ntasks << 1) | owner } */
    int num_tasks;
    int heavy_begin;
    void *hacc;                /* per heavy vertex: partial min / max (credit type) */
    int *hrem;                 /* per heavy vertex: tasks still to report          */
    int profile;               /* non-zero: accumulate the phase timers of Ctrl    */
    int lean;                  /* AUTO layout: use the lean kernel instantiation   */
    /* round kinds (lean layout): frontier rounds in k_lift, rounds over
     * every vertex in k_lift_dense; the host alternates the two launches */
    uint32_t *CH0, *CH1;       /* vertices raised in a recording dense round, by parity */
    long long dense_min_changes, sparse_max_changes;
    int direction;             /* eg_direction                                     */
    /* the dense kernel's pair stream: E4 cut into equal slices of `slice`
     * pairs (a multiple of 32), one per warp */
    const uint16_t *PM;        /* per pair: owner << 15 | last pair of its vertex << 14
                                  | vertex - CB[pair / 32]                        */
    const int *CB;             /* per 32-pair chunk: the vertex of its first pair  */
    int npairs;                /* pairs in E4                                      */
    int slice;                 /* pairs per warp                                   */
    void *dacc;                /* per vertex cut by slice edges: partial min / max */
    int *drem;                 /* per cut vertex: slices still to report           */
    const int2 *E8;            /* the pairs packed in 8 bytes, or null             */
    int wbits, wbias;          /* packed edge: (succ << wbits) | (w + wbias)       */
    int fast32;                /* 32-bit credits whose differences fit 32 bits     */
    int dense_depth;           /* chunks in flight per warp: 1 (3 CTAs per SM) or 2 */
    int dense_sweeps;          /* sweeps of every slice per grid barrier: 1 .. 4    */
};

/* Round kinds, as Ctrl::next_mode holds them between rounds and launches. */
enum { ROUND_SPARSE = 0, ROUND_DENSE = 1, ROUND_SEED = 2, ROUND_RECORD = 3, ROUND_DONE = 4 };

/* Stop conditions checked by a round's last arriver when work is left: the
 * round cap, the timeout, and (every 64 rounds) the cancel flag. */
__device__ __forceinline__ void check_stop(const LiftParams &p, Ctrl *c, long long round)
{
    if (p.max_rounds >= 0 && round + 1 >= p.max_rounds) {
        c->stop = (int)EG_ERR_LOOPCAP;
    } else if (p.timeout_ns && globaltimer_ns() - c->t_start > p.timeout_ns) {
        c->stop = (int)EG_ERR_TIMEOUT;
    } else if (p.cancel && (round & 63) == 0 && ld_volatile(p.cancel)) {
        c->stop = (int)EG_ERR_CANCELLED;
    }
}

/* Edge pairs per heavy task (256 edges). */
constexpr int kTaskPairs = 128;

/* Cooperative launch of the persistent lifting kernel on `st`; *grid gets
 * the number of CTAs used. */
eg_status launch_lift(const LiftParams &p, int credit_bits, cudaStream_t st, int *grid, int *block, int max_ctas);
/* One-CTA launch for small games (frontier in shared memory). */
eg_status launch_lift_cta(const LiftParams &p, int credit_bits, cudaStream_t st);
/* Cooperative launch of the dense-round kernel (eg_dense.cu) with `grid`
 * CTAs of 512 threads: the grid that p.slice was computed for. */
eg_status launch_lift_dense(const LiftParams &p, int credit_bits, cudaStream_t st, int grid);
/* CTAs of a full-occupancy dense launch of pipeline depth 1 or 2, at most
 * max_ctas when > 0. */
eg_status dense_grid(int credit_bits, int depth, int max_ctas, int *grid);
/* Pair-stream metadata PM / CB of a prepared layout; *err (device) is
 * raised when a chunk's vertex offsets do not fit 14 bits. */
struct ClassTable;
void build_pair_meta(const int *P, int n_pad, int npairs, const ClassTable &ct, uint16_t *PM, int *CB, int *err,
                     cudaStream_t st);
/* Packs the 16-byte pairs of E4 into 8 bytes (E8). */
void launch_pack_pairs(const int4 *E4, int npairs, int wbits, int wbias, int2 *E8, cudaStream_t st);
/* Per-solve reporter counts of the vertices cut by slice edges. */
void launch_dense_setup(const LiftParams &p, int credit_bits, cudaStream_t st);

}  // namespace eg

#endif
