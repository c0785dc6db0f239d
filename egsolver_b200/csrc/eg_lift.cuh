/*
 * eg_lift.cuh -- parameters of the persistent lifting kernel.
 */
#ifndef EG_LIFT_CUH
#define EG_LIFT_CUH

#include "eg_device.cuh"

namespace eg {

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
    /* direction switching (lean kernel): a round is dense (every vertex
     * lifted, no frontier) after >= dense_min_changes raises, and goes back to
     * the frontier below sparse_max_changes raises */
    uint32_t *CH0, *CH1;       /* raised-in-round bitmaps, by parity               */
    long long dense_min_changes, sparse_max_changes;
    int direction;             /* 0 switch, 1 sparse only, 2 dense only           */
    int light_word_end;        /* words [0, light_word_end) are light             */
    int words;                 /* frontier words                                  */
};

/* Edge pairs per heavy task (256 edges). */
constexpr int kTaskPairs = 128;

/* Cooperative launch of the persistent lifting kernel on `st`; *grid gets
 * the number of CTAs used. */
eg_status launch_lift(const LiftParams &p, int credit_bits, cudaStream_t st, int *grid, int *block, int max_ctas);
/* One-CTA launch for small games (frontier in shared memory). */
eg_status launch_lift_cta(const LiftParams &p, int credit_bits, cudaStream_t st);

}  // namespace eg

#endif
