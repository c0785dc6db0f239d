/*
 * egsolver_b200_serve.h -- serving API of the B200 energy-game solver:
 * mean-payoff threshold queries with continuous batching.  Part of the same
 * library (libegsolver_b200.so) as egsolver_b200.h.
 */
#ifndef EGSOLVER_B200_SERVE_H
#define EGSOLVER_B200_SERVE_H

#include "egsolver_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Serving: mean-payoff threshold queries with continuous batching      */
/* ------------------------------------------------------------------ */

/* New (the reference is a one-shot command-line program).  A server owns a
 * worker thread that admits queries by free device memory, keeps every
 * admitted game's packed layout resident on the device across its queries, and
 * launches whatever is admitted as one micro-batch while earlier
 * micro-batches still run on other streams, so that their work overlaps on
 * the GPU.  Games of at most 2^19 vertices run in the unit kernel (one CTA
 * per game x group of thresholds, credits in shared memory); larger games,
 * and games whose credits miss shared memory while the queue is shallow,
 * run one threshold at a time on the persistent grid solver with at most
 * `large_ctas` CTAs, which leaves the remaining SMs to the micro-batches. */
typedef struct eg_server eg_server;

typedef struct eg_serve_opts {
    int32_t device;
    int32_t max_inflight;        /* queries admitted at once (0 = 1024)              */
    int32_t streams;             /* micro-batches in flight at once (0 = 4)          */
    int32_t block;               /* threads per CTA of the batched kernel (0 = 1024) */
    int64_t hbm_reserve_bytes;   /* device memory admission leaves free (0 = 1 GiB)  */
    int64_t max_rounds;          /* per query; < 0: no cap                           */
    int32_t large_ctas;          /* CTAs of the grid solver for large games (0: 148)  */
    int32_t reserved[5];
} eg_serve_opts;

typedef struct eg_serve_stats {
    int64_t submitted, admitted, completed, failed;
    int64_t games_registered, games_resident, game_uploads, evictions;
    int64_t micro_batches, threshold_solves;
    double  latency_p50_ms, latency_p99_ms, latency_mean_ms, latency_max_ms;
    double  elapsed_s, queries_per_s, solves_per_s;
    int64_t device_bytes;
    int32_t reserved[6];
} eg_serve_stats;

/* Device-clock span of one micro-batch (one launch of the unit kernel):
 * from its first CTA's start to its last CTA's end, in ms since the first
 * micro-batch's start.  Spans of different micro-batches that intersect
 * show their work overlapping on the GPU. */
typedef struct eg_serve_span {
    int64_t batch;               /* micro-batch number, from 0                */
    int32_t queries, units;
    double  begin_ms, end_ms;
} eg_serve_span;

/* Query states reported by eg_serve_poll. */
#define EG_QUERY_QUEUED 0
#define EG_QUERY_RUNNING 1
#define EG_QUERY_DONE 2
#define EG_QUERY_FAILED 3

eg_status eg_serve_create(const eg_serve_opts *opts, eg_server **out);
/* Registers a game (copied; uploaded when a query of it is admitted). */
eg_status eg_serve_add_game(eg_server *s, const eg_game *game, int64_t *game_id);
/* Drops a game once no query of it is pending; frees its device memory. */
eg_status eg_serve_remove_game(eg_server *s, int64_t game_id);
/* Queues "credits of every vertex of game_id for thresholds p[0..K-1] with
 * scale d" (weights w*d - p_k); returns at once. */
eg_status eg_serve_submit(eg_server *s, int64_t game_id, const int32_t *p, int32_t K, int32_t d, int64_t *query_id);
eg_status eg_serve_poll(eg_server *s, int64_t query_id, int32_t *state, double *latency_ms);
/* Blocks until the query finished or timeout_ms passed (EG_ERR_TIMEOUT). */
eg_status eg_serve_wait(eg_server *s, int64_t query_id, double timeout_ms);
/* Credits of a finished query, threshold-major (credits[k * n + v]); the
 * query's storage is released afterwards.  *rounds may be NULL. */
eg_status eg_serve_result(eg_server *s, int64_t query_id, int64_t *credits, int64_t *rounds);
eg_status eg_serve_stats_get(eg_server *s, eg_serve_stats *stats);
/* Copies up to cap spans of finished micro-batches; *count receives how
 * many were recorded. */
eg_status eg_serve_trace(eg_server *s, eg_serve_span *spans, int32_t cap, int32_t *count);
/* Stops the worker after the queued queries finished and frees everything. */
eg_status eg_serve_destroy(eg_server *s);

#ifdef __cplusplus
}
#endif

#endif /* EGSOLVER_B200_SERVE_H */
