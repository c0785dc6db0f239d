/*
 * egsolver_b200.h -- C-ABI of the B200 energy-game solver.
 *
 * An energy game is a directed graph whose vertices belong to player 0 or
 * player 1 and whose edges carry integer weights.  For every vertex v the
 * solver computes the minimal initial credit f(v): the least value that the
 * lifting operator of Brim, Chaloupka, Doyen, Gentilini and Raskin reaches
 * from f = 0,
 *
 *     f(v) = min_{(v,w)} OMINUS(f(w), wt(v,w))   if v belongs to player 0
 *     f(v) = max_{(v,w)} OMINUS(f(w), wt(v,w))   if v belongs to player 1
 *     OMINUS(a, b) = (a < TOP && a - b <= MG) ? max(0, a - b) : TOP
 *     MG = sum_v max(0, -min_{(v,w)} wt(v,w))
 *
 * TOP marks a vertex from which player 0 cannot keep the energy non-negative
 * with any finite credit.  Player 0 is the owner the reference text format
 * calls MAX (reference: src/the_parser.y:87), player 1 is MIN (:88); the
 * operator is the macro OMINUS of reference src/common.h:270-272.
 *
 * Every result is bit-exact against the reference CPU solver
 * (reference src/cpu_solver.c:190-333): the least fixed point is unique, so
 * any fair schedule of lifts reaches the same f.
 *
 * All entry points return an eg_status; none calls exit().  Buffers are owned
 * by the caller unless an entry point says otherwise.  No torch type appears
 * in any signature.
 */
#ifndef EGSOLVER_B200_H
#define EGSOLVER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EG_ABI_VERSION 1

/* TOP as stored in 32-bit credits: INT_MAX, the value the reference prints
 * for an unbounded credit (reference src/common.h:271, src/egsolver.c:103). */
#define EG_TOP32 ((int32_t)2147483647)
/* TOP as stored in 64-bit credits. */
#define EG_TOP64 ((int64_t)9223372036854775807LL)

typedef enum eg_status {
    EG_OK = 0,
    EG_ERR_INVALID = 1,      /* malformed game or option (message in eg_last_error) */
    EG_ERR_CUDA = 2,         /* a CUDA call failed (message in eg_last_error)       */
    EG_ERR_OOM = 3,          /* device or host allocation failed / admission denied */
    EG_ERR_TIMEOUT = 4,      /* opts.timeout_ms expired or a device wait ran out    */
    EG_ERR_OVERFLOW = 5,     /* MG does not fit the chosen credit width             */
    EG_ERR_LOOPCAP = 6,      /* opts.max_rounds reached with work left (partial f)  */
    EG_ERR_CANCELLED = 7,    /* the cancel flag was raised                          */
    EG_ERR_NO_DEVICE = 8,    /* no CUDA device, or not an sm_100 device             */
    EG_ERR_BUSY = 9,         /* serving queue full                                  */
    EG_ERR_NOT_FOUND = 10,   /* unknown request / game handle                       */
    EG_ERR_IO = 11           /* file could not be read or parsed                    */
} eg_status;

/* Kernel variants for the lifting step, per out-degree bucket.  The names
 * follow the reference's kinds of parallelism (reference src/common.h:195-202,
 * --shuffling K): one thread per vertex, a group of lanes per vertex with
 * shuffle min/max reductions, and (new) one CTA per vertex. */
typedef enum eg_variant {
    EG_VARIANT_AUTO = 0,     /* autotuned per degree bucket                          */
    EG_VARIANT_THREAD = 1,   /* thread-per-vertex  (reference --shuffling 1)         */
    EG_VARIANT_WARP = 2,     /* warp-per-vertex, __shfl reductions (--shuffling 32) */
    EG_VARIANT_CTA = 3,      /* CTA-per-vertex for high out-degree                   */
    EG_VARIANT_SMEM = 4      /* whole game resident in one CTA's shared memory       */
} eg_variant;

/* Round kinds of the lean grid kernel (eg_opts.direction).  A sparse round
 * lifts the frontier and pushes predecessors of raised vertices, as the
 * reference's worklist does; a dense round lifts every vertex and pushes
 * nothing.  Both are fair chaotic iterations of the same operator, so the
 * credits do not depend on the choice. */
typedef enum eg_direction {
    EG_DIRECTION_SWITCH = 0, /* dense while many credits rise, sparse otherwise      */
    EG_DIRECTION_SPARSE = 1,
    EG_DIRECTION_DENSE = 2
} eg_direction;

/* A game in compressed sparse row form, vertices 0..num_nodes-1.
 * Owners are given either by a split index (the reference layout:
 * vertices [0, num_nodes0) belong to player 0, the rest to player 1;
 * reference src/egsolver.c:253-281, counter_nodi0) when owner == NULL, or by
 * a per-vertex owner array (0 or 1) when owner != NULL.  Every vertex must
 * have at least one successor, as in the reference. */
typedef struct eg_game {
    int32_t num_nodes;
    int32_t num_nodes0;          /* used only when owner == NULL           */
    int64_t num_edges;
    const int64_t *row_ptr;      /* num_nodes + 1 offsets into succ/weight */
    const int32_t *succ;         /* num_edges successor ids                */
    const int32_t *weight;       /* num_edges edge weights                 */
    const uint8_t *owner;        /* optional, num_nodes entries            */
} eg_game;

typedef struct eg_opts {
    int32_t credit_bits;         /* 32, 64, or 0 = 64                                 */
    int32_t variant;             /* eg_variant; AUTO picks per bucket                 */
    int32_t small_max_deg;       /* bucket bound: deg <= this -> small bucket (0=auto) */
    int32_t large_min_deg;       /* bucket bound: deg >= this -> large bucket (0=auto) */
    int64_t max_rounds;          /* <0: no cap (reference default n*m*MG+1)           */
    double  timeout_ms;          /* <=0: none; checked on the device every round      */
    volatile int32_t *cancel;    /* optional flag from eg_cancel_flag_alloc()         */
    int32_t device;              /* CUDA device ordinal                                */
    int32_t lanes_per_vertex;    /* with EG_VARIANT_WARP: 2,4,8,16 or 32 lanes per
                                    vertex (reference --shuffling K); 0 means 32       */
    int32_t keep_layout;         /* non-zero: reuse the transpose/renumbering of the
                                    previous solve of the same resident game           */
    int32_t grid_ctas;           /* cap on the lifting grid's CTAs (0: every SM, full
                                    occupancy); a smaller grid leaves SMs to other work */
    int32_t task_edges;          /* edges per task of a heavy vertex, 32..256 (0: 256) */
    int32_t schedule;            /* light words: 0 dealt evenly to warps, 1 taken in
                                    increasing order from a counter                   */
    int32_t profile;             /* non-zero: report the kernel's phase timers        */
    int32_t ctas_per_sm;         /* AUTO layout: 3 = lean kernel at three CTAs per SM,
                                    2 = full kernel at two (0: 3)                     */
    int32_t direction;           /* lean kernel rounds: 0 switch between frontier
                                    (sparse) and full (dense) rounds, 1 sparse only,
                                    2 dense only                                      */
    int32_t dense_permille;      /* a round after >= this many raises per thousand
                                    vertices is dense (0: 40)                         */
    int32_t sparse_permille;     /* a dense round with fewer raises per thousand
                                    vertices is followed by sparse ones (0: 15)       */
    int32_t narrow;              /* non-zero: a 64-bit solve computes in 32 bits when
                                    MG + max |weight| < 2^31 - 1 (identical credits;
                                    eg_dgame_credits_device then reports 32)          */
    int32_t wide_pairs;          /* non-zero: dense rounds read 16-byte edge pairs
                                    even when successor and weight fit 32 bits        */
    int32_t dense_depth;         /* chunks in flight per warp in dense rounds: 1 (three
                                    CTAs per SM) or 2 (two CTAs per SM); 0: 2         */
    int32_t dense_sweeps;        /* sweeps of the edge stream per grid barrier in dense
                                    rounds: 1 to 4; 0: 4                              */
} eg_opts;

typedef struct eg_stats {
    int64_t mg;                  /* MG of the game (reference MG_pesi)                */
    int64_t rounds;              /* synchronous rounds run on the device              */
    int64_t lifts;               /* vertices lifted (reference processedNodes)        */
    int64_t edges;               /* sum of out-degrees of lifted vertices             */
    int64_t num_top;             /* vertices whose credit is TOP                       */
    double  solve_ms;            /* device time of the solve (transpose included)    */
    double  lift_ms;             /* device time of the lifting loop alone            */
    int64_t kernel_launches;     /* kernels launched by the solve                     */
    int32_t credit_bits;         /* width of the credits on the device                 */
    int32_t variant_small, variant_mid, variant_large; /* variants used per bucket   */
    int32_t small_max_deg, large_min_deg;               /* bucket bounds used         */
    int64_t changes;             /* lifts that raised a credit                        */
    int64_t pushes;              /* predecessor entries scanned after those raises    */
    int32_t grid, block;         /* launch shape of the lifting kernel                */
    int32_t dense_rounds;        /* sweeps that lifted every vertex (no frontier); a
                                    dense round is dense_sweeps sweeps               */
    int32_t dense_launches;      /* launches of the dense-round kernel                */
    /* with opts.profile, in nanoseconds.  Frontier rounds only: mean time per
     * warp and round in heavy tasks, in word classes, and waiting at the round
     * barrier.  With dense rounds: the slowest slice per dense round (heavy),
     * the mean slice per warp (light), and the mean round-to-round time (wait) */
    double  phase_heavy_ns, phase_light_ns, phase_wait_ns;
    double  dense_ms;            /* device time of the dense-round kernel's launches  */
    int64_t dense_changes;       /* credits raised in dense rounds                    */
} eg_stats;

/* ------------------------------------------------------------------ */
/* Library and device                                                   */
/* ------------------------------------------------------------------ */

/* Message of the last failing call on this thread (never NULL). */
const char *eg_last_error(void);
/* EG_ABI_VERSION of the loaded library. */
int32_t eg_abi_version(void);
/* Fills opts with defaults: 64-bit credits, autotuned variants, no cap. */
void eg_opts_default(eg_opts *opts);
/* Number of usable sm_100 devices (0 when none). */
eg_status eg_device_count(int32_t *count);

/* ------------------------------------------------------------------ */
/* Host-side helpers that mirror the reference's preprocessing          */
/* ------------------------------------------------------------------ */

/* MG = sum over vertices of max(0, -(min out-weight)).  Mirrors
 * reference src/egsolver.c:283-304; returns EG_ERR_OVERFLOW when
 * limit_bits == 32 and the sum exceeds INT_MAX, like the reference's
 * "too high weights" exit. */
eg_status eg_compute_mg(const eg_game *game, int32_t limit_bits, int64_t *mg);

/* Round cap used by the reference when none is given:
 * n*m*MG+1, or LONG_MAX-1 on overflow (reference src/egsolver.c:64-90). */
int64_t eg_default_max_loop(int64_t num_edges, int64_t num_nodes, int64_t mg, int64_t max_loop);

/* Checks the CSR: offsets monotone, ids in range, no vertex without a
 * successor, owner values 0/1. */
eg_status eg_validate(const eg_game *game);

/* ------------------------------------------------------------------ */
/* One-call solve (host buffers in, host buffers out)                   */
/* ------------------------------------------------------------------ */

/* Copies the game to the device, transposes it, lifts to the least fixed
 * point and copies the credits back.  Replaces the reference's
 * copia_dati_su_device + gpu_solver + result copy
 * (reference src/dev_solver.cu:81-139, :142-149).  credits has num_nodes
 * entries; TOP is EG_TOP32 / EG_TOP64. */
eg_status eg_solve_i32(const eg_game *game, const eg_opts *opts, int32_t *credits, eg_stats *stats);
eg_status eg_solve_i64(const eg_game *game, const eg_opts *opts, int64_t *credits, eg_stats *stats);

/* ------------------------------------------------------------------ */
/* Device-resident games (inputs already in HBM)                        */
/* ------------------------------------------------------------------ */

typedef struct eg_dgame eg_dgame;

/* Uploads a host game: allocates device memory for its CSR and all solve
 * state.  The handle keeps them resident until eg_dgame_free. */
eg_status eg_dgame_upload(const eg_game *game, const eg_opts *opts, eg_dgame **out);
/* Same, from a CSR that is already in device memory (pointers are device
 * pointers; owner may be NULL).  The arrays are copied, not adopted. */
eg_status eg_dgame_from_device(const eg_game *dev_game, const eg_opts *opts, eg_dgame **out);
/* Solves a resident game from f = 0: transpose, bucket, init, lift.  The
 * credits stay on the device; stats are filled. */
eg_status eg_dgame_solve(eg_dgame *g, const eg_opts *opts, eg_stats *stats);
/* Copies the credits of the last solve to the host (original vertex ids). */
eg_status eg_dgame_credits_i32(eg_dgame *g, int32_t *credits);
eg_status eg_dgame_credits_i64(eg_dgame *g, int64_t *credits);
/* Device pointer to the credits of the last solve, in original vertex order
 * (int32 or int64 as solved); valid until the next solve or free. */
eg_status eg_dgame_credits_device(eg_dgame *g, void **dev_ptr, int32_t *credit_bits);
/* Device bytes held by the handle. */
int64_t eg_dgame_device_bytes(const eg_dgame *g);

/* Autotuner of the AUTO layout (new; the reference picks its kernel from the
 * command line).  Times capped solves (`rounds` rounds each, from f = 0) of
 * the resident game, one knob at a time per degree bucket and round kind:
 * the light/heavy out-degree bound (large_min_deg), the heavy vertices'
 * task size (task_edges), the thread-per-vertex bucket (small_max_deg), the
 * sweeps per dense round and the chunks in flight per warp (dense_sweeps,
 * dense_depth); a value is kept when it lifts edges at least 2% faster.
 * *tuned receives base with the chosen knobs.  The choice is cached per
 * game shape (size and out-degree histogram), so a later game of the same
 * shape takes it without timing.  Every setting gives the same credits. */
typedef struct eg_tune_report {
    int32_t candidates;          /* capped solves timed                               */
    int32_t from_cache;          /* 1: the choice came from the shape cache           */
    double  default_rate;        /* edge relaxations per ms with base's settings      */
    double  best_rate;           /* with the chosen settings                          */
    int32_t reserved[4];
} eg_tune_report;
eg_status eg_dgame_tune(eg_dgame *g, const eg_opts *base, int64_t rounds, eg_opts *tuned, eg_tune_report *rep);
void eg_dgame_free(eg_dgame *g);

/* ------------------------------------------------------------------ */
/* CSR -> CSC transpose (the reference's csr2csc / host_csr2csc)        */
/* ------------------------------------------------------------------ */

/* Deterministic counting-sort transpose on the device of a host CSR:
 * csc_ptr (n+1), csc_src (m), csc_val (m) come out array-equal to the
 * reference's host_csr2csc (reference src/host_csr2csc.c:15-46): within
 * each column the entries keep their source order.  Replaces
 * cusparseScsr2csc (reference src/csr2csc.cu:54-66). */
eg_status eg_csr2csc_i32(int32_t num_rows, int32_t num_cols, int64_t nnz,
                         const int64_t *row_ptr, const int32_t *col_idx, const int32_t *val,
                         int64_t *csc_ptr, int32_t *csc_row, int32_t *csc_val);

/* ------------------------------------------------------------------ */
/* Batched solving: many games x K thresholds in one persistent launch  */
/* ------------------------------------------------------------------ */

/* A mean-payoff query "is the mean payoff of v at least p/d?" is the
 * energy game with weights w*d - p (new; the reference solves one energy
 * game per process).  A batch packs many games into one device-resident
 * layout; one persistent launch then solves every (game, threshold) pair.
 * The work is cut into units of one game at a group of 1, 2, 4 or 8
 * thresholds, one CTA per unit with the unit's credits in shared memory,
 * taken from a device queue heaviest first.  When the queue runs dry, the
 * units still running hand their open thresholds to a cluster tail: each
 * (game, threshold) on a thread-block cluster whose CTAs each hold a
 * replica of its credits. */
#define EG_BATCH_MAX_K 32

typedef struct eg_batch eg_batch;

typedef struct eg_batch_opts {
    int32_t thresholds;          /* K thresholds per game, 1..EG_BATCH_MAX_K        */
    int32_t scale;               /* d >= 1: threshold p turns w into w*d - p        */
    int32_t block;               /* threads per CTA (64..1024); 0 = 1024 (eg_batch_tune picks 512 or 1024) */
    int32_t device;
    int64_t max_rounds;          /* per game; < 0: no cap                           */
    double  timeout_ms;          /* per launch; <= 0: none                          */
    int32_t use_graph;           /* non-zero: the solve's launches are captured in a
                                    CUDA graph on the first solve and replayed      */
    int32_t group_max;           /* most thresholds per work unit: 1, 2, 4 or 8
                                    (0: 8)                                          */
    int32_t tail_rows;           /* games of at least this many vertices go straight
                                    to the cluster tail (0: none)                   */
    int32_t park_percent;        /* running units move to the cluster tail once this
                                    share of phase-1 CTAs is idle (0: 10; above 100:
                                    never)                                          */
    int32_t tail_sweeps;         /* sweeps a cluster CTA runs between two cluster
                                    barriers in the tail, 1..16 (0: 4)              */
    int32_t tail_cluster;        /* CTAs per tail cluster: 1, 2, 4, 8 or 16 (0: 16;
                                    halved down to 8 where it cannot be scheduled) */
    int32_t reserved[2];
} eg_batch_opts;

typedef struct eg_batch_stats {
    int32_t num_games, thresholds;
    int64_t total_nodes, total_edges;
    int64_t rounds_max, rounds_sum;  /* over games                                   */
    int64_t lifts;                   /* vertex lifts (all K thresholds at once)       */
    int64_t edges;                   /* edge relaxations summed over the K thresholds */
    int64_t num_top;                 /* (vertex, threshold) pairs at TOP              */
    double  solve_ms;                /* device time of the launch                     */
    int32_t block, grid, games_failed, graph_replayed;
    int32_t num_units;               /* work units (game x threshold group)           */
    int32_t smem_bytes;              /* dynamic shared memory per CTA                 */
    int32_t tail_entries;            /* (unit, threshold) pairs the cluster tail ran  */
    int32_t reserved[1];
    double  phase1_ms;               /* device clock: first to last phase-1 CTA       */
    double  tail_ms;                 /* device clock: first to last tail CTA          */
} eg_batch_stats;

/* Packs the games (each in eg_game form; all at most 2^19 vertices) on the
 * host cores and uploads them. */
eg_status eg_batch_create(const eg_game *games, int32_t num_games, const eg_batch_opts *opts, eg_batch **out);
/* Thresholds p[g*K + k] for every game g and threshold k; plans the work
 * units (credit width and threshold groups per game). */
eg_status eg_batch_set_thresholds(eg_batch *b, const int32_t *p);
/* Solves every (game, threshold); credits stay on the device. */
eg_status eg_batch_solve(eg_batch *b, eg_batch_stats *stats);
/* Credits of one game, threshold-major: credits[k * n_g + v] (TOP = EG_TOP64). */
eg_status eg_batch_credits(eg_batch *b, int32_t game, int64_t *credits);
/* Per-game outcome of the last solve: sweeps (the most of its units) and an
 * eg_status. */
eg_status eg_batch_game_result(eg_batch *b, int32_t game, int64_t *rounds, int32_t *status);
/* Autotuner: times the candidate CTA sizes on the whole batch under a
 * sweep cap and keeps the fastest for later solves (*block receives the CTA
 * size); the threshold group size stays as configured. */
eg_status eg_batch_tune(eg_batch *b, int32_t *block);
int64_t eg_batch_device_bytes(const eg_batch *b);
void eg_batch_free(eg_batch *b);

/* ------------------------------------------------------------------ */
/* Allocation-free transpose                                            */
/* ------------------------------------------------------------------ */

/* No counterpart in the reference.  The same transpose as eg_csr2csc_i32,
 * for callers that must not allocate device memory when they need it: an
 * application that gives all of a GPU's memory to its own pool at start-up,
 * a serving process that cannot afford cudaMalloc / cudaFree (cudaFree
 * waits for the whole device) on its request path, or a plugin whose host
 * forbids allocation after initialisation.  All pointers are device
 * pointers owned by the caller; stream is a cudaStream_t (NULL: the legacy
 * default stream).  Temporaries live in one static device array sized for
 * EG_NOALLOC_MAX_NNZ entries and EG_NOALLOC_MAX_COLS columns (about 25 MB,
 * held by every GPU that loads the library until the process exits);
 * larger inputs are rejected with EG_ERR_INVALID.  The call allocates
 * nothing, reads the error word back and synchronises the stream before it
 * returns.  The first call on each device looks the static array up
 * (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  Every call shares the array: calls that overlap on the GPU
 * race, so serialise them. */
#define EG_NOALLOC_MAX_NNZ (1LL << 20)
#define EG_NOALLOC_MAX_COLS (1LL << 20)
eg_status eg_csr2csc_device_noalloc(int32_t num_rows, int32_t num_cols, int64_t nnz,
                                    const int64_t *row_ptr, const int32_t *col_idx, const int32_t *val,
                                    int64_t *csc_ptr, int32_t *csc_row, int32_t *csc_val, void *stream);

/* ------------------------------------------------------------------ */
/* Cancellation                                                         */
/* ------------------------------------------------------------------ */

/* Allocates a flag in mapped pinned host memory that a running solve polls
 * once per round; writing a non-zero value makes the solve stop with
 * EG_ERR_CANCELLED. */
eg_status eg_cancel_flag_alloc(volatile int32_t **flag);
void eg_cancel_flag_free(volatile int32_t *flag);

/* ------------------------------------------------------------------ */
/* Game reader (reference text format, optionally gzip-compressed)      */
/* ------------------------------------------------------------------ */

/* An owned game as read from a file: CSR in owner-sorted internal order
 * (player 0 first, as reference src/egsolver.c:107-281 builds it), plus
 * the external name of every internal vertex. */
typedef struct eg_owned_game {
    eg_game game;                /* pointers below, owner == NULL          */
    int64_t *row_ptr;
    int32_t *succ;
    int32_t *weight;
    int32_t *ext_id;             /* ext_id[internal] = id in the file      */
    int32_t max_abs_weight;      /* reference max_pesi                     */
} eg_owned_game;

/* Weight rewrite modes of the reader (reference src/the_parser.y:324-327,
 * --unit-weights / --rnd-weights). */
typedef struct eg_read_opts {
    int32_t weight_mode;         /* 0 keep, 1 unit, 3 random in [lo, hi]   */
    int32_t rnd_lo, rnd_hi;
    uint64_t rnd_seed;
} eg_read_opts;

/* Parses "MAX [EDGES];" then "v MAX|MIN s:w,...,s:w ["name"];" lines
 * (reference src/the_lex.l:33-52, src/the_parser.y:121-160). */
eg_status eg_read_game_file(const char *path, const eg_read_opts *ropts, eg_owned_game **out);
eg_status eg_read_game_buffer(const char *text, size_t len, const eg_read_opts *ropts, eg_owned_game **out);
void eg_owned_game_free(eg_owned_game *g);

/* Binary CSR cache (new; the reference re-parses the text every run): the
 * game as read, with the reader options that shaped it, in one flat file
 * (64-byte header with a checksum, then row_ptr, succ, weight, ext_id).
 * eg_read_game_binary rejects a file written with other options (when
 * ropts != NULL) or whose checksum fails. */
eg_status eg_write_game_binary(const char *path, const eg_owned_game *g, const eg_read_opts *ropts);
eg_status eg_read_game_binary(const char *path, const eg_read_opts *ropts, eg_owned_game **out);
/* eg_read_game_file through a cache: loads cache_path when it is at least as
 * new as path and matches ropts, else parses path and (re)writes the cache. */
eg_status eg_read_game_file_cached(const char *path, const eg_read_opts *ropts, const char *cache_path,
                                   eg_owned_game **out);

/* Streaming form of the same parser: each grammar action calls back, in the
 * order of the reference's parser actions (reference src/the_parser.y:186-301:
 * header, per line node + edges + node_end, footer).  owner is 0 for MAX and
 * 1 for MIN; name points into the text without its quotes (NULL if absent).
 * A callback returns 0 to continue or an eg_status to stop. */
typedef struct eg_parse_cb {
    void *ctx;
    int (*header)(void *ctx, int32_t max_id);
    int (*node)(void *ctx, int32_t id, int32_t owner, int line);
    int (*edge)(void *ctx, int32_t succ, int32_t weight, int line);
    int (*node_end)(void *ctx, const char *name, size_t name_len);
    int (*footer)(void *ctx);
} eg_parse_cb;
eg_status eg_parse_text(const char *text, size_t len, const eg_parse_cb *cb);
/* Reads a whole file, gunzipping it when compressed; *buf is malloc'd. */
eg_status eg_read_file_bytes(const char *path, char **buf, size_t *len);

/* ------------------------------------------------------------------ */
/* Seeded generators for the benchmark workloads                        */
/* ------------------------------------------------------------------ */

/* Generates a random game in owner-sorted order.
 *   kind 1: n vertices, exactly `deg` distinct successors (no self-loops),
 *           weights uniform in [-wmax, wmax]
 *   kind 2: out-degree floor of a continuous power law x^-2 on
 *           [1, deg+1) clipped to [1, deg], distinct, no self-loops
 *   kind 3: complete digraph without self-loops
 *   kind 4: out-degree uniform in {deg_lo..deg} (deg_lo = `param`)
 *   kind 5: out-degree 1 + geometric with mean `param` - 1 (mean `param`)
 * Owners are independent fair coins.  Deterministic in `seed`. */
eg_status eg_generate(int32_t kind, int32_t n, int32_t deg, int32_t wmax, int32_t param,
                      uint64_t seed, eg_owned_game **out);

/* ------------------------------------------------------------------ */
/* The reference's fixture generators (same text, byte for byte)        */
/* ------------------------------------------------------------------ */

/* "Clique" game of vertices 0..number-1 (reference script/multi/mkclique.c):
 * every vertex steps to every other, even ids belong to player 0 (MAX),
 * odd ids to player 1 (MIN).  *text is malloc'd (eg_free_text). */
eg_status eg_fixture_clique_text(int32_t number, char **text, size_t *len);
/* "Ladder" game of 2 * number vertices (reference script/multi/mkladder.c). */
eg_status eg_fixture_ladder_text(int32_t number, char **text, size_t *len);
/* `copies` renamed copies of a game given as text, where every vertex of the
 * first copy also steps to the successors' homologues in every other copy
 * (reference script/multi/multi.c and the actions of its the_parser.y). */
eg_status eg_fixture_copies_text(const char *in, size_t in_len, int32_t copies, char **text, size_t *len);
void eg_free_text(char *text);

#ifdef __cplusplus
}
#endif

#endif /* EGSOLVER_B200_H */
