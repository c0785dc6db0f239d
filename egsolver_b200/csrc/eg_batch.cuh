/*
 * eg_batch.cuh -- the packed game layout, the work units and the launch
 * interface of the batched solver (many games x K thresholds per launch),
 * shared by the batch API (eg_batch.cu) and the serving loop (eg_serve.cu).
 *
 * Packed layout of one game.  Vertices are renumbered by (owner, out-degree):
 * player-0 vertices first, each owner class padded with dummy vertices to a
 * multiple of 32, so that slice s = new ids [32 s, 32 s + 32) belongs to one
 * owner.  Each slice stores its out-edges column-major (an ELL block of
 * width = the slice's largest out-degree): slot (j, lane) holds edge j of
 * vertex 32 s + lane, so a warp reads one column as one 128-byte line.
 * Missing edges are pads that cannot change the vertex's min (player 0:
 * an edge to the sentinel row TOPROW, credit TOP, weight -wpad) or max
 * (player 1: an edge to the sentinel row LOWROW, credit far below 0, weight
 * +wpad), where wpad = max |w| + 1.  A slot is 4 bytes {u16 successor,
 * i16 weight} when the ids and weights fit, else 8 bytes {i32, i32}.
 *
 * The weight of threshold p at scale d is w * d - p (a mean-payoff query
 * "mean payoff >= p/d" as an energy game).  The slots keep w; the kernel
 * forms w * d and adds p once per vertex (OMINUS's clamp is monotone, so
 * min/max over the edges commute with it).
 */
#ifndef EG_BATCH_CUH
#define EG_BATCH_CUH

#include "eg_prep.cuh"

#include <vector>

namespace eg {

/* Largest game the batched paths take (larger games go to the grid solver). */
constexpr int kBatchMaxGameNodes = 1 << 19;

/* Host image of one packed game. */
struct HostPacked {
    int n = 0, n0 = 0, n1 = 0;   /* vertices, of player 0, of player 1         */
    int ns = 0, s0 = 0;          /* slices; first slice of player 1            */
    long long m = 0;             /* real edges                                 */
    long long slots = 0;         /* slots incl. pads (32 per column)           */
    int wide = 0;                /* 8-byte slots                               */
    int wpad = 1;                /* max |w| + 1                                */
    int maxdeg = 0;
    std::vector<uint32_t> e32;   /* narrow slots                               */
    std::vector<int2> e64;       /* wide slots                                 */
    std::vector<int> slice_off;  /* ns + 1 slot offsets                        */
    std::vector<int> orig;       /* 32 ns: new id -> original id, -1 dummy     */
    std::vector<int> minw;       /* per original vertex: min out-weight        */
    int rows() const { return 32 * ns + 2; }
};

/* Builds the packed layout of g (owners from g.owner or the n0 split). */
eg_status pack_game(const eg_game &g, HostPacked *out);

/* Device image of one packed game (E, slice_off and orig in one block). */
struct PackedDev {
    void *E = nullptr;
    int *slice_off = nullptr;
    int *orig = nullptr;
    void *block = nullptr;       /* the one allocation holding all three       */
    size_t bytes = 0;
};
size_t packed_dev_bytes(const HostPacked &h);
/* Uploads into `block` (caller-allocated, packed_dev_bytes(h) bytes). */
eg_status packed_upload(const HostPacked &h, void *block, cudaStream_t st, PackedDev *out);

/* MG of threshold p at scale d: sum_v max(0, p - d * minw(v)). */
long long threshold_mg(const HostPacked &h, int p, int d);

/* Unit variant bits. */
enum : int {
    kUnitKgMask = 3,       /* log2 of the thresholds in the unit (1, 2, 4, 8) */
    kUnitCredit64 = 4,     /* 64-bit credits                                    */
    kUnitWide = 8,         /* 8-byte slots                                      */
    kUnitGlobal = 16,      /* credits in global scratch (too large for a cluster) */
    kUnitTail = 32         /* solved by a cluster only (too large for one CTA)  */
};

/* One work unit: a game at a group of kg = 2^(variant & 3) consecutive
 * thresholds k0 .. k0 + kg - 1, solved by one CTA. */
struct UnitDesc {
    const void *E;
    const int *slice_off;
    const int *orig;
    const int *p;              /* thresholds of the game (index k)            */
    const long long *mg;       /* MG per threshold (index k)                  */
    long long *F;              /* credits out: F[k * n + v], TOP = INT64_MAX  */
    void *gscratch;            /* kUnitGlobal: rows >= srows live here        */
    long long *rounds;         /* out: sweeps run                             */
    int *status;               /* out: eg_status                              */
    long long m;
    int n, n0, n1, ns, s0;
    int d, k0, variant;
    int pad;                   /* tail units: thresholds the host lists        */
    int srows;                 /* kUnitGlobal: rows held in shared memory       */
    int pad2;
};

struct UnitCtrl {
    int next;
    int pad;
    unsigned long long lifts, edges, num_top;
    unsigned long long t_begin, t_end; /* device clock (ns): first CTA start, last CTA end */
};

/* The tail: (unit, threshold) pairs solved by thread-block clusters with the
 * credits spread over the cluster's shared memory.  One list per tail class
 * (credit width x slot width).  Entries come from units too large for one
 * CTA (listed by the host, solved from 0) and from units that phase 1 parks
 * when the GPU runs out of other work (resumed from their credits). */
/* tail classes: (64-bit credits ? 1 : 0) | (8-byte slots ? 2 : 0) | (hybrid ? 4 : 0);
 * a hybrid unit keeps rows >= srows in global memory (each cluster CTA its
 * own copy there) */
constexpr int kTailClasses = 8;
constexpr int kTailSweeps = 4;   /* default sweeps between two cluster barriers */
constexpr int kTailCluster = 16; /* CTAs per cluster (8 where 16 cannot be scheduled) */
struct TailEntry {
    int unit;                  /* index into the unit array                   */
    int k;                     /* threshold                                   */
    long long sweeps;          /* sweeps already run (parked units)           */
    int resume;                /* 1: start from the credits in F              */
    int pad;
};
struct TailList {
    int count, next, cap, init;  /* entries, taken, capacity, listed by the host */
    int cap2, pad;               /* capacity rounded up to a power of two        */
    TailEntry *e;                /* cap2 entries                                 */
    const TailEntry *ie;         /* the init host-listed entries, kept intact    */
};
__host__ __device__ inline int tail_class(int variant)
{
    return ((variant & kUnitCredit64) ? 1 : 0) | ((variant & kUnitWide) ? 2 : 0) | ((variant & kUnitGlobal) ? 4 : 0);
}

struct UnitParams {
    const UnitDesc *units;     /* this variant's units                        */
    UnitCtrl *ctrl;
    TailList *tails;           /* kTailClasses lists (parking), or NULL       */
    int *idle;                 /* CTAs of phase 1 that found their queue empty */
    int num_units;
    int unit_base;             /* index of units[0] in the whole unit array    */
    int park_total;            /* CTAs of all phase-1 kernels of the launch    */
    int park_percent;          /* park when this share of them is idle         */
    unsigned long long *t_start;   /* device clock of the launch's first CTA      */
    long long max_rounds;          /* per unit; < 0: none                        */
    unsigned long long timeout_ns; /* per launch, from t_start; 0: none          */
};

struct TailParams {
    const UnitDesc *units;     /* the whole unit array                        */
    TailList *list;            /* this class's list                           */
    UnitCtrl *ctrl;
    unsigned long long *t_start;
    char *gscratch;            /* hybrid classes: one region per cluster CTA   */
    long long gstride;         /* bytes per region                             */
    long long max_rounds;
    unsigned long long timeout_ns;
    int smem_bytes;            /* dynamic shared memory of the launch          */
    int sweeps;                /* sweeps between two cluster barriers          */
};

/* Choice of credit width and group size for a game. */
struct UnitPlan {
    int credit64;   /* 1: 64-bit credits needed                               */
    int kg_max;     /* largest group that fits one CTA's shared memory (0: none) */
    int tail;       /* with kg_max 0: a cluster holds it (else global scratch)  */
};
/* True when 32-bit credits are exact for every threshold of the list:
 * MG + wpad * d + |p| < 2^30 (the sentinel TOP is 2^30). */
bool credits32_ok(const HostPacked &h, const int *p, int K, int d, const long long *mg);
UnitPlan plan_game(const HostPacked &h, bool credit64, int smem_budget, int kg_cap, int tail_rows = 0);
/* Splits K thresholds into groups of 8/4/2/1 of at most kg_max (kg_max 0:
 * groups of one, credits in global scratch); appends (k0, log2 kg). */
void split_thresholds(int K, int kg_max, std::vector<std::pair<int, int>> *groups);

/* Appends the units of one game at K thresholds: p / mg are the host
 * values, p_dev / mg_dev / F_dev the device arrays the units read and
 * write (F_dev[k * n + v]).  Per unit it also appends the global scratch
 * bytes it needs (0: shared memory) and a cost estimate; *smem grows to
 * the shared memory the units need.  Fails with EG_ERR_OVERFLOW when a
 * threshold's MG does not fit 61 bits. */
eg_status make_units(const HostPacked &h, const PackedDev &pd, int K, int d, const int *p, const long long *mg,
                     const int *p_dev, const long long *mg_dev, long long *F_dev, int smem_budget, int kg_cap,
                     std::vector<UnitDesc> *units, std::vector<size_t> *gneed, std::vector<long long> *cost,
                     int *smem, int tail_rows = 0);
/* Rows a cluster CTA holds for a unit of `rows` rows: a full replica,
 * rounded up to a multiple of 32. */
int tail_rows_per_cta(int rows);

/* Unit variants are indexes 0 .. kNumVariants - 1 (the bits above). */
constexpr int kNumVariants = 32;
/* Counters per launch: one per unit variant and one per tail class. */
constexpr int kNumCtrl = kNumVariants + kTailClasses;

/* Units grouped by variant, heaviest first within a variant:
 * units[off[v] .. off[v + 1]) have variant v. */
struct UnitSet {
    std::vector<UnitDesc> units;      /* phase-1 units by variant, then tail units */
    std::vector<size_t> gneed;        /* global scratch bytes per unit          */
    int off[kNumVariants + 1];
    int smem[kNumVariants];           /* dynamic shared memory per variant      */
    long long top_cost[kNumVariants]; /* heaviest unit of the variant           */
    std::vector<TailEntry> tail_init[kTailClasses]; /* entries of the tail units */
    int tail_cap[kTailClasses];       /* most entries a solve can list          */
    int tail_smem[kTailClasses];      /* shared memory per cluster CTA          */
    long long tail_gbytes[kTailClasses]; /* hybrid: global bytes per cluster CTA */
};
/* Global scratch the hybrid tail classes of S need on a GPU of num_sms SMs. */
size_t tail_scratch_bytes(const UnitSet &S, int num_sms);
/* Device image of a unit set's tail lists: kTailClasses TailList headers
 * followed by their entries (initial entries in place). */
size_t tail_bytes(const UnitSet &S);
eg_status tail_upload(const UnitSet &S, void *block, cudaStream_t st, TailList **lists);
/* Groups units (with their costs and scratch needs); perm[i] = index in
 * `units` of the i-th grouped unit. */
void group_units(const std::vector<UnitDesc> &units, const std::vector<long long> &cost,
                 const std::vector<size_t> &gneed, UnitSet *out, std::vector<int> *perm);

/* Shared memory the kernels can be launched with (the opt-in maximum). */
int unit_smem_budget(int device);
/* Opts every unit kernel in to that much dynamic shared memory (per device). */
eg_status unit_kernel_setup(int device);

/* Side streams on which the variants of a unit set run concurrently: the
 * launch forks from a main stream and joins back into it, so it can be
 * captured into a CUDA graph. */
struct UnitLauncher {
    cudaStream_t aux[kNumCtrl] = {};
    cudaEvent_t join[kNumCtrl] = {};
    cudaEvent_t fork = nullptr, fork2 = nullptr;
    eg_status init();
    void destroy();
};
/* Counters of one launch: a UnitCtrl per variant and per tail class, and
 * the idle count of phase 1. */
struct LaunchCtrl {
    UnitCtrl c[kNumCtrl];
    unsigned long long t_start; /* device clock of the launch's first CTA */
    int idle;
    int pad[3];
};
/* Launches one persistent kernel per variant present in S (the variant
 * holding the heaviest unit first), each taking its units from its own
 * queue, then one cluster kernel per tail class for the tail lists.  ctrl
 * is reset and the tail lists rewound on `main` first. */
eg_status launch_unit_set(UnitLauncher &L, cudaStream_t main, const UnitSet &S, const UnitDesc *units_dev,
                          TailList *tails, void *tail_scratch, LaunchCtrl *ctrl, int block, int num_sms,
                          long long max_rounds, unsigned long long timeout_ns, int *grid_total,
                          int park_percent = 10, int tail_sweeps = kTailSweeps,
                          int tail_cluster = kTailCluster);
/* Totals of the per-variant and per-tail-class counters. */
void sum_ctrl(const LaunchCtrl &c, UnitCtrl *out);

}  // namespace eg

#endif
