/*
 * eg_oracle.c -- CPU restatement of the reference solver, used ONLY as test
 * infrastructure: by tests/, by __graft_entry__.smoke() as the checker and by
 * bench.py's cpu_baseline / reference arm.  Nothing in the product links it.
 *
 * Restated from fvella/EGSolver:
 *   oracle_ominus        <- src/common.h:270-272 (OMINUS)
 *   oracle_mg            <- src/egsolver.c:288-304 (MG_pesi)
 *   oracle_max_loop      <- src/egsolver.c:64-90 (aggiorna_max_loop)
 *   oracle_csr2csc       <- src/host_csr2csc.c:15-46
 *   oracle_eg_solve_i32  <- src/cpu_solver.c:190-333 (EG_cpu_solver), int32
 *   oracle_eg_solve_i64  <- the same algorithm with 64-bit credits and TOP
 *   oracle_eg0_solve_i32 <- src/cpu_solver.c:50-106 (EG0_scpu_solver, serial Jacobi)
 *   oracle_eg0_omp_i32   <- src/cpu_solver.c:109-185 with its two thread-safety
 *                           defects fixed (private inner index, per-thread flags
 *                           sized by the thread count)
 *   oracle_generate      the benchmark's seeded game generator (not part of the
 *                        reference), so that reference-side timings build their
 *                        inputs without the solver library
 *
 * Parity pins: the int32 worklist solver is checked against the reference's
 * own cpu_solver.c compiled under oracle/_ref (same pop count and credits),
 * and against the reference's golden output script/sol.txt for
 * script/clique_500_cp4.txt.gz.
 *
 * Conventions as in the reference: vertices [0, n0) belong to player 0 (the
 * file's MAX, minimising), [n0, n) to player 1 (maximising); TOP is INT_MAX
 * (int32) or INT64_MAX (int64).  row_ptr is int64 here; the reference's int
 * offsets are the same numbers.
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TOP32 INT32_MAX
#define TOP64 INT64_MAX

/* OMINUS with the reference's compare order: a < TOP and a - b <= MG give
 * max(0, a - b), anything else TOP.  a - b is formed in 64 bits, which equals
 * the reference's int arithmetic whenever that does not overflow. */
static inline int32_t ominus32(int32_t a, int32_t b, int64_t mg)
{
    int64_t d = (int64_t)a - (int64_t)b;
    return (a < TOP32 && d <= mg) ? (int32_t)(d > 0 ? d : 0) : TOP32;
}
static inline int64_t ominus64(int64_t a, int32_t b, int64_t mg)
{
    return (a < TOP64 && a - b <= mg) ? ((a - b) > 0 ? a - b : 0) : TOP64;
}

int64_t oracle_ominus(int64_t a, int64_t b, int64_t mg, int32_t bits)
{
    return bits == 32 ? ominus32((int32_t)a, (int32_t)b, mg) : ominus64(a, (int32_t)b, mg);
}

/* Returns -1 when limit_bits == 32 and the sum passes INT_MAX (the reference
 * exits with "too high weights" there). */
int64_t oracle_mg(int32_t n, const int64_t *ptr, const int32_t *w, int32_t limit_bits)
{
    int64_t mg = 0;
    for (int32_t v = 0; v < n; v++) {
        int64_t worst = 0;
        for (int64_t j = ptr[v]; j < ptr[v + 1]; j++)
            if (-(int64_t)w[j] > worst) worst = -(int64_t)w[j];
        if (limit_bits == 32 && mg > (int64_t)INT_MAX - worst) return -1;
        mg += worst;
    }
    return mg;
}

int64_t oracle_max_loop(int64_t m, int64_t n, int64_t mg, int64_t max_loop)
{
    if (max_loop >= 0) return max_loop;
    if (mg > (LLONG_MAX - 1) / (n * m)) return LLONG_MAX - 1;
    return n * m * mg + 1;
}

/* host_csr2csc: count per column, prefix-sum, scatter rows in order, shift. */
void oracle_csr2csc(int32_t nrow, int32_t ncol, int64_t nnz, const int32_t *val, const int32_t *col,
                    const int64_t *rowptr, int32_t *cscval, int32_t *cscrow, int64_t *cscptr)
{
    for (int32_t i = 0; i <= ncol; i++) cscptr[i] = 0;
    for (int64_t i = 0; i < nnz; i++) cscptr[col[i] + 1]++;
    for (int32_t i = 0; i < ncol; i++) cscptr[i + 1] += cscptr[i];
    for (int32_t i = 0; i < nrow; i++) {
        for (int64_t j = rowptr[i]; j < rowptr[i + 1]; j++) {
            int32_t k = col[j];
            int64_t l = cscptr[k]++;
            cscrow[l] = i;
            cscval[l] = val[j];
        }
    }
    for (int32_t i = ncol; i > 0; i--) cscptr[i] = cscptr[i - 1];
    cscptr[0] = 0;
}

typedef struct oracle_stats {
    int64_t loops;        /* reference "loop-1": pops for EG, sweeps for EG0 */
    int64_t processed;    /* reference statistics.processedNodes            */
    int64_t edges;        /* out-degrees summed over lifted vertices         */
    int64_t finished;     /* 1 when the worklist emptied / the sweep was stable */
} oracle_stats;

/* EG_cpu_solver (reference src/cpu_solver.c:190-333): initial queue of
 * player-0 vertices whose out-edges are all negative and player-1 vertices
 * with a negative out-edge (:218-246), FIFO ring of n slots with a flag per
 * vertex (:283-329), lift on pop (:297-306), on increase push every
 * unflagged predecessor (:310-323).  max_loop < 0 means the reference
 * default.  credits holds n entries and must be zero on entry, as
 * host_ResNodeValues1 is (src/dev_solver.cu:193). */
#define DEFINE_EG_SOLVE(NAME, T, OMINUS_FN)                                                       \
    int NAME(int32_t n, int32_t n0, int64_t m, const int64_t *ptr, const int32_t *succ,             \
             const int32_t *w, int64_t mg, int64_t max_loop, T *f, oracle_stats *st)                \
    {                                                                                               \
        int64_t *cptr = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));                       \
        int32_t *cpred = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));              \
        int32_t *cval = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));               \
        int32_t *queue = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);                            \
        char *flag = (char *)calloc((size_t)n, 1);                                                  \
        if (!cptr || !cpred || !cval || !queue || !flag) {                                          \
            free(cptr); free(cpred); free(cval); free(queue); free(flag);                           \
            return -1;                                                                              \
        }                                                                                           \
        max_loop = oracle_max_loop(m, n, mg, max_loop);                                             \
        int32_t in_q = 0, out_q = 0, len_q = 0;                                                     \
        for (int32_t v = 0; v < n0; v++) {                                                          \
            int all_neg = 1;                                                                        \
            for (int64_t j = ptr[v]; all_neg && j < ptr[v + 1]; j++)                                \
                if (w[j] >= 0) all_neg = 0;                                                         \
            if (all_neg) { flag[v] = 1; queue[in_q++] = v; }                                        \
        }                                                                                           \
        for (int32_t v = n0; v < n; v++) {                                                          \
            int any_neg = 0;                                                                        \
            for (int64_t j = ptr[v]; !any_neg && j < ptr[v + 1]; j++)                               \
                if (w[j] < 0) any_neg = 1;                                                          \
            if (any_neg) { flag[v] = 1; queue[in_q++] = v; }                                        \
        }                                                                                           \
        len_q = in_q;                                                                               \
        in_q = in_q % n;                                                                            \
        oracle_csr2csc(n, n, m, w, succ, ptr, cval, cpred, cptr);                                   \
        int64_t loop = 1, edges = 0;                                                                \
        int changed = 0;                                                                            \
        while (len_q > 0 && loop <= max_loop) {                                                     \
            loop++;                                                                                 \
            changed = 0;                                                                            \
            int32_t v = queue[out_q];                                                               \
            out_q = (out_q + 1) % n;                                                                \
            len_q--;                                                                                \
            flag[v] = 0;                                                                            \
            int64_t b = ptr[v], e = ptr[v + 1];                                                     \
            T t = OMINUS_FN(f[succ[b]], w[b], mg);                                                  \
            for (int64_t j = b + 1; j < e; j++) {                                                   \
                T val = OMINUS_FN(f[succ[j]], w[j], mg);                                            \
                if (v < n0 && t > val) t = val;                                                     \
                if (v >= n0 && t < val) t = val;                                                    \
            }                                                                                       \
            edges += e - b;                                                                         \
            if (f[v] < t) {                                                                         \
                f[v] = t;                                                                           \
                changed = 1;                                                                        \
                for (int64_t z = cptr[v]; z < cptr[v + 1]; z++) {                                   \
                    int32_t p = cpred[z];                                                           \
                    if (!flag[p]) {                                                                 \
                        queue[in_q] = p;                                                            \
                        in_q = (in_q + 1) % n;                                                      \
                        flag[p] = 1;                                                                \
                        len_q++;                                                                    \
                    }                                                                               \
                }                                                                                   \
            }                                                                                       \
            if (!changed && len_q == 0) break;                                                      \
        }                                                                                           \
        if (st) {                                                                                   \
            st->loops = loop - 1;                                                                   \
            st->processed = loop - 1;                                                               \
            st->edges = edges;                                                                      \
            st->finished = len_q == 0;                                                              \
        }                                                                                           \
        free(cptr); free(cpred); free(cval); free(queue); free(flag);                               \
        return 0;                                                                                   \
    }

DEFINE_EG_SOLVE(oracle_eg_solve_i32, int32_t, ominus32)
DEFINE_EG_SOLVE(oracle_eg_solve_i64, int64_t, ominus64)

/* EG0_scpu_solver (reference src/cpu_solver.c:50-106): Jacobi sweeps from
 * data1 into data2 until a sweep changes nothing.  The reference's final
 * array choice tests max_loop % 2 (:99), which after convergence is
 * immaterial because both arrays hold the fixed point; here the most recent
 * sweep's array is returned. */
int oracle_eg0_solve_i32(int32_t n, int32_t n0, int64_t m, const int64_t *ptr, const int32_t *succ,
                         const int32_t *w, int64_t mg, int64_t max_loop, int32_t *f, oracle_stats *st)
{
    int32_t *d1 = f;
    int32_t *d2 = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    if (!d2) return -1;
    memset(d1, 0, sizeof(int32_t) * (size_t)n);
    max_loop = oracle_max_loop(m, n, mg, max_loop);
    int64_t loop, edges = 0;
    int flag1 = 0;
    for (loop = 1; loop <= max_loop; loop++) {
        flag1 = 0;
        for (int32_t v = 0; v < n; v++) {
            int32_t t = ominus32(d1[succ[ptr[v]]], w[ptr[v]], mg);
            for (int64_t j = ptr[v] + 1; j < ptr[v + 1]; j++) {
                int32_t val = ominus32(d1[succ[j]], w[j], mg);
                if (v < n0 && t > val) t = val;
                if (v >= n0 && t < val) t = val;
            }
            edges += ptr[v + 1] - ptr[v];
            if (d2[v] < t) { flag1 = 1; d2[v] = t; }
        }
        int32_t *tmp = d1; d1 = d2; d2 = tmp;
        if (!flag1) break;
    }
    if (d1 != f) { memcpy(f, d1, sizeof(int32_t) * (size_t)n); free(d1); }
    else free(d2);
    if (st) {
        st->loops = loop - 1; /* the reference reports loop-1 (src/cpu_solver.c:104-105) */
        st->processed = st->loops * (int64_t)n;
        st->edges = edges;
        st->finished = !flag1;
    }
    return 0;
}

/* EG0_cpu_solver (reference src/cpu_solver.c:109-185) with OpenMP, its inner
 * index made private and its change flag a reduction, so that it is safe
 * with any number of threads.  Used as the multi-core CPU baseline. */
int oracle_eg0_omp_i32(int32_t n, int32_t n0, int64_t m, const int64_t *ptr, const int32_t *succ,
                       const int32_t *w, int64_t mg, int64_t max_loop, int32_t *f, oracle_stats *st,
                       int32_t threads)
{
    int32_t *d1 = f;
    int32_t *d2 = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    if (!d2) return -1;
    memset(d1, 0, sizeof(int32_t) * (size_t)n);
    max_loop = oracle_max_loop(m, n, mg, max_loop);
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    int64_t loop, edges = 0;
    int any = 0;
    for (loop = 1; loop <= max_loop; loop++) {
        any = 0;
        int32_t *src = d1, *dst = d2;
#pragma omp parallel for schedule(guided, 4) reduction(| : any)
        for (int32_t v = 0; v < n; v++) {
            int32_t t = ominus32(src[succ[ptr[v]]], w[ptr[v]], mg);
            for (int64_t j = ptr[v] + 1; j < ptr[v + 1]; j++) {
                int32_t val = ominus32(src[succ[j]], w[j], mg);
                if (v < n0 && t > val) t = val;
                if (v >= n0 && t < val) t = val;
            }
            if (dst[v] < t) { any = 1; dst[v] = t; }
        }
        edges += m;
        int32_t *tmp = d1; d1 = d2; d2 = tmp;
        if (!any) break;
    }
    if (d1 != f) { memcpy(f, d1, sizeof(int32_t) * (size_t)n); free(d1); }
    else free(d2);
    if (st) {
        st->loops = loop - 1; /* the reference reports loop-1 (src/cpu_solver.c:104-105) */
        st->processed = st->loops * (int64_t)n;
        st->edges = edges;
        st->finished = !any;
    }
    return 0;
}

/* Fixed-point check used on results too large for the worklist oracle:
 * returns the number of vertices whose lift differs from f (0 means f is a
 * fixed point of the lifting operator). */
int64_t oracle_count_inconsistent_i64(int32_t n, int32_t n0, const int64_t *ptr, const int32_t *succ,
                                      const int32_t *w, int64_t mg, const int64_t *f)
{
    int64_t bad = 0;
    for (int32_t v = 0; v < n; v++) {
        int64_t t = ominus64(f[succ[ptr[v]]], w[ptr[v]], mg);
        for (int64_t j = ptr[v] + 1; j < ptr[v + 1]; j++) {
            int64_t val = ominus64(f[succ[j]], w[j], mg);
            if (v < n0 && t > val) t = val;
            if (v >= n0 && t < val) t = val;
        }
        if (t != f[v]) bad++;
    }
    return bad;
}

/* ------------------------------------------------------------------ */
/* Seeded benchmark games, restated for the checker side                */
/* ------------------------------------------------------------------ */

/* The benchmark's seeded game generator, restated here so that the
 * reference arm of the benchmark and the CPU baselines build their inputs
 * without loading the solver library.  Same definition as the library's
 * eg_generate: splitmix64 (Steele, Lea, Flood 2014) drives, in order, one
 * owner bit per vertex (the top bit), the out-degrees (kind 1: deg; kind 2:
 * floor of the inverse-CDF sample 1 / (1 - u (1 - 1/(deg+1))) of a
 * continuous x^-2 law on [1, deg+1), clipped to [1, deg]; kind 3: n - 1;
 * kind 4: uniform in [param, deg]; kind 5: 1 + floor(log1p(-u) /
 * log1p(-1/param)) capped at deg), then per vertex its distinct successors
 * without self-loops (rejection sampling; kind 3 takes all others in order)
 * followed by its weights uniform in [-wmax, wmax].  Uniform integers are
 * the multiply-shift map of the top 32 bits.  The result is renumbered
 * owner-sorted (player 0 first, each class in increasing index, edge order
 * kept), the layout the reference's postparsing builds.
 *
 * Outputs are malloc'd (free with oracle_free); returns 0, -1 on bad
 * arguments, -2 on allocation failure. */
typedef struct { uint64_t s; } orng;
static inline uint64_t orng_next(orng *r)
{
    uint64_t z = (r->s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static inline uint32_t orng_below(orng *r, uint32_t bound)
{
    return (uint32_t)(((orng_next(r) >> 32) * (uint64_t)bound) >> 32);
}
static inline double orng_unit(orng *r) { return (double)(orng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

int oracle_generate(int32_t kind, int32_t n, int32_t deg, int32_t wmax, int32_t param, uint64_t seed,
                    int64_t **ptr_out, int32_t **succ_out, int32_t **w_out, int64_t *m_out, int32_t *n0_out)
{
    if (n < 2 || wmax < 0 || kind < 1 || kind > 5) return -1;
    if (kind != 3 && (deg < 1 || deg > n - 1)) return -1;
    if (kind == 4 && (param < 1 || param > deg)) return -1;
    if (kind == 5 && param < 1) return -1;
    orng r = {seed};
    uint8_t *own = malloc((size_t)n);
    int64_t *deg_of = malloc(sizeof(int64_t) * (size_t)n);
    int32_t *seen = calloc((size_t)n, sizeof(int32_t));
    if (!own || !deg_of || !seen) {
        free(own); free(deg_of); free(seen);
        return -2;
    }
    for (int32_t v = 0; v < n; v++) own[v] = (uint8_t)(orng_next(&r) >> 63);
    int64_t m = 0;
    for (int32_t v = 0; v < n; v++) {
        int64_t d;
        if (kind == 1) {
            d = deg;
        } else if (kind == 2) {
            const double u = orng_unit(&r);
            d = (int64_t)floor(1.0 / (1.0 - u * (1.0 - 1.0 / ((double)deg + 1.0))));
            d = d < 1 ? 1 : (d > deg ? deg : d);
        } else if (kind == 3) {
            d = n - 1;
        } else if (kind == 4) {
            d = param + (int64_t)orng_below(&r, (uint32_t)(deg - param + 1));
        } else {
            const double q = 1.0 / (double)param;
            d = 1;
            if (q < 1.0) d = 1 + (int64_t)floor(log1p(-orng_unit(&r)) / log1p(-q));
            if (d > deg) d = deg;
        }
        deg_of[v] = d;
        m += d;
    }
    int32_t *s0 = malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    int32_t *w0 = malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    int64_t *p0 = malloc(sizeof(int64_t) * ((size_t)n + 1));
    int64_t *ptr = malloc(sizeof(int64_t) * ((size_t)n + 1));
    int32_t *succ = malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    int32_t *w = malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    int32_t *nid = malloc(sizeof(int32_t) * (size_t)n);
    int32_t *oid = malloc(sizeof(int32_t) * (size_t)n);
    if (!s0 || !w0 || !p0 || !ptr || !succ || !w || !nid || !oid) {
        free(own); free(deg_of); free(seen); free(s0); free(w0); free(p0); free(ptr); free(succ); free(w);
        free(nid); free(oid);
        return -2;
    }
    p0[0] = 0;
    for (int32_t v = 0; v < n; v++) p0[v + 1] = p0[v] + deg_of[v];
    for (int32_t v = 0; v < n; v++) {
        const int64_t b = p0[v], d = deg_of[v];
        if (kind == 3) {
            int64_t k = 0;
            for (int32_t x = 0; x < n; x++)
                if (x != v) s0[b + k++] = x;
        } else {
            seen[v] = v + 1;
            for (int64_t k = 0; k < d;) {
                const int32_t x = (int32_t)orng_below(&r, (uint32_t)n);
                if (seen[x] == v + 1) continue;
                seen[x] = v + 1;
                s0[b + k++] = x;
            }
        }
        for (int64_t k = 0; k < d; k++) w0[b + k] = -wmax + (int32_t)orng_below(&r, (uint32_t)(2 * wmax + 1));
    }
    int32_t n0 = 0;
    for (int32_t v = 0; v < n; v++) n0 += own[v] == 0;
    int32_t c0 = 0, c1 = n0;
    for (int32_t v = 0; v < n; v++) nid[v] = own[v] == 0 ? c0++ : c1++;
    for (int32_t v = 0; v < n; v++) oid[nid[v]] = v;
    int64_t e = 0;
    for (int32_t u = 0; u < n; u++) {
        const int32_t v = oid[u];
        ptr[u] = e;
        for (int64_t j = p0[v]; j < p0[v + 1]; j++, e++) {
            succ[e] = nid[s0[j]];
            w[e] = w0[j];
        }
    }
    ptr[n] = e;
    free(own); free(deg_of); free(seen); free(s0); free(w0); free(p0); free(nid); free(oid);
    *ptr_out = ptr;
    *succ_out = succ;
    *w_out = w;
    *m_out = m;
    *n0_out = n0;
    return 0;
}

void oracle_free(void *p) { free(p); }
