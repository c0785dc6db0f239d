/*
 * eg_host.c -- host-side C of the solver library: error reporting, option
 * defaults, the reference's preprocessing arithmetic (MG, round cap), game
 * validation, owned games and the seeded workload generators.
 */
#include "eg_internal.h"

#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_last_error[512] = "no error";

eg_status eg_set_error(eg_status st, const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof g_last_error, fmt, ap);
    va_end(ap);
    return st;
}

const char *eg_last_error(void) { return g_last_error; }

int32_t eg_abi_version(void) { return EG_ABI_VERSION; }

void eg_opts_default(eg_opts *opts)
{
    memset(opts, 0, sizeof *opts);
    opts->credit_bits = 64;
    opts->variant = EG_VARIANT_AUTO;
    opts->max_rounds = -1;
    opts->timeout_ms = 0.0;
    opts->cancel = NULL;
    opts->device = 0;
}

/* Owner of vertex v under either owner convention of eg_game. */
static inline int owner_of(const eg_game *g, int64_t v)
{
    return g->owner ? (int)g->owner[v] : (v >= g->num_nodes0 ? 1 : 0);
}

/* Mirrors reference src/egsolver.c:288-304: per vertex the largest negated
 * out-weight clipped at 0, summed; with a 32-bit limit the sum must stay
 * <= INT_MAX exactly as the reference's overflow check demands. */
eg_status eg_compute_mg(const eg_game *game, int32_t limit_bits, int64_t *mg)
{
    int64_t sum = 0;
    for (int64_t v = 0; v < game->num_nodes; v++) {
        int64_t worst = 0;
        for (int64_t j = game->row_ptr[v]; j < game->row_ptr[v + 1]; j++) {
            int64_t d = -(int64_t)game->weight[j];
            if (d > worst) worst = d;
        }
        if (limit_bits == 32 && sum > (int64_t)INT_MAX - worst)
            return eg_set_error(EG_ERR_OVERFLOW, "MG overflows 32-bit credits: %lld + %lld > INT_MAX",
                                (long long)sum, (long long)worst);
        if (sum > INT64_MAX / 4 - worst)
            return eg_set_error(EG_ERR_OVERFLOW, "MG overflows 64-bit credits");
        sum += worst;
    }
    *mg = sum;
    return EG_OK;
}

/* Mirrors reference src/egsolver.c:64-90 (aggiorna_max_loop). */
int64_t eg_default_max_loop(int64_t num_edges, int64_t num_nodes, int64_t mg, int64_t max_loop)
{
    if (max_loop >= 0) return max_loop;
    if (num_nodes <= 0 || num_edges <= 0) return 1;
    if (num_nodes > (LLONG_MAX - 1) / num_edges) return LLONG_MAX - 1;
    if (mg > (LLONG_MAX - 1) / (num_nodes * num_edges)) return LLONG_MAX - 1;
    return num_nodes * num_edges * mg + 1;
}

eg_status eg_validate(const eg_game *g)
{
    if (!g) return eg_set_error(EG_ERR_INVALID, "game is NULL");
    if (g->num_nodes <= 0) return eg_set_error(EG_ERR_INVALID, "game has no vertices");
    if (g->num_edges < 0 || g->num_edges > (int64_t)INT32_MAX - 64)
        return eg_set_error(EG_ERR_INVALID, "num_edges %lld out of range [0, 2^31-64]", (long long)g->num_edges);
    if (g->num_nodes > INT32_MAX - 4096)
        return eg_set_error(EG_ERR_INVALID, "num_nodes %d too large", g->num_nodes);
    if (!g->row_ptr || (g->num_edges > 0 && (!g->succ || !g->weight)))
        return eg_set_error(EG_ERR_INVALID, "NULL CSR array");
    if (!g->owner && (g->num_nodes0 < 0 || g->num_nodes0 > g->num_nodes))
        return eg_set_error(EG_ERR_INVALID, "num_nodes0 %d outside [0, %d]", g->num_nodes0, g->num_nodes);
    if (g->row_ptr[0] != 0 || g->row_ptr[g->num_nodes] != g->num_edges)
        return eg_set_error(EG_ERR_INVALID, "row_ptr must start at 0 and end at num_edges");
    for (int64_t v = 0; v < g->num_nodes; v++) {
        if (g->row_ptr[v + 1] <= g->row_ptr[v])
            return eg_set_error(EG_ERR_INVALID, "vertex %lld has no successor", (long long)v);
        if (g->owner && g->owner[v] > 1)
            return eg_set_error(EG_ERR_INVALID, "vertex %lld has owner %d (expected 0 or 1)",
                                (long long)v, (int)g->owner[v]);
    }
    for (int64_t j = 0; j < g->num_edges; j++) {
        if (g->succ[j] < 0 || g->succ[j] >= g->num_nodes)
            return eg_set_error(EG_ERR_INVALID, "edge %lld has successor %d outside [0, %d)",
                                (long long)j, g->succ[j], g->num_nodes);
    }
    (void)owner_of;
    return EG_OK;
}

/* ------------------------------------------------------------------ */
/* Owned games                                                          */
/* ------------------------------------------------------------------ */

eg_owned_game *eg_owned_game_alloc(int32_t n, int64_t m)
{
    eg_owned_game *g = (eg_owned_game *)calloc(1, sizeof *g);
    if (!g) return NULL;
    g->row_ptr = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));
    g->succ = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    g->weight = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    g->ext_id = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + 1));
    if (!g->row_ptr || !g->succ || !g->weight || !g->ext_id) {
        eg_owned_game_free(g);
        return NULL;
    }
    g->game.num_nodes = n;
    g->game.num_edges = m;
    g->game.row_ptr = g->row_ptr;
    g->game.succ = g->succ;
    g->game.weight = g->weight;
    g->game.owner = NULL;
    return g;
}

void eg_owned_game_free(eg_owned_game *g)
{
    if (!g) return;
    free(g->row_ptr);
    free(g->succ);
    free(g->weight);
    free(g->ext_id);
    free(g);
}

/* Builds the owner-sorted internal CSR from a CSR in file order: player-0
 * vertices first, each class in increasing file order, successors renamed,
 * edges of a vertex kept in their order.  This is the layout the reference
 * builds in postparsing (reference src/egsolver.c:253-281); the reference
 * orders each class with an unstable qsort (src/sorting_criteria.h:91-99),
 * which changes only the internal numbering, never a vertex's credit. */
eg_status eg_owner_sort(int32_t n, int64_t m, const int64_t *ptr, const int32_t *succ,
                        const int32_t *w, const uint8_t *owner, const int32_t *ext_of_file,
                        eg_owned_game **out)
{
    eg_owned_game *g = eg_owned_game_alloc(n, m);
    int32_t *newid = (int32_t *)malloc(sizeof(int32_t) * ((size_t)n + 1));
    if (!g || !newid) {
        free(newid);
        eg_owned_game_free(g);
        return eg_set_error(EG_ERR_OOM, "host allocation failed (%d vertices, %lld edges)", n, (long long)m);
    }
    int32_t n0 = 0;
    for (int32_t v = 0; v < n; v++)
        if (owner[v] == 0) n0++;
    int32_t c0 = 0, c1 = n0;
    for (int32_t v = 0; v < n; v++) newid[v] = owner[v] == 0 ? c0++ : c1++;
    int32_t *oldid = g->ext_id; /* temporarily: oldid[new] = file index */
    for (int32_t v = 0; v < n; v++) oldid[newid[v]] = v;
    int64_t e = 0;
    for (int32_t nv = 0; nv < n; nv++) {
        int32_t v = oldid[nv];
        g->row_ptr[nv] = e;
        for (int64_t j = ptr[v]; j < ptr[v + 1]; j++) {
            g->succ[e] = newid[succ[j]];
            g->weight[e] = w[j];
            e++;
        }
    }
    g->row_ptr[n] = e;
    for (int32_t nv = 0; nv < n; nv++) g->ext_id[nv] = ext_of_file ? ext_of_file[oldid[nv]] : oldid[nv];
    g->game.num_nodes0 = n0;
    int32_t mx = 0;
    for (int64_t j = 0; j < m; j++) {
        int32_t a = w[j] < 0 ? -w[j] : w[j];
        if (a > mx) mx = a;
    }
    g->max_abs_weight = mx;
    free(newid);
    *out = g;
    return EG_OK;
}

/* ------------------------------------------------------------------ */
/* Seeded generators                                                    */
/* ------------------------------------------------------------------ */

typedef struct { uint64_t s; } eg_rng;

/* splitmix64 (Steele, Lea, Flood 2014). */
static inline uint64_t rng_next(eg_rng *r)
{
    uint64_t z = (r->s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
/* Uniform in [0, bound) by the multiply-shift map of the top 32 bits. */
static inline uint32_t rng_below(eg_rng *r, uint32_t bound)
{
    return (uint32_t)(((rng_next(r) >> 32) * (uint64_t)bound) >> 32);
}
static inline double rng_unit(eg_rng *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static inline int32_t rng_range(eg_rng *r, int32_t lo, int32_t hi)
{
    return lo + (int32_t)rng_below(r, (uint32_t)(hi - lo + 1));
}

eg_status eg_generate(int32_t kind, int32_t n, int32_t deg, int32_t wmax, int32_t param,
                      uint64_t seed, eg_owned_game **out)
{
    if (n < 2) return eg_set_error(EG_ERR_INVALID, "generator needs n >= 2");
    if (wmax < 0) return eg_set_error(EG_ERR_INVALID, "wmax must be >= 0");
    if (kind != 3 && (deg < 1 || deg > n - 1))
        return eg_set_error(EG_ERR_INVALID, "degree bound %d outside [1, n-1]", deg);
    if (kind == 4 && (param < 1 || param > deg))
        return eg_set_error(EG_ERR_INVALID, "kind 4 needs 1 <= deg_lo <= deg");
    if (kind == 5 && param < 1)
        return eg_set_error(EG_ERR_INVALID, "kind 5 needs mean >= 1");
    if (kind < 1 || kind > 5) return eg_set_error(EG_ERR_INVALID, "unknown generator kind %d", kind);

    eg_rng r = {seed};
    uint8_t *owner = (uint8_t *)malloc((size_t)n);
    int64_t *ptr = (int64_t *)malloc(sizeof(int64_t) * ((size_t)n + 1));
    int32_t *mark = (int32_t *)calloc((size_t)n, sizeof(int32_t));
    if (!owner || !ptr || !mark) {
        free(owner); free(ptr); free(mark);
        return eg_set_error(EG_ERR_OOM, "generator allocation failed");
    }
    for (int32_t v = 0; v < n; v++) owner[v] = (uint8_t)(rng_next(&r) >> 63);
    /* degrees */
    ptr[0] = 0;
    for (int32_t v = 0; v < n; v++) {
        int64_t d;
        switch (kind) {
        case 1: d = deg; break;
        case 2: {
            double u = rng_unit(&r);
            double x = 1.0 / (1.0 - u * (1.0 - 1.0 / ((double)deg + 1.0)));
            d = (int64_t)floor(x);
            if (d < 1) d = 1;
            if (d > deg) d = deg;
            break;
        }
        case 3: d = n - 1; break;
        case 4: d = rng_range(&r, param, deg); break;
        default: { /* 1 + geometric with success probability 1/param */
            double p = 1.0 / (double)param;
            d = 1;
            if (p < 1.0) {
                double u = rng_unit(&r);
                d = 1 + (int64_t)floor(log1p(-u) / log1p(-p));
            }
            if (d > deg) d = deg;
            break;
        }
        }
        ptr[v + 1] = ptr[v] + d;
    }
    int64_t m = ptr[n];
    if (m > (int64_t)INT32_MAX - 64) {
        free(owner); free(ptr); free(mark);
        return eg_set_error(EG_ERR_INVALID, "generated game has too many edges");
    }
    int32_t *succ = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    int32_t *w = (int32_t *)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    if (!succ || !w) {
        free(owner); free(ptr); free(mark); free(succ); free(w);
        return eg_set_error(EG_ERR_OOM, "generator allocation failed (%lld edges)", (long long)m);
    }
    for (int32_t v = 0; v < n; v++) {
        int64_t b = ptr[v], d = ptr[v + 1] - ptr[v];
        if (kind == 3) {
            int64_t k = 0;
            for (int32_t x = 0; x < n; x++)
                if (x != v) succ[b + k++] = x;
        } else {
            /* distinct successors without self-loops; mark[x] == v+1 means taken */
            int64_t k = 0;
            mark[v] = v + 1;
            while (k < d) {
                int32_t x = (int32_t)rng_below(&r, (uint32_t)n);
                if (mark[x] == v + 1) continue;
                mark[x] = v + 1;
                succ[b + k++] = x;
            }
        }
        for (int64_t k = 0; k < d; k++) w[b + k] = rng_range(&r, -wmax, wmax);
    }
    eg_status st = eg_owner_sort(n, m, ptr, succ, w, owner, NULL, out);
    free(owner); free(ptr); free(mark); free(succ); free(w);
    return st;
}
