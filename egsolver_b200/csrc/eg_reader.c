/*
 * eg_reader.c -- reader for the reference's text game format, gzip or plain.
 *
 *   MAXNODE [NUMEDGES] ;              (optionally preceded by "arena")
 *   v MAX|MIN s:w, ..., s:w ["name"] ;
 *
 * Tokens follow reference src/the_lex.l:33-52 (blanks skipped, "#", "%" and
 * "//" comments to end of line, any other unknown character ignored,
 * integers range-checked like a2int at :8-24); the grammar follows reference
 * src/the_parser.y:121-160 and the checks of its actions (:234-256 repeated
 * or out-of-range vertex ids, :315-336 out-of-range successors, :283-301
 * vertex count).  flex and bison are not needed: the parser is a hand-written
 * recursive descent over the same grammar, driving the callbacks of
 * eg_parse_cb so that other consumers (for instance the reference's own
 * parser actions) can reuse it.
 */
#include "eg_internal.h"

#include <ctype.h>
#include <errno.h>
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <zlib.h>

enum { T_EOF = 0, T_INT, T_FLOAT, T_STRING, T_ARENA, T_MAX, T_MIN, T_SEMI, T_COL, T_COMMA, T_MINUS, T_ERR };

typedef struct lexer {
    const char *p, *end;
    int line;
    int tok;
    int32_t ival;
    const char *sval;
    size_t slen;
    char err[256];
} lexer;

static int lex_next(lexer *L)
{
    for (;;) {
        if (L->p >= L->end) return L->tok = T_EOF;
        char c = *L->p;
        if (c == ' ' || c == '\t') { L->p++; continue; }
        if (c == '\n') { L->line++; L->p++; continue; }
        if (c == '#' || c == '%' || (c == '/' && L->p + 1 < L->end && L->p[1] == '/')) {
            while (L->p < L->end && *L->p != '\n') L->p++;
            continue;
        }
        if (c == ';') { L->p++; return L->tok = T_SEMI; }
        if (c == ':') { L->p++; return L->tok = T_COL; }
        if (c == ',') { L->p++; return L->tok = T_COMMA; }
        if (c == '-') { L->p++; return L->tok = T_MINUS; }
        if (c >= '0' && c <= '9') {
            const char *s = L->p;
            while (L->p < L->end && *L->p >= '0' && *L->p <= '9') L->p++;
            if (L->p + 1 < L->end && *L->p == '.' && L->p[1] >= '0' && L->p[1] <= '9') {
                L->p++;
                while (L->p < L->end && *L->p >= '0' && *L->p <= '9') L->p++;
                return L->tok = T_FLOAT;
            }
            /* a2int: decimal, must fit int */
            long long v = 0;
            for (const char *q = s; q < L->p; q++) {
                v = v * 10 + (*q - '0');
                if (v > INT_MAX) {
                    snprintf(L->err, sizeof L->err, "out-of-range integer in input (line %d)", L->line);
                    return L->tok = T_ERR;
                }
            }
            L->ival = (int32_t)v;
            return L->tok = T_INT;
        }
        if (c == '"') {
            const char *s = L->p++;
            while (L->p < L->end && *L->p != '"') {
                if (*L->p == '\\' && L->p + 1 < L->end) L->p++;
                if (*L->p == '\n') L->line++;
                L->p++;
            }
            if (L->p >= L->end) {
                snprintf(L->err, sizeof L->err, "unterminated string (line %d)", L->line);
                return L->tok = T_ERR;
            }
            L->p++;
            L->sval = s;
            L->slen = (size_t)(L->p - s);
            return L->tok = T_STRING;
        }
        if (L->end - L->p >= 5 && memcmp(L->p, "arena", 5) == 0) { L->p += 5; return L->tok = T_ARENA; }
        if (L->end - L->p >= 3 && memcmp(L->p, "MAX", 3) == 0) { L->p += 3; return L->tok = T_MAX; }
        if (L->end - L->p >= 3 && memcmp(L->p, "MIN", 3) == 0) { L->p += 3; return L->tok = T_MIN; }
        L->p++; /* any other character is ignored by the reference lexer */
    }
}

static eg_status syntax(lexer *L, const char *what)
{
    if (L->tok == T_ERR) return eg_set_error(EG_ERR_IO, "error reading input: %s", L->err);
    return eg_set_error(EG_ERR_IO, "error reading input: syntax error (%s) line %d", what, L->line);
}

eg_status eg_parse_text(const char *text, size_t len, const eg_parse_cb *cb)
{
    lexer L;
    memset(&L, 0, sizeof L);
    L.p = text;
    L.end = text + len;
    L.line = 1;
    int rc;
    /* header */
    lex_next(&L);
    if (L.tok == T_ARENA) lex_next(&L);
    if (L.tok != T_INT) return syntax(&L, "header: expected the maximum vertex id");
    int32_t maxid = L.ival;
    lex_next(&L);
    if (L.tok == T_INT) lex_next(&L); /* NUMEDGES is read and ignored */
    if (L.tok != T_SEMI) return syntax(&L, "header: expected ';'");
    if ((rc = cb->header(cb->ctx, maxid)) != 0) return (eg_status)rc;
    lex_next(&L);
    int lines = 0;
    while (L.tok == T_INT) {
        int32_t id = L.ival;
        lex_next(&L);
        int owner;
        if (L.tok == T_MAX) owner = 0;
        else if (L.tok == T_MIN) owner = 1;
        else return syntax(&L, "expected MAX or MIN after the vertex id");
        if ((rc = cb->node(cb->ctx, id, owner, L.line)) != 0) return (eg_status)rc;
        /* edges: edge (',' edge)* */
        for (;;) {
            lex_next(&L);
            if (L.tok != T_INT) return syntax(&L, "expected a successor id");
            int32_t s = L.ival;
            lex_next(&L);
            if (L.tok != T_COL) return syntax(&L, "expected ':' after the successor id");
            lex_next(&L);
            int neg = 0;
            if (L.tok == T_MINUS) { neg = 1; lex_next(&L); }
            if (L.tok != T_INT) return syntax(&L, "expected an edge weight");
            int32_t w = neg ? -L.ival : L.ival;
            if ((rc = cb->edge(cb->ctx, s, w, L.line)) != 0) return (eg_status)rc;
            lex_next(&L);
            if (L.tok != T_COMMA) break;
        }
        const char *name = NULL;
        size_t nlen = 0;
        if (L.tok == T_STRING) {
            name = L.sval + 1;
            nlen = L.slen - 2;
            lex_next(&L);
        }
        if (L.tok != T_SEMI) return syntax(&L, "expected ';' at the end of a vertex line");
        if ((rc = cb->node_end(cb->ctx, name, nlen)) != 0) return (eg_status)rc;
        lines++;
        lex_next(&L);
    }
    if (lines == 0) return syntax(&L, "expected at least one vertex line");
    if (L.tok != T_EOF) return syntax(&L, "unexpected token after the last vertex line");
    return cb->footer ? (eg_status)cb->footer(cb->ctx) : EG_OK;
}

/* ------------------------------------------------------------------ */
/* Default consumer: a CSR in file order, then the owner sort.          */
/* ------------------------------------------------------------------ */

typedef struct csr_builder {
    int32_t maxid, nnodes;        /* header max id; number of lines read */
    int32_t *ext_of_file;         /* [nnodes] */
    int32_t *file_of_ext;         /* [maxid+1], -1 = unseen */
    uint8_t *owner;
    int64_t *ptr;
    int32_t *succ, *w;
    int64_t m, cap;
    const eg_read_opts *ro;
} csr_builder;

static int cb_header(void *ctx, int32_t maxid)
{
    csr_builder *b = (csr_builder *)ctx;
    if (maxid < 0 || maxid >= INT32_MAX - 4096)
        return eg_set_error(EG_ERR_IO, "error in input: maximum vertex id %d out of range", maxid);
    size_t n = (size_t)maxid + 1;
    b->maxid = maxid;
    b->ext_of_file = (int32_t *)malloc(n * sizeof(int32_t));
    b->file_of_ext = (int32_t *)malloc(n * sizeof(int32_t));
    b->owner = (uint8_t *)malloc(n);
    b->ptr = (int64_t *)malloc((n + 1) * sizeof(int64_t));
    b->cap = 2 * (int64_t)(n + 1);
    b->succ = (int32_t *)malloc((size_t)b->cap * sizeof(int32_t));
    b->w = (int32_t *)malloc((size_t)b->cap * sizeof(int32_t));
    if (!b->ext_of_file || !b->file_of_ext || !b->owner || !b->ptr || !b->succ || !b->w)
        return eg_set_error(EG_ERR_OOM, "reader allocation failed for %d vertices", maxid + 1);
    for (size_t i = 0; i < n; i++) b->file_of_ext[i] = -1;
    return 0;
}

static int cb_node(void *ctx, int32_t id, int32_t owner, int line)
{
    csr_builder *b = (csr_builder *)ctx;
    if (id > b->maxid)
        return eg_set_error(EG_ERR_IO, "error in input. Unexpected node identifier: %d greater than %d (input line %d)",
                            id, b->maxid, line);
    if (b->file_of_ext[id] != -1)
        return eg_set_error(EG_ERR_IO, "error in input. Repeated node identifier: %d (input line %d)", id, line);
    if (b->nnodes > b->maxid)
        return eg_set_error(EG_ERR_IO, "error in input: more vertex lines than declared (line %d)", line);
    b->file_of_ext[id] = b->nnodes;
    b->ext_of_file[b->nnodes] = id;
    b->owner[b->nnodes] = (uint8_t)owner;
    b->ptr[b->nnodes] = b->m;
    return 0;
}

static int cb_edge(void *ctx, int32_t s, int32_t w, int line)
{
    csr_builder *b = (csr_builder *)ctx;
    if (s > b->maxid)
        return eg_set_error(EG_ERR_IO, "error in input. Unexpected successor identifier: %d greater than %d (input line %d)",
                            s, b->maxid, line);
    if (b->m >= b->cap) {
        if (b->cap > (int64_t)INT32_MAX)
            return eg_set_error(EG_ERR_IO, "error in input: too many edges");
        b->cap *= 2;
        int32_t *ns = (int32_t *)realloc(b->succ, (size_t)b->cap * sizeof(int32_t));
        if (ns) b->succ = ns;
        int32_t *nw = (int32_t *)realloc(b->w, (size_t)b->cap * sizeof(int32_t));
        if (nw) b->w = nw;
        if (!ns || !nw) return eg_set_error(EG_ERR_OOM, "reader allocation failed (%lld edges)", (long long)b->cap);
    }
    const eg_read_opts *ro = b->ro;
    int32_t weight = w;
    if (ro && ro->weight_mode == 1) weight = 1;
    else if (ro && ro->weight_mode == 3) weight = ro->rnd_lo + (rand() % (1 + ro->rnd_hi - ro->rnd_lo));
    b->succ[b->m] = s;
    b->w[b->m] = weight;
    b->m++;
    return 0;
}

static int cb_node_end(void *ctx, const char *name, size_t len)
{
    (void)name; (void)len;
    csr_builder *b = (csr_builder *)ctx;
    b->nnodes++;
    return 0;
}

static int cb_footer(void *ctx)
{
    csr_builder *b = (csr_builder *)ctx;
    if (b->nnodes != b->maxid + 1)
        return eg_set_error(EG_ERR_IO, "error in input. Expecting %d nodes, read %d nodes", b->maxid + 1, b->nnodes);
    b->ptr[b->nnodes] = b->m;
    return 0;
}

static void builder_free(csr_builder *b)
{
    free(b->ext_of_file); free(b->file_of_ext); free(b->owner); free(b->ptr); free(b->succ); free(b->w);
}

eg_status eg_read_game_buffer(const char *text, size_t len, const eg_read_opts *ropts, eg_owned_game **out)
{
    if (!text || !out) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    csr_builder b;
    memset(&b, 0, sizeof b);
    b.ro = ropts;
    if (ropts && ropts->weight_mode == 3) {
        if (ropts->rnd_hi < ropts->rnd_lo) return eg_set_error(EG_ERR_INVALID, "random weight range is empty");
        srand((unsigned)ropts->rnd_seed);
    }
    eg_parse_cb cb = {&b, cb_header, cb_node, cb_edge, cb_node_end, cb_footer};
    eg_status st = eg_parse_text(text, len, &cb);
    if (st != EG_OK) { builder_free(&b); return st; }
    int32_t n = b.nnodes;
    /* successor ids: external -> file order (reference nomeInt_of_nomeExt) */
    for (int64_t j = 0; j < b.m; j++) {
        int32_t f = b.file_of_ext[b.succ[j]];
        if (f < 0) { builder_free(&b); return eg_set_error(EG_ERR_IO, "error in input: successor %d is not a vertex", b.succ[j]); }
        b.succ[j] = f;
    }
    for (int32_t v = 0; v < n; v++)
        if (b.ptr[v + 1] == b.ptr[v]) {
            int32_t id = b.ext_of_file[v];
            builder_free(&b);
            return eg_set_error(EG_ERR_IO, "error in input: vertex %d has no successor", id);
        }
    st = eg_owner_sort(n, b.m, b.ptr, b.succ, b.w, b.owner, b.ext_of_file, out);
    builder_free(&b);
    return st;
}

eg_status eg_read_file_bytes(const char *path, char **buf, size_t *len)
{
    gzFile f = gzopen(path, "rb");
    if (!f) return eg_set_error(EG_ERR_IO, "cannot open %s: %s", path, strerror(errno));
    size_t cap = 1 << 20, n = 0;
    char *b = (char *)malloc(cap);
    if (!b) { gzclose(f); return eg_set_error(EG_ERR_OOM, "reader allocation failed"); }
    for (;;) {
        if (cap - n < (1 << 16)) {
            cap *= 2;
            char *nb = (char *)realloc(b, cap);
            if (!nb) { free(b); gzclose(f); return eg_set_error(EG_ERR_OOM, "reader allocation failed"); }
            b = nb;
        }
        int r = gzread(f, b + n, (unsigned)(cap - n));
        if (r < 0) { free(b); gzclose(f); return eg_set_error(EG_ERR_IO, "error reading %s (gzread)", path); }
        if (r == 0) break;
        n += (size_t)r;
    }
    gzclose(f);
    *buf = b;
    *len = n;
    return EG_OK;
}

eg_status eg_read_game_file(const char *path, const eg_read_opts *ropts, eg_owned_game **out)
{
    char *buf;
    size_t len;
    eg_status st = eg_read_file_bytes(path, &buf, &len);
    if (st != EG_OK) return st;
    st = eg_read_game_buffer(buf, len, ropts, out);
    free(buf);
    return st;
}

/* ------------------------------------------------------------------ */
/* Binary CSR cache                                                     */
/* ------------------------------------------------------------------ */

/* A game as read (owner-sorted CSR, external names, reader options) in a
 * flat little-endian file, so that a large game parsed once from text is
 * loaded again at memory speed:
 *
 *   header (64 bytes): magic "EGCSR\1\0\0", n, n0 (int32), m (int64),
 *       max |w| (int32), weight mode, rnd lo, rnd hi (int32), rnd seed
 *       (uint64), FNV-1a 64 checksum of the arrays (uint64), 8 bytes zero
 *   row_ptr int64[n + 1] | succ int32[m] | weight int32[m] | ext_id int32[n]
 */
typedef struct {
    char magic[8];
    int32_t n, n0;
    int64_t m;
    int32_t max_abs_weight, weight_mode, rnd_lo, rnd_hi;
    uint64_t rnd_seed, checksum, zero;
} egb_header;

static const char EGB_MAGIC[8] = {'E', 'G', 'C', 'S', 'R', 1, 0, 0};

static uint64_t fnv1a(uint64_t h, const void *p, size_t len)
{
    const unsigned char *c = (const unsigned char *)p;
    for (size_t i = 0; i < len; i++) {
        h ^= c[i];
        h *= 0x100000001b3ULL;
    }
    return h;
}

static uint64_t egb_checksum(const eg_owned_game *g)
{
    const int32_t n = g->game.num_nodes;
    const int64_t m = g->game.num_edges;
    uint64_t h = 0xcbf29ce484222325ULL;
    h = fnv1a(h, g->row_ptr, sizeof(int64_t) * ((size_t)n + 1));
    h = fnv1a(h, g->succ, sizeof(int32_t) * (size_t)m);
    h = fnv1a(h, g->weight, sizeof(int32_t) * (size_t)m);
    return fnv1a(h, g->ext_id, sizeof(int32_t) * (size_t)n);
}

static void egb_opts(const eg_read_opts *ro, egb_header *h)
{
    h->weight_mode = ro ? ro->weight_mode : 0;
    h->rnd_lo = ro && ro->weight_mode == 3 ? ro->rnd_lo : 0;
    h->rnd_hi = ro && ro->weight_mode == 3 ? ro->rnd_hi : 0;
    h->rnd_seed = ro && ro->weight_mode == 3 ? ro->rnd_seed : 0;
}

eg_status eg_write_game_binary(const char *path, const eg_owned_game *g, const eg_read_opts *ropts)
{
    if (!path || !g) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    egb_header h;
    memset(&h, 0, sizeof h);
    memcpy(h.magic, EGB_MAGIC, 8);
    h.n = g->game.num_nodes;
    h.n0 = g->game.num_nodes0;
    h.m = g->game.num_edges;
    h.max_abs_weight = g->max_abs_weight;
    egb_opts(ropts, &h);
    h.checksum = egb_checksum(g);
    FILE *f = fopen(path, "wb");
    if (!f) return eg_set_error(EG_ERR_IO, "cannot create %s: %s", path, strerror(errno));
    int ok = fwrite(&h, sizeof h, 1, f) == 1;
    ok = ok && fwrite(g->row_ptr, sizeof(int64_t), (size_t)h.n + 1, f) == (size_t)h.n + 1;
    ok = ok && fwrite(g->succ, sizeof(int32_t), (size_t)h.m, f) == (size_t)h.m;
    ok = ok && fwrite(g->weight, sizeof(int32_t), (size_t)h.m, f) == (size_t)h.m;
    ok = ok && fwrite(g->ext_id, sizeof(int32_t), (size_t)h.n, f) == (size_t)h.n;
    ok = (fclose(f) == 0) && ok;
    if (!ok) return eg_set_error(EG_ERR_IO, "error writing %s", path);
    return EG_OK;
}

eg_status eg_read_game_binary(const char *path, const eg_read_opts *ropts, eg_owned_game **out)
{
    if (!path || !out) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    FILE *f = fopen(path, "rb");
    if (!f) return eg_set_error(EG_ERR_IO, "cannot open %s: %s", path, strerror(errno));
    egb_header h;
    if (fread(&h, sizeof h, 1, f) != 1 || memcmp(h.magic, EGB_MAGIC, 8) != 0 || h.n <= 0 || h.m < 0 ||
        h.n0 < 0 || h.n0 > h.n || h.m > (int64_t)INT32_MAX) {
        fclose(f);
        return eg_set_error(EG_ERR_IO, "%s is not a binary game file", path);
    }
    egb_header want;
    memset(&want, 0, sizeof want);
    egb_opts(ropts, &want);
    if (ropts && (want.weight_mode != h.weight_mode || want.rnd_lo != h.rnd_lo || want.rnd_hi != h.rnd_hi ||
                  want.rnd_seed != h.rnd_seed)) {
        fclose(f);
        return eg_set_error(EG_ERR_IO, "%s was written with other reader options", path);
    }
    eg_owned_game *g = eg_owned_game_alloc(h.n, h.m);
    if (!g) {
        fclose(f);
        return eg_set_error(EG_ERR_OOM, "host allocation failed");
    }
    int ok = fread(g->row_ptr, sizeof(int64_t), (size_t)h.n + 1, f) == (size_t)h.n + 1;
    ok = ok && fread(g->succ, sizeof(int32_t), (size_t)h.m, f) == (size_t)h.m;
    ok = ok && fread(g->weight, sizeof(int32_t), (size_t)h.m, f) == (size_t)h.m;
    ok = ok && fread(g->ext_id, sizeof(int32_t), (size_t)h.n, f) == (size_t)h.n;
    fclose(f);
    g->game.num_nodes0 = h.n0;
    g->max_abs_weight = h.max_abs_weight;
    if (!ok || egb_checksum(g) != h.checksum) {
        eg_owned_game_free(g);
        return eg_set_error(EG_ERR_IO, "%s is truncated or corrupt (checksum)", path);
    }
    eg_status st = eg_validate(&g->game);
    if (st != EG_OK) {
        eg_owned_game_free(g);
        return st;
    }
    *out = g;
    return EG_OK;
}

eg_status eg_read_game_file_cached(const char *path, const eg_read_opts *ropts, const char *cache_path,
                                   eg_owned_game **out)
{
    if (!path || !cache_path || !out) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    struct stat sp, sc;
    if (stat(path, &sp) == 0 && stat(cache_path, &sc) == 0 && sc.st_mtime >= sp.st_mtime) {
        eg_owned_game *g = NULL;
        if (eg_read_game_binary(cache_path, ropts, &g) == EG_OK) {
            *out = g;
            return EG_OK;
        }
    }
    eg_status st = eg_read_game_file(path, ropts, out);
    if (st != EG_OK) return st;
    /* best effort: a cache that cannot be written leaves the result alone */
    size_t len = strlen(cache_path);
    char *tmp = (char *)malloc(len + 8);
    if (tmp) {
        memcpy(tmp, cache_path, len);
        memcpy(tmp + len, ".tmp", 5);
        if (eg_write_game_binary(tmp, *out, ropts) == EG_OK) {
            if (rename(tmp, cache_path) != 0) remove(tmp);
        } else {
            remove(tmp);
        }
        free(tmp);
    }
    return EG_OK;
}
