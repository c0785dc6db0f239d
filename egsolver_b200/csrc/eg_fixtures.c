/*
 * eg_fixtures.c -- the reference's fixture generators for benchmark games,
 * producing the same text, byte for byte:
 *
 *   eg_fixture_clique_text   reference script/multi/mkclique.c:19-72
 *   eg_fixture_ladder_text   reference script/multi/mkladder.c:19-58
 *   eg_fixture_copies_text   reference script/multi/multi.c with the grammar
 *                            actions of script/multi/the_parser.y:128-180
 *
 * The text is the reference game format (the_lex.l / the_parser.y), so any
 * of these games can be read back with eg_read_game_buffer.  The output is
 * built in one growing host buffer; writing text is host work with nothing
 * for a GPU to do.
 */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "eg_internal.h"

typedef struct {
    char *p;
    size_t len, cap;
    int oom;
} sbuf;

static void sb_printf(sbuf *b, const char *fmt, ...)
{
    if (b->oom) return;
    for (;;) {
        va_list ap;
        va_start(ap, fmt);
        const size_t room = b->cap - b->len;
        const int k = vsnprintf(b->p ? b->p + b->len : NULL, b->p ? room : 0, fmt, ap);
        va_end(ap);
        if (k < 0) {
            b->oom = 1;
            return;
        }
        if (b->p && (size_t)k < room) {
            b->len += (size_t)k;
            return;
        }
        size_t nc = b->cap ? b->cap * 2 : 1 << 16;
        while (nc - b->len <= (size_t)k) nc *= 2;
        char *q = (char *)realloc(b->p, nc);
        if (!q) {
            b->oom = 1;
            return;
        }
        b->p = q;
        b->cap = nc;
    }
}

static eg_status sb_finish(sbuf *b, char **text, size_t *len)
{
    if (b->oom || !b->p) {
        free(b->p);
        return eg_set_error(EG_ERR_OOM, "fixture text allocation failed");
    }
    *text = b->p;
    *len = b->len;
    return EG_OK;
}

void eg_free_text(char *text) { free(text); }

eg_status eg_fixture_clique_text(int32_t number, char **text, size_t *len)
{
    if (!text || !len) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    if (number < 1) return eg_set_error(EG_ERR_INVALID, "clique size must be a positive int");
    const int maxnode = number - 1;
    sbuf b = {0};
    sb_printf(&b, "%d;\n", maxnode);
    /* vertices of the first player (even ids), then of the second (odd ids);
     * edge i -> j weighs 1 when i < j, else -1, negated for the second player;
     * the last edge of a line ends with ';' */
    for (int pass = 0; pass < 2; pass++) {
        for (int i = 0; i <= maxnode; i++) {
            if ((i % 2) != pass) continue;
            sb_printf(&b, "%d %s ", i, pass == 0 ? "MAX" : "MIN");
            for (int j = 0; j <= maxnode; j++) {
                if (i == j) continue;
                const int w = (i < j) ? 1 : -1;
                const int last = (i < maxnode && j == maxnode) || (i == maxnode && j == maxnode - 1);
                sb_printf(&b, "%d:%d%s", j, pass == 0 ? w : -w, last ? ";" : ",");
            }
            sb_printf(&b, "\n");
        }
    }
    return sb_finish(&b, text, len);
}

eg_status eg_fixture_ladder_text(int32_t number, char **text, size_t *len)
{
    if (!text || !len) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    if (number < 1 || number > (int32_t)(0x7fffffff / 2)) return eg_set_error(EG_ERR_INVALID, "ladder size out of range");
    const int span = 2 * number, maxnode = span - 1;
    sbuf b = {0};
    sb_printf(&b, "%d;\n", maxnode);
    /* rungs: even vertex 2k (first player) steps to 2k+1 and 2k+2 at no
     * cost; odd vertex 2k+1 (second player) steps to 2k+2 for free or to
     * 2k+3 at cost 1, all indexes modulo 2 * number */
    for (int i = 0; i <= maxnode; i += 2) sb_printf(&b, "%d MAX %d:%d,%d:%d;\n", i, (i + 1) % span, 0, (i + 2) % span, 0);
    for (int i = 0; i <= maxnode; i += 2)
        sb_printf(&b, "%d MIN %d:%d,%d:%d;\n", i + 1, (i + 2) % span, 0, (i + 3) % span, -1);
    return sb_finish(&b, text, len);
}

/* ---- copies: a streaming rewrite through the game parser's callbacks ---- */

typedef struct {
    sbuf *b;
    int copies, max_id, owner, node;
    int nsucc, cap;
    int32_t *succ, *w;
    int oom;
} copies_ctx;

static int cp_header(void *c, int32_t max_id)
{
    copies_ctx *x = (copies_ctx *)c;
    x->max_id = max_id;
    sb_printf(x->b, "%d;\n", max_id + (x->copies - 1) * (max_id + 1));
    return 0;
}

static int cp_node(void *c, int32_t id, int32_t owner, int line)
{
    (void)line;
    copies_ctx *x = (copies_ctx *)c;
    x->node = id;
    x->owner = owner;
    x->nsucc = 0;
    sb_printf(x->b, "%d %s ", id, owner == 0 ? "MAX" : "MIN");
    return 0;
}

static int cp_edge(void *c, int32_t succ, int32_t w, int line)
{
    (void)line;
    copies_ctx *x = (copies_ctx *)c;
    if (x->nsucc == x->cap) {
        const int nc = x->cap ? 2 * x->cap : 64;
        int32_t *s = (int32_t *)realloc(x->succ, sizeof(int32_t) * (size_t)nc);
        if (s) x->succ = s;
        int32_t *q = (int32_t *)realloc(x->w, sizeof(int32_t) * (size_t)nc);
        if (q) x->w = q;
        if (!s || !q) return EG_ERR_OOM;
        x->cap = nc;
    }
    /* the grammar prints the separator before every edge after the first */
    sb_printf(x->b, "%s%d:%d", x->nsucc ? "," : "", succ, w);
    x->succ[x->nsucc] = succ;
    x->w[x->nsucc++] = w;
    return 0;
}

static int cp_node_end(void *c, const char *name, size_t name_len)
{
    copies_ctx *x = (copies_ctx *)c;
    const long long stride = (long long)x->max_id + 1;
    /* the vertex of the first copy also steps into every other copy */
    for (int j = 1; j < x->copies; j++)
        for (int i = 0; i < x->nsucc; i++) sb_printf(x->b, ",%lld:%d", x->succ[i] + j * stride, x->w[i]);
    if (name) sb_printf(x->b, "; \"%.*s\"\n", (int)name_len, name);
    else sb_printf(x->b, ";\n");
    for (int j = 1; j < x->copies; j++) {
        sb_printf(x->b, "%lld %s ", x->node + j * stride, x->owner == 0 ? "MAX" : "MIN");
        for (int i = 0; i < x->nsucc; i++) sb_printf(x->b, "%s%lld:%d", i ? "," : "", x->succ[i] + j * stride, x->w[i]);
        if (name) sb_printf(x->b, "; \"%.*s\"X\n", (int)name_len, name);
        else sb_printf(x->b, ";\n");
    }
    x->nsucc = 0;
    return 0;
}

static int cp_footer(void *c)
{
    (void)c;
    return 0;
}

eg_status eg_fixture_copies_text(const char *in, size_t in_len, int32_t copies, char **text, size_t *len)
{
    if (!in || !text || !len) return eg_set_error(EG_ERR_INVALID, "NULL argument");
    if (copies < 2) return eg_set_error(EG_ERR_INVALID, "copies must be at least 2");
    sbuf b = {0};
    copies_ctx x;
    memset(&x, 0, sizeof x);
    x.b = &b;
    x.copies = copies;
    eg_parse_cb cb = {&x, cp_header, cp_node, cp_edge, cp_node_end, cp_footer};
    eg_status st = eg_parse_text(in, in_len, &cb);
    free(x.succ);
    free(x.w);
    if (st != EG_OK) {
        free(b.p);
        return st;
    }
    return sb_finish(&b, text, len);
}
