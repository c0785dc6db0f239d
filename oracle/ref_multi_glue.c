/*
 * ref_multi_glue.c -- test infrastructure only.  flex and bison are not
 * installed, so the reference's fixture tool script/multi/multi.c (compiled
 * unmodified into oracle/_ref/multi) gets its yyparse() from here: the whole
 * input is read through multi.c's my_abstractread and parsed by the
 * library's eg_parse_text, whose callbacks invoke multi's own grammar
 * actions (the C epilogue of script/multi/the_parser.y, extracted at build
 * time) in the order bison would.  The grammar's one mid-rule action, the
 * "," printed between two edges of a line (script/multi/the_parser.y:91),
 * is issued here before every edge after the first.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "egsolver_b200.h"

int linenum = 1;

extern int my_abstractread(char *buff, int buffsize);
void mpg_arena_header_proc(int max);
void mpg_arena_footer_proc(void);
void mpg_arena_body_line_proc1(int identifier, int owner);
void mpg_arena_body_line_proc2(void);
void mpg_arena_thename_proc(char *name);
void mpg_arena_edge_proc(int succ, int w);

static int edges_on_line;

static int on_header(void *ctx, int32_t max_id)
{
    (void)ctx;
    mpg_arena_header_proc(max_id);
    return 0;
}
static int on_node(void *ctx, int32_t id, int32_t owner, int line)
{
    (void)ctx;
    linenum = line;
    edges_on_line = 0;
    mpg_arena_body_line_proc1(id, owner);
    return 0;
}
static int on_edge(void *ctx, int32_t succ, int32_t w, int line)
{
    (void)ctx;
    linenum = line;
    if (edges_on_line++) fprintf(stdout, ",");
    mpg_arena_edge_proc(succ, w);
    return 0;
}
static int on_node_end(void *ctx, const char *name, size_t len)
{
    (void)ctx;
    if (!name) {
        mpg_arena_thename_proc(NULL);
    } else {
        /* the lexer's string token keeps its quotes */
        char *q = (char *)malloc(len + 3);
        q[0] = '"';
        memcpy(q + 1, name, len);
        q[len + 1] = '"';
        q[len + 2] = '\0';
        mpg_arena_thename_proc(q);
        free(q);
    }
    mpg_arena_body_line_proc2();
    return 0;
}
static int on_footer(void *ctx)
{
    (void)ctx;
    mpg_arena_footer_proc();
    return 0;
}

int yyparse(void)
{
    size_t cap = 1 << 20, len = 0;
    char *buf = (char *)malloc(cap);
    for (;;) {
        if (cap - len < (1 << 16)) {
            cap *= 2;
            buf = (char *)realloc(buf, cap);
        }
        int r = my_abstractread(buf + len, (int)(cap - len));
        if (r <= 0) break;
        len += (size_t)r;
    }
    eg_parse_cb cb = {NULL, on_header, on_node, on_edge, on_node_end, on_footer};
    eg_status st = eg_parse_text(buf, len, &cb);
    free(buf);
    if (st != EG_OK) {
        fprintf(stderr, "Error reading input:  %s line %d\n", eg_last_error(), linenum);
        exit(-1);
    }
    return 0;
}
