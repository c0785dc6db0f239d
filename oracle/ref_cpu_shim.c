/*
 * ref_cpu_shim.c -- test infrastructure only.  Compiled together with the
 * reference's unmodified src/cpu_solver.c, src/host_csr2csc.c and
 * src/errori.c (from the reference tree, into oracle/_ref/libegref.so) so
 * that tests can run the reference's own CPU solvers on a CSR in memory.
 *
 * It defines the process globals that cpu_solver.c reads through extern
 * declarations (the reference defines them in src/egsolver.h:24-119), lays
 * the host buffers out as reference src/dev_solver.cu:178-213 does, computes
 * MG_pesi as reference src/egsolver.c:288-304 does, and calls cpu_solver().
 */
#include "common.h"
#include "errori.h"
#include "host_csr2csc.h"

#include <omp.h>

char str[256];
int counter_nodi, counter_nodi0, counter_nodi0_1, counter_nodi0_2;
int num_nodi, num_archi, max_pesi, MG_pesi;
char *nodeFlags;
int *host_csrPtrInSuccLists, *host_csrSuccLists, *host_csrPesiArchi;
int *host_cscPtrInPredLists, *host_cscPredLists, *host_cscPesiArchiPred;
int numLowInDegree[4];
int numAllInDegree[LEN_DEGREEHIST];
int numAllOutDegree[LEN_DEGREEHIST];
int *host_ResNodeValues1, *host_ResNodeValues2, *host_ResNodeValuesAux;
int *host_csrDataArchiAux;
uint timeout_expired;
config configuration;
stat statistics;

void cpu_solver(void);

/* The reference's loop cap (src/egsolver.c:64-90), restated because the rest
 * of egsolver.c (its main) cannot be linked into a library. */
long aggiorna_max_loop(long Narchi, long Nnodi, long MGpesi, long maxloop)
{
    long res = maxloop;
    if (res < 0) {
        if (MGpesi > (LONG_MAX - 1) / (Nnodi * Narchi)) res = LONG_MAX - 1;
        else res = Nnodi * Narchi * MGpesi + 1;
    }
    return res;
}

/* algo: ALGOR_EG (6) or ALGOR_EG0 (7).  Returns 0, or -1 when MG overflows
 * int (the reference exits there), -2 on allocation failure. */
int ref_cpu_solve(int algo, int n, int n0, int m, const int *ptr, const int *succ, const int *w, long max_loop,
                  int threads, int *out, long *processed, int *mg_out, double *seconds)
{
    memset(&configuration, 0, sizeof configuration);
    memset(&statistics, 0, sizeof statistics);
    memset(numLowInDegree, 0, sizeof numLowInDegree);
    memset(numAllInDegree, 0, sizeof numAllInDegree);
    memset(numAllOutDegree, 0, sizeof numAllOutDegree);
    configuration.algoritmo = algo;
    configuration.max_loop_val = max_loop;
    configuration.print_degree_hist = NO_PRINT_DEGREEHIST;
    configuration.stdinputsource = 1;
    timeout_expired = 0;
    counter_nodi = num_nodi = n;
    counter_nodi0 = n0;
    num_archi = m;
    /* host layout of alloca_memoria_host (src/dev_solver.cu:178-213) */
    long total = (long)n + 1 + m + m + n + n + 1 + 1 + m;
    int *all = (int *)calloc((size_t)total, sizeof(int));
    int *trans = (int *)malloc(sizeof(int) * ((size_t)n + 1 + 2 * (size_t)m));
    nodeFlags = (char *)calloc((size_t)n + 1, 1);
    if (!all || !trans || !nodeFlags) {
        free(all); free(trans); free(nodeFlags);
        return -2;
    }
    host_csrPtrInSuccLists = all;
    host_csrSuccLists = all + n + 1;
    host_csrPesiArchi = host_csrSuccLists + m;
    host_ResNodeValues1 = host_csrPesiArchi + m;
    host_ResNodeValues2 = (algo == ALGOR_EG0) ? host_ResNodeValues1 + n : host_ResNodeValues1;
    host_csrDataArchiAux = host_ResNodeValues2 + n + 1;
    host_ResNodeValuesAux = NULL;
    host_cscPtrInPredLists = trans;
    host_cscPredLists = trans + n + 1;
    host_cscPesiArchiPred = host_cscPredLists + m;
    int *res_base = host_ResNodeValues1;
    memcpy(host_csrPtrInSuccLists, ptr, sizeof(int) * ((size_t)n + 1));
    memcpy(host_csrSuccLists, succ, sizeof(int) * (size_t)m);
    memcpy(host_csrPesiArchi, w, sizeof(int) * (size_t)m);
    max_pesi = 0;
    for (int j = 0; j < m; j++) max_pesi = MAX(max_pesi, abs(w[j]));
    /* MG_pesi as in postparsing */
    MG_pesi = 0;
    for (int v = 0; v < n; v++) {
        int maxdelnodo = 0;
        for (int j = ptr[v]; j < ptr[v + 1]; j++) maxdelnodo = MAX(maxdelnodo, -(w[j]));
        if (MG_pesi > (INT_MAX - maxdelnodo)) {
            free(all); free(trans); free(nodeFlags);
            return -1;
        }
        MG_pesi += maxdelnodo;
    }
    if (threads > 0) omp_set_num_threads(threads);
    cpu_solver();
    memcpy(out, host_ResNodeValues1, sizeof(int) * (size_t)n);
    if (processed) *processed = statistics.processedNodes;
    if (mg_out) *mg_out = MG_pesi;
    if (seconds) *seconds = statistics.solvingtime;
    (void)res_base;
    free(all);
    free(trans);
    free(nodeFlags);
    return 0;
}
