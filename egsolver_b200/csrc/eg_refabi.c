/*
 * eg_refabi.c -- the reference's GPU module boundary, re-implemented on top
 * of this library so that the reference driver (src/egsolver.c) links and
 * runs unchanged against the B200 solver.
 *
 * Exported symbols, with the reference declarations they replace:
 *   int  alloca_memoria_host(void)      reference src/dev_solver.h:9,  src/dev_solver.cu:152-191
 *   int  alloca_memoria_device(void)    reference src/dev_solver.h:10, src/dev_solver.cu:193-239
 *   int  copia_dati_su_device(void)     reference src/dev_solver.h:15, src/dev_solver.cu:142-150
 *   void gpu_solver(void)               reference src/dev_solver.h:20, src/dev_solver.cu:81-139
 *   int  dealloca_memoria_host(void)    reference src/dev_solver.h:12, src/dev_solver.cu:241-260
 *   int  dealloca_memoria_device(void)  reference src/dev_solver.h:13, src/dev_solver.cu:262-266
 *   void checkDevice(int*, config*)     reference src/utils.h:20,      src/utils.cu:51-75
 *   void checkCUDAError(const char*)    reference src/utils.cu:38-47
 *
 * Data flows through the driver's process globals exactly as in the
 * reference (declared extern below with the reference's names and types):
 * the owner-sorted CSR in host_csr*, counter_nodi0, the configuration and
 * statistics structs, and the result in host_ResNodeValues1.  The host
 * buffer layout is the reference's (one pinned block; src/dev_solver.cu:
 * 152-178).  On the device the game becomes one resident eg_dgame.
 *
 * Like the reference module this file ends the process on errors: the
 * driver that calls it expects that.  The library's own API (eg_*) never
 * exits.
 */
#include <cuda_runtime.h>
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "egsolver_b200.h"
#include "eg_refabi.h"

/* driver globals (reference src/egsolver.h:24-119) */
extern int num_nodi, num_archi, counter_nodi0, MG_pesi, max_pesi;
extern int *host_allData, *host_csrPtrInSuccLists, *host_csrSuccLists, *host_revSuccLists, *host_csrPesiArchi;
extern int *host_ResNodeValues1, *host_ResNodeValues2, *host_ResNodeValuesAux, *host_flag, *host_csrDataArchiAux;
extern int *host_transData, *host_cscPtrInPredLists, *host_cscPredLists, *host_cscPesiArchiPred;
extern int *csrPtrInSuccLists, *nodePriority, *csrPesiArchi, *csrSuccLists, *nomeExt_of_nomeInt, *nomeInt_of_nomeExt;
extern int *mapping, *revmapping;
extern char *nodeOwner, *nodeFlags;
extern char **nodeName;
extern unsigned int timeout_expired;
extern eg_ref_config configuration;
extern eg_ref_stat statistics;

static int g_host_pinned;          /* host_allData came from cudaMallocHost */
static eg_dgame *g_dgame;          /* the resident game of this process     */

static void die(const char *what, const char *detail)
{
    fprintf(stderr, "ERROR: %s: %s\n", what, detail);
    fflush(stderr);
    exit(EXIT_FAILURE);
}

int alloca_memoria_host(void)
{
    /* one block: ptr n+1 | succ m | weights m | credits n | (credits n) | flag 1 | aux m */
    long total = (long)num_nodi + 1 + num_archi + num_archi + num_nodi + num_nodi + 1 + 1 + num_archi;
    void *p = NULL;
    g_host_pinned = 0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) == cudaSuccess && ndev > 0 &&
        cudaMallocHost(&p, (size_t)total * sizeof(int)) == cudaSuccess) {
        g_host_pinned = 1;
    } else {
        cudaGetLastError();
        p = malloc((size_t)total * sizeof(int));
    }
    if (!p) die("alloca_memoria_host", "host allocation failed");
    host_allData = (int *)p;
    host_csrPtrInSuccLists = host_allData;
    host_csrSuccLists = host_allData + num_nodi + 1;
    host_csrPesiArchi = host_csrSuccLists + num_archi;
    host_ResNodeValues1 = host_csrPesiArchi + num_archi;
    host_ResNodeValues2 = (configuration.algoritmo == EG_REF_ALGOR_EG0) ? host_ResNodeValues1 + num_nodi : host_ResNodeValues1;
    host_flag = host_ResNodeValues2 + num_nodi;
    host_csrDataArchiAux = host_flag + 1;
    memset(host_ResNodeValues1, 0, (size_t)num_nodi * sizeof(int));
    host_ResNodeValuesAux = NULL;
    if (configuration.algoritmo != EG_REF_ALGOR_EG && configuration.algoritmo != EG_REF_ALGOR_EG0) host_revSuccLists = NULL;
    if (configuration.algoritmo == EG_REF_ALGOR_EG || configuration.algoritmo == EG_REF_ALGOR_EG0) {
        size_t trans = (size_t)num_nodi + 1 + 2 * (size_t)num_archi;
        host_transData = (int *)malloc(trans * sizeof(int));
        if (!host_transData) die("alloca_memoria_host", "host allocation failed (transData)");
        host_cscPtrInPredLists = host_transData;
        host_cscPredLists = host_transData + num_nodi + 1;
        host_cscPesiArchiPred = host_cscPredLists + num_archi;
    }
    return 0;
}

/* The device arrays are created when the data are copied (they are sized by
 * the CSR that the driver fills in between). */
int alloca_memoria_device(void) { return 0; }

int copia_dati_su_device(void)
{
    if (configuration.computationType != EG_REF_GPU_COMPUTATION) return 0;
    int64_t *ptr64 = (int64_t *)malloc(sizeof(int64_t) * ((size_t)num_nodi + 1));
    if (!ptr64) die("copia_dati_su_device", "host allocation failed");
    for (int v = 0; v <= num_nodi; v++) ptr64[v] = host_csrPtrInSuccLists[v];
    eg_game g;
    g.num_nodes = num_nodi;
    g.num_nodes0 = counter_nodi0;
    g.num_edges = num_archi;
    g.row_ptr = ptr64;
    g.succ = host_csrSuccLists;
    g.weight = host_csrPesiArchi;
    g.owner = NULL;
    eg_opts o;
    eg_opts_default(&o);
    o.device = configuration.deviceid;
    if (g_dgame) eg_dgame_free(g_dgame);
    g_dgame = NULL;
    eg_status s = eg_dgame_upload(&g, &o, &g_dgame);
    free(ptr64);
    if (s != EG_OK) die("copia_dati_su_device", eg_last_error());
    return 0;
}

void gpu_solver(void)
{
    if (!g_dgame) die("gpu_solver", "no game on the device (copia_dati_su_device not called)");
    eg_opts o;
    eg_opts_default(&o);
    o.device = configuration.deviceid;
    o.credit_bits = 32; /* the reference's int credits, TOP = INT_MAX */
    switch (configuration.kinfOfParallelism) {
    case EG_REF_KIND_VERTEXPAR: o.variant = EG_VARIANT_THREAD; break;
    case 2: case 4: case 8: case 16: case 32:
        o.variant = EG_VARIANT_WARP;
        o.lanes_per_vertex = configuration.kinfOfParallelism;
        break;
    default: o.variant = EG_VARIANT_AUTO; break;
    }
    o.max_rounds = configuration.max_loop_val > 0 ? configuration.max_loop_val : -1;
    if (configuration.timeoutOpt == 1 && configuration.timeoutSeconds > 0)
        o.timeout_ms = 1000.0 * configuration.timeoutSeconds;
    eg_stats st;
    printf("Running EG on GPU (B200 persistent solver, variant %d). (MG_pesi=%d num nodes=%d max weight=%d)\n",
           o.variant, MG_pesi, num_nodi, max_pesi);
    fflush(stdout);
    eg_status s = eg_dgame_solve(g_dgame, &o, &st);
    if (s == EG_ERR_TIMEOUT) timeout_expired = 1;
    if (s != EG_OK && s != EG_ERR_LOOPCAP && s != EG_ERR_TIMEOUT) die("gpu_solver", eg_last_error());
    if (eg_dgame_credits_i32(g_dgame, host_ResNodeValues1) != EG_OK) die("gpu_solver", eg_last_error());
    printf("End EG on GPU after %lld loops (each loop involves one or more active nodes). Processed nodes %lld\n",
           (long long)st.rounds, (long long)st.lifts);
    statistics.solvingtime = st.solve_ms; /* milliseconds, as the reference's GPU path reports */
    statistics.processedNodes = (long)st.lifts;
    statistics.numkernelscalls = (unsigned int)st.kernel_launches;
}

int dealloca_memoria_host(void)
{
    if (g_host_pinned) cudaFreeHost(host_allData);
    else free(host_allData);
    host_allData = NULL;
    free(host_transData);
    free(csrPtrInSuccLists);
    free(nodePriority);
    free(nodeOwner);
    free(nodeFlags);
    free(csrPesiArchi);
    free(csrSuccLists);
    free(nomeExt_of_nomeInt);
    free(nomeInt_of_nomeExt);
    free(mapping);
    free(revmapping);
    for (int i = 0; i < num_nodi; i++) free(nodeName[i]);
    free(nodeName);
    return 0;
}

int dealloca_memoria_device(void)
{
    if (g_dgame) eg_dgame_free(g_dgame);
    g_dgame = NULL;
    return 0;
}

void checkCUDAError(const char *msg)
{
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        fprintf(stderr, "CUDA error: >%s<: >%s<. Exiting\n", msg, cudaGetErrorString(err));
        exit(-1);
    }
}

void checkDevice(int *deviceCount, eg_ref_config *conf)
{
    cudaError_t e = cudaGetDeviceCount(deviceCount);
    if (e != cudaSuccess) die("cudaGetDeviceCount returned", cudaGetErrorString(e));
    if (*deviceCount <= conf->deviceid) die("checkDevice returned", "Selected device not available");
    struct cudaDeviceProp p;
    cudaGetDeviceProperties(&p, conf->deviceid);
    conf->deviceProp_totalGlobalMem = p.totalGlobalMem;
    conf->maxThreadsPerBlock = (unsigned int)p.maxThreadsPerBlock;
    conf->sharedMemPerBlock = p.sharedMemPerBlock;
    conf->warpSize = (unsigned short)p.warpSize;
    conf->capabilityMajor = p.major;
    conf->capabilityMinor = p.minor;
    int clock = 0, ecc = 0;
    cudaDeviceGetAttribute(&clock, cudaDevAttrClockRate, conf->deviceid);
    cudaDeviceGetAttribute(&ecc, cudaDevAttrEccEnabled, conf->deviceid);
    conf->clockRate = clock;
    conf->ECCEnabled = ecc;
    memcpy(conf->devicename, p.name, sizeof conf->devicename);
}
