/*
 * eg_refabi.h -- layouts of the reference driver's configuration and
 * statistics structs, which the reference-ABI shim reads and writes through
 * the driver's globals.  The field order and types must stay identical to
 * reference src/common.h:314-321 (struct _stat) and :325-371 (struct
 * _config); the names here are this library's own.
 */
#ifndef EG_REFABI_H
#define EG_REFABI_H

#include <stddef.h>

/* reference src/common.h:147-148, :161-162, :195 */
#define EG_REF_GPU_COMPUTATION 1
#define EG_REF_ALGOR_EG 6
#define EG_REF_ALGOR_EG0 7
#define EG_REF_KIND_VERTEXPAR 1

typedef struct eg_ref_stat {
    double inputtime;
    double alloctime;
    double solvingtime;
    long processedNodes;
    unsigned int numkernelscalls;
    unsigned long device_usedGlobalMem;
} eg_ref_stat;

typedef struct eg_ref_config {
    int computationType;
    int algoritmo;
    int stdinputsource;
    char filename[256];
    int onelineout;
    int add_weights_mode;
    int rndWeightLow;
    int rndWeightHigh;
    int rndSeed;
    int deviceid;
    char devicename[256];
    unsigned short warpSize;
    int capabilityMajor;
    int capabilityMinor;
    size_t deviceProp_totalGlobalMem;
    size_t sharedMemPerBlock;
    unsigned int maxThreadsPerBlock;
    int clockRate;
    int ECCEnabled;
    unsigned int threadsPerBlock;
    unsigned int deviceCount;
    int kinfOfParallelism;
    int shuffleThreshold;
    int shuffleSplit_val;
    int shuffleSplit_low;
    int shuffleSplit_up;
    int shuffleSplit_index;
    int shuffleSplit_soglia;
    int shuffleSplit_double;
    long max_loop_val;
    unsigned int nodesorting;
    unsigned int timeoutOpt;
    unsigned int timeoutSeconds;
    int print_degree_hist;
} eg_ref_config;

#endif
