/*
 * eg_prep.cuh -- declarations of the preprocessing kernels and the layout
 * tables they produce.
 */
#ifndef EG_PREP_CUH
#define EG_PREP_CUH

#include "eg_device.cuh"

namespace eg {

/* Out-degree buckets: bucket i holds deg <= upper[i] (and > upper[i-1]);
 * the last bucket is unbounded.  nb <= EG_MAX_CLASSES / 2. */
struct BucketBounds {
    int nb;
    int upper[EG_MAX_CLASSES / 2];
};

/* Where each class (bucket * 2 + owner) lives in the renumbered id space.
 * Every class starts on a multiple of 32 so that a frontier word never
 * mixes classes (and so never mixes owners). */
struct ClassTable {
    int nc;
    int start[EG_MAX_CLASSES];
    int count[EG_MAX_CLASSES];
    long long sorted_begin[EG_MAX_CLASSES];
    __device__ __forceinline__ int owner_of_new(int u) const
    {
        for (int c = 0; c < nc; c++)
            if (u >= start[c] && u < start[c] + count[c]) return c & 1;
        return 0;
    }
};

long long scan_scratch_ints(long long len);
void excl_scan(int *data, long long len, int *scratch, cudaStream_t st);
long long radix_scratch_ints(long long count);
void radix_sort_pairs(int *k0, int *v0, int *k1, int *v1, long long count, int bits, int *scratch,
                      cudaStream_t st, int **kres, int **vres);
int bits_for(long long max_key);

__global__ void k_classify(int n, int n0, const long long *row_ptr, const int *w, const unsigned char *owner,
                           BucketBounds bb, int *cls_key, int *cls_val, unsigned char *active0,
                           unsigned long long *mg_acc, int *class_count);
__global__ void k_build_perm(int n, const int *sorted_cls, const int *sorted_v, ClassTable ct, int *perm, int *iperm);
__global__ void k_new_degree(int n_pad, const int *perm, const long long *row_ptr, int *pdeg);
__global__ void k_copy_edges(int n_pad, const int *perm, const int *iperm, const long long *row_ptr, const int *succ,
                             const int *w, const int *P, int2 *E, int *csc_key, int *csc_val, int *indeg,
                             ClassTable ct, int topv, int zerov);
__global__ void k_init_frontier(int n_pad, const int *perm, const unsigned char *active0, uint32_t *B);
__global__ void k_round4(int len, const int *in, int *out);
__global__ void k_csc_pad(int n_pad, const int *dense_off, const int *pad_off, const int *dense, int *padded);
/* heavy tasks: per heavy vertex the number of 256-edge tasks, then the tasks */
__global__ void k_task_count(int heavy_begin, int n_pad, const int *P, int task_pairs, int *count);
__global__ void k_task_fill(int heavy_begin, int n_pad, const int *P, int task_pairs, const int *toff, ClassTable ct,
                            int4 *tasks);
/* per solve: tasks-to-report counters and identity partials */
void launch_task_reset(int bits, int heavy_begin, int n_pad, const int *toff, ClassTable ct, void *hacc, int *hrem,
                       cudaStream_t st);
/* credits: 0 everywhere except TOP at the sentinel topv */
void launch_init_credits(int bits, int n_alloc, void *F, int topv, cudaStream_t st);
/* number of TOP credits among the first n_pad, added to *out */
void launch_count_top(int bits, int n_pad, const void *F, unsigned long long *out, cudaStream_t st);
/* out[v] = F[iperm[v]] converted between widths, TOP kept as TOP */
void launch_gather_out(int in_bits, int out_bits, int n, const int *iperm, const void *F, void *out, cudaStream_t st);

__global__ void k_csr_expand(int nrows, const long long *row_ptr, const int *col, int *key, int *val, int *colcount);
__global__ void k_edge_rows(int nrows, const long long *row_ptr, int *row_of_edge);
__global__ void k_csc_gather(long long nnz, const int *sorted_edge, const int *row_of_edge, const int *val,
                             int *csc_row, int *csc_val);
__global__ void k_widen(long long len, const int *in, long long *out);

}  // namespace eg

#endif
