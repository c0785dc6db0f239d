/*
 * eg_noalloc.cu -- a CSR -> CSC transpose on device buffers that allocates
 * nothing.
 *
 * Who needs it: a caller that is not allowed to allocate device memory at
 * the moment it wants a transpose.  Typical cases are an application that
 * hands all of a GPU's memory to its own pool at start-up (a cudaMalloc
 * from inside it then fails, or steals memory the pool has promised to
 * someone else), a serving process whose latency budget has no room for
 * cudaMalloc / cudaFree (cudaFree waits for the whole device), and a plugin
 * whose host application forbids allocation after initialisation.  Such a
 * caller passes its own input and output buffers; the temporaries of the
 * counting sort live in one file-scope __device__ array of fixed size
 * instead of in cudaMalloc'd scratch.
 *
 * The array holds room for EG_NOALLOC_MAX_NNZ entries and
 * EG_NOALLOC_MAX_COLS columns (about 25 MB).  Every GPU that loads the
 * library keeps it until the process exits.  All calls share it, so two
 * calls whose work overlaps on the GPU (on different streams, or from
 * different host threads) race on it.  The array keeps the contents of the
 * last call; each call clears the column counters and the error word and
 * rewrites every sort entry below its nnz before anything reads them.
 *
 * Host code cannot name the array as a device address: its name on the
 * host is only a stand-in for the symbol.  So, once per device, with that
 * device current, the first call asks the runtime for the array's device
 * address (cudaGetSymbolAddress, return code checked) and caches it; that
 * first call on a device should therefore come before any stream capture.
 * Each call ends by reading the error word back and synchronising the
 * stream.
 */
#include "eg_prep.cuh"

#include <pthread.h>

using namespace eg;

namespace {

constexpr long long kMaxNnz = EG_NOALLOC_MAX_NNZ;
constexpr long long kMaxCols = EG_NOALLOC_MAX_COLS;
constexpr long long kSortScratch = 96 * 1024;  /* histograms + scan sums; checked against the need below */
constexpr long long kScratchInts = 5 * kMaxNnz + (kMaxCols + 1) + 32 + kSortScratch;

/* layout (ints): k0 | v0 | k1 | v1 | rows | counts (cols+1) | error word (32) | sort scratch */
constexpr long long kOffK0 = 0, kOffV0 = kMaxNnz, kOffK1 = 2 * kMaxNnz, kOffV1 = 3 * kMaxNnz, kOffRows = 4 * kMaxNnz;
constexpr long long kOffCounts = 5 * kMaxNnz;
constexpr long long kOffError = kOffCounts + kMaxCols + 1;
constexpr long long kOffSort = kOffError + 32;

pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;
constexpr int kMaxDevices = 64;
int *g_addr[kMaxDevices];

/* Every sort entry below nnz gets a defined key, edge index and row before
 * the expansion runs, so that entries a malformed row_ptr leaves unvisited
 * still hold in-range values (the sort and the gather then read only
 * indexes below nnz), never the leftovers of an earlier, larger call. */
__global__ void k_noalloc_init(long long nnz, int *key, int *val, int *rows)
{
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nnz; j += (long long)gridDim.x * blockDim.x) {
        key[j] = 0;
        val[j] = (int)j;
        rows[j] = 0;
    }
}

/* Rows with offsets outside [0, nnz] or not monotone, and columns outside
 * [0, num_cols), are skipped and flagged in the error word instead of being
 * followed out of bounds. */
__global__ void k_noalloc_expand(int nrows, int ncols, long long nnz, const long long *row_ptr, const int *col,
                                 int *key, int *val, int *rows, int *colcount, int *err)
{
    const int lane = threadIdx.x & 31;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    if (w0 == 0 && lane == 0 && (row_ptr[0] != 0 || row_ptr[nrows] != nnz)) atomicOr(err, 1);
    for (long long r = w0; r < nrows; r += nw) {
        const long long b = row_ptr[r], e = row_ptr[r + 1];
        if (b < 0 || e > nnz || b > e) {
            if (lane == 0) atomicOr(err, 1);
            continue;
        }
        for (long long j = b + lane; j < e; j += 32) {
            const int c = col[j];
            if (c < 0 || c >= ncols) {
                atomicOr(err, 2);
                key[j] = 0;
            } else {
                key[j] = c;
                atomicAdd(&colcount[c], 1);
            }
            val[j] = (int)j;
            rows[j] = (int)r;
        }
    }
}

__global__ void k_noalloc_gather(long long nnz, const int *sorted_edge, const int *rows, const int *val, int *csc_row,
                                 int *csc_val)
{
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < nnz; l += (long long)gridDim.x * blockDim.x) {
        const int j = sorted_edge[l];
        csc_row[l] = rows[j];
        csc_val[l] = val[j];
    }
}

__global__ void k_noalloc_widen(long long len, const int *in, long long *out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
        out[i] = in[i];
}

unsigned grid_of(long long items, int block)
{
    long long g = (items + block - 1) / block;
    return (unsigned)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace

static __device__ __align__(256) int g_noalloc_scratch[kScratchInts];

/* Device address of the static scratch on the current device (set-up on
 * the first call per device). */
static eg_status noalloc_scratch(int **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_NO_DEVICE, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return eg_set_error(EG_ERR_INVALID, "device ordinal %d not supported", dev);
    pthread_mutex_lock(&g_lock);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            pthread_mutex_unlock(&g_lock);
            return eg_set_error(EG_ERR_CUDA, "cudaGetSymbolAddress of the transpose scratch failed: %s",
                                cudaGetErrorString(e));
        }
        g_addr[dev] = (int *)p;
    }
    *out = g_addr[dev];
    pthread_mutex_unlock(&g_lock);
    return EG_OK;
}

extern "C" eg_status eg_csr2csc_device_noalloc(int32_t num_rows, int32_t num_cols, int64_t nnz, const int64_t *row_ptr,
                                              const int32_t *col_idx, const int32_t *val, int64_t *csc_ptr,
                                              int32_t *csc_row, int32_t *csc_val, void *stream)
{
    if (num_rows < 0 || num_cols < 0 || nnz < 0)
        return eg_set_error(EG_ERR_INVALID, "negative size");
    if (nnz > kMaxNnz || num_cols > kMaxCols)
        return eg_set_error(EG_ERR_INVALID,
                            "the allocation-free transpose holds at most %lld entries and %lld columns "
                            "(got %lld entries, %d columns); use eg_csr2csc_i32",
                            kMaxNnz, kMaxCols, (long long)nnz, num_cols);
    if (!row_ptr || !csc_ptr || (nnz && (!col_idx || !val || !csc_row || !csc_val)))
        return eg_set_error(EG_ERR_INVALID, "NULL buffer");
    if (radix_scratch_ints(nnz) + scan_scratch_ints((long long)num_cols + 1) > kSortScratch)
        return eg_set_error(EG_ERR_INVALID, "sort scratch too small for %lld entries", (long long)nnz);
    int *s = nullptr;
    eg_status st = noalloc_scratch(&s);
    if (st != EG_OK) return st;
    cudaStream_t cs = (cudaStream_t)stream;
    int *k0 = s + kOffK0, *v0 = s + kOffV0, *k1 = s + kOffK1, *v1 = s + kOffV1, *rows = s + kOffRows;
    int *counts = s + kOffCounts, *err = s + kOffError, *sort = s + kOffSort;
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(int) * ((size_t)num_cols + 1), cs);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), cs);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    k_noalloc_init<<<grid_of(nnz, 256), 256, 0, cs>>>(nnz, k0, v0, rows);
    k_noalloc_expand<<<grid_of((long long)num_rows * 32, 256), 256, 0, cs>>>(num_rows, num_cols, nnz, (const long long *)row_ptr, col_idx,
                                                                              k0, v0, rows, counts, err);
    excl_scan(counts, (long long)num_cols + 1, sort, cs);
    int *sk, *sv;
    radix_sort_pairs(k0, v0, k1, v1, nnz, bits_for(num_cols), sort, cs, &sk, &sv);
    k_noalloc_gather<<<grid_of(nnz, 256), 256, 0, cs>>>(nnz, sv, rows, val, csc_row, csc_val);
    k_noalloc_widen<<<grid_of((long long)num_cols + 1, 256), 256, 0, cs>>>((long long)num_cols + 1, counts, (long long *)csc_ptr);
    int herr = 0;
    e = cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) return eg_set_error(EG_ERR_CUDA, "allocation-free transpose failed: %s", cudaGetErrorString(e));
    if (herr & 1) return eg_set_error(EG_ERR_INVALID, "row offsets outside [0, nnz] or not monotone");
    if (herr & 2) return eg_set_error(EG_ERR_INVALID, "column index outside [0, num_cols)");
    return EG_OK;
}
