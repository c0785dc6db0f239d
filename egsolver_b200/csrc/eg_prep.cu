/*
 * eg_prep.cu -- device preprocessing of a game before lifting:
 *
 *   - an exclusive prefix sum and a stable LSD radix sort of (key, value)
 *     pairs (8-bit digits: one counting sort per digit);
 *   - classification of vertices into (out-degree bucket, owner) classes,
 *     MG and the initial frontier (reference src/dev_EG_alg.cu:176-205,
 *     kernel_EG_initialize; reference src/egsolver.c:283-304, MG_pesi);
 *   - renumbering so that every class occupies whole 32-vertex bitmap
 *     words, with each vertex's edges packed as {successor, weight} pairs
 *     and padded to an even count for 128-bit loads;
 *   - the CSR -> CSC transpose as a deterministic counting sort (replaces
 *     cusparseScsr2csc of reference src/csr2csc.cu:57; its order equals
 *     reference src/host_csr2csc.c:15-46).
 */
#include "eg_prep.cuh"

#include <algorithm>
#include <cstdio>

namespace eg {

/* ------------------------------------------------------------------ */
/* Exclusive scan (int32), three-phase with recursion on block sums.    */
/* ------------------------------------------------------------------ */

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

/* Block-wide exclusive scan of one value per thread; returns the prefix and
 * writes the block total to *total. */
__device__ __forceinline__ int block_excl_scan(int v, int *total)
{
    __shared__ int warp_sums[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
    int incl = warp_incl_scan(v);
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        int s = lane < nw ? warp_sums[lane] : 0;
        int si = warp_incl_scan(s);
        if (lane < nw) warp_sums[lane] = si - s;
        if (lane == nw - 1) warp_sums[31] = si;
    }
    __syncthreads();
    int res = warp_sums[wid] + incl - v;
    *total = warp_sums[31];
    __syncthreads();
    return res;
}

__global__ void k_scan_tile(int *data, long long len, int *block_sums)
{
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = (base + i < len) ? data[base + i] : 0;
        s += v[i];
    }
    int total;
    int run = block_excl_scan(s, &total);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (base + i < len) data[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == 0 && block_sums) block_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(int *data, long long len, const int *block_offsets)
{
    const long long base = (long long)blockIdx.x * SCAN_TILE;
    const int add = block_offsets[blockIdx.x];
    for (int i = threadIdx.x; i < SCAN_TILE; i += blockDim.x)
        if (base + i < len) data[base + i] += add;
}

long long scan_scratch_ints(long long len)
{
    long long total = 0;
    while (len > SCAN_TILE) {
        len = (len + SCAN_TILE - 1) / SCAN_TILE;
        total += len + 1;
    }
    return total + 1;
}

void excl_scan(int *data, long long len, int *scratch, cudaStream_t st)
{
    if (len <= 0) return;
    const long long blocks = (len + SCAN_TILE - 1) / SCAN_TILE;
    if (blocks == 1) {
        k_scan_tile<<<1, SCAN_THREADS, 0, st>>>(data, len, nullptr);
        return;
    }
    int *sums = scratch;
    k_scan_tile<<<(unsigned)blocks, SCAN_THREADS, 0, st>>>(data, len, sums);
    excl_scan(sums, blocks, scratch + blocks + 1, st);
    k_scan_add<<<(unsigned)blocks, SCAN_THREADS, 0, st>>>(data, len, sums);
}

/* ------------------------------------------------------------------ */
/* Stable LSD radix sort of (key, value) pairs, 8-bit digits.           */
/* ------------------------------------------------------------------ */

constexpr int RADIX_THREADS = 256;
constexpr int RADIX_ROUNDS = 16;
constexpr int RADIX_TILE = RADIX_THREADS * RADIX_ROUNDS;

__global__ void k_radix_hist(const int *keys, long long count, int shift, int *hist, int tiles)
{
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * RADIX_TILE;
    for (int r = 0; r < RADIX_ROUNDS; r++) {
        long long i = base + (long long)r * RADIX_THREADS + threadIdx.x;
        if (i < count) atomicAdd(&h[(keys[i] >> shift) & 255], 1);
    }
    __syncthreads();
    hist[(long long)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

/* Scatter of one tile: keys are visited in index order, 256 per step; the
 * rank of a key among equal digits is (keys of this digit in earlier steps)
 * + (in earlier warps of this step) + (in earlier lanes of its warp). */
__global__ void k_radix_scatter(const int *kin, const int *vin, int *kout, int *vout, long long count,
                                int shift, const int *offsets, int tiles)
{
    __shared__ int run[256];
    __shared__ int base_off[256];
    __shared__ int wcnt[RADIX_THREADS / 32][256];
    __shared__ int step_total[256];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    run[threadIdx.x] = 0;
    base_off[threadIdx.x] = offsets[(long long)threadIdx.x * tiles + blockIdx.x];
    const long long base = (long long)blockIdx.x * RADIX_TILE;
    for (int r = 0; r < RADIX_ROUNDS; r++) {
        for (int w = 0; w < RADIX_THREADS / 32; w++) wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        const long long i = base + (long long)r * RADIX_THREADS + threadIdx.x;
        const bool valid = i < count;
        int key = 0, val = 0;
        int digit;
        if (valid) {
            key = kin[i];
            val = vin[i];
            digit = (key >> shift) & 255;
        } else {
            digit = 256 + lane; /* unique, never counted */
        }
        const unsigned peers = __match_any_sync(0xffffffffu, digit);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        if (valid && rank == 0) wcnt[wid][digit] = __popc(peers);
        __syncthreads();
        {
            int acc = 0;
            for (int w = 0; w < RADIX_THREADS / 32; w++) {
                int c = wcnt[w][threadIdx.x];
                wcnt[w][threadIdx.x] = acc;
                acc += c;
            }
            step_total[threadIdx.x] = acc;
        }
        __syncthreads();
        if (valid) {
            const long long pos = (long long)base_off[digit] + run[digit] + wcnt[wid][digit] + rank;
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
        run[threadIdx.x] += step_total[threadIdx.x];
        __syncthreads();
    }
}

long long radix_scratch_ints(long long count)
{
    long long tiles = (count + RADIX_TILE - 1) / RADIX_TILE;
    if (tiles < 1) tiles = 1;
    return 256 * tiles + scan_scratch_ints(256 * tiles) + 16;
}

/* Sorts count pairs by key (stable), keys in [0, 2^bits).  The data
 * alternate between (k0, v0) and (k1, v1); the result's buffers are
 * returned through kres / vres. */
void radix_sort_pairs(int *k0, int *v0, int *k1, int *v1, long long count, int bits, int *scratch,
                      cudaStream_t st, int **kres, int **vres)
{
    *kres = k0;
    *vres = v0;
    if (count <= 0) return;
    const int tiles = (int)((count + RADIX_TILE - 1) / RADIX_TILE);
    int *hist = scratch;
    int *scan_scr = scratch + 256LL * tiles;
    int *ka = k0, *va = v0, *kb = k1, *vb = v1;
    for (int shift = 0; shift < bits; shift += 8) {
        k_radix_hist<<<tiles, RADIX_THREADS, 0, st>>>(ka, count, shift, hist, tiles);
        excl_scan(hist, 256LL * tiles, scan_scr, st);
        k_radix_scatter<<<tiles, RADIX_THREADS, 0, st>>>(ka, va, kb, vb, count, shift, hist, tiles);
        std::swap(ka, kb);
        std::swap(va, vb);
    }
    *kres = ka;
    *vres = va;
}

int bits_for(long long max_key)
{
    int b = 0;
    while (b < 31 && (1LL << b) <= max_key) b++;
    return b < 1 ? 1 : b;
}

/* ------------------------------------------------------------------ */
/* Classification, MG and the initial frontier                          */
/* ------------------------------------------------------------------ */

/* One thread per vertex of the input CSR.  The class of v is
 * bucket(out-degree) * 2 + owner; the initial frontier follows reference
 * src/dev_EG_alg.cu:176-205: a player-0 vertex whose out-edges are all
 * negative, a player-1 vertex with a negative out-edge. */
__global__ void k_classify(int n, int n0, const long long *row_ptr, const int *w, const unsigned char *owner,
                           BucketBounds bb, int *cls_key, int *cls_val, unsigned char *active0,
                           unsigned long long *mg_acc, int *class_count)
{
    __shared__ int s_cnt[EG_MAX_CLASSES];
    __shared__ unsigned long long s_mg, s_wmax;
    if (threadIdx.x < EG_MAX_CLASSES) s_cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0) s_mg = s_wmax = 0;
    __syncthreads();
    unsigned long long mg_local = 0, wmax_local = 0;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const long long b = row_ptr[v], e = row_ptr[v + 1];
        const long long deg = e - b;
        const int own = owner ? (int)owner[v] : (v >= n0 ? 1 : 0);
        long long worst = 0; /* max(0, -min weight) */
        bool any_neg = false, all_neg = true;
        for (long long j = b; j < e; j++) {
            const long long x = w[j];
            const unsigned long long ax = (unsigned long long)(x < 0 ? -x : x);
            if (ax > wmax_local) wmax_local = ax;
            if (x < 0) {
                any_neg = true;
                if (-x > worst) worst = -x;
            } else {
                all_neg = false;
            }
        }
        mg_local += (unsigned long long)worst;
        int bucket = bb.nb - 1;
        for (int i = 0; i < bb.nb - 1; i++)
            if (deg <= bb.upper[i]) { bucket = i; break; }
        const int c = bucket * 2 + own;
        cls_key[v] = c;
        cls_val[v] = (int)v;
        active0[v] = (unsigned char)(own == 0 ? all_neg : any_neg);
        atomicAdd(&s_cnt[c], 1);
    }
    atomicAdd(&s_mg, mg_local);
    atomicMax(&s_wmax, wmax_local);
    __syncthreads();
    if (threadIdx.x < EG_MAX_CLASSES && s_cnt[threadIdx.x]) atomicAdd(&class_count[threadIdx.x], s_cnt[threadIdx.x]);
    if (threadIdx.x == 0) {
        atomicAdd(mg_acc, s_mg);
        atomicMax(mg_acc + 1, s_wmax); /* largest |weight| */
    }
}

/* sorted position i (class-major, original order inside a class) -> new id */
__global__ void k_build_perm(int n, const int *sorted_cls, const int *sorted_v, ClassTable ct, int *perm, int *iperm)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = sorted_cls[i];
        const int u = ct.start[c] + (int)(i - ct.sorted_begin[c]);
        const int v = sorted_v[i];
        perm[u] = v;
        iperm[v] = u;
    }
}

/* Padded degree of every new id (0 for ids in alignment gaps). */
__global__ void k_new_degree(int n_pad, const int *perm, const long long *row_ptr, int *pdeg)
{
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u <= n_pad; u += (long long)gridDim.x * blockDim.x) {
        int d = 0;
        if (u < n_pad) {
            const int v = perm[u];
            if (v >= 0) {
                const long long deg = row_ptr[v + 1] - row_ptr[v];
                d = (int)((deg + 1) & ~1LL);
            }
        }
        pdeg[u] = d;
    }
}

/* One warp per new vertex: writes its edge pairs {new successor, weight},
 * padding an odd count with a neutral pair (successor TOPV for a player-0
 * vertex, ZEROV for a player-1 vertex, weight 0), and the (successor,
 * source) pairs whose sort by successor gives the CSC. */
__global__ void k_copy_edges(int n_pad, const int *perm, const int *iperm, const long long *row_ptr, const int *succ,
                             const int *w, const int *P, int2 *E, int *csc_key, int *csc_val, int *indeg,
                             ClassTable ct, int topv, int zerov)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long u = warp0; u < n_pad; u += nwarps) {
        const int v = perm[u];
        if (v < 0) continue;
        const long long b = row_ptr[v], e = row_ptr[v + 1];
        const int out = P[u];
        for (long long j = b + lane; j < e; j += 32) {
            const int s = iperm[succ[j]];
            E[out + (j - b)] = make_int2(s, w[j]);
            csc_key[j] = s;
            csc_val[j] = (int)u;
            atomicAdd(&indeg[s], 1);
        }
        if (((e - b) & 1) && lane == 0) {
            const int own = ct.owner_of_new((int)u);
            E[out + (e - b)] = make_int2(own == 0 ? topv : zerov, 0);
        }
    }
}

template <class T>
__global__ void k_init_credits(int n_alloc, T *F, int topv)
{
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n_alloc; u += (long long)gridDim.x * blockDim.x)
        F[u] = (u == topv) ? credit_traits<T>::top : (T)0;
}

/* One thread per new id; a warp ballot forms each 32-vertex frontier word. */
__global__ void k_init_frontier(int n_pad, const int *perm, const unsigned char *active0, uint32_t *B)
{
    /* n_pad is a multiple of 32 and the stride a multiple of 32, so the loop
     * condition is uniform across each warp */
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n_pad; u += (long long)gridDim.x * blockDim.x) {
        const int v = perm[u];
        const bool a = v >= 0 && active0[v];
        const unsigned word = __ballot_sync(0xffffffffu, a);
        if ((threadIdx.x & 31) == 0) B[u >> 5] = word;
    }
}

/* Predecessor lists padded to a multiple of 4 entries (pad = -1), so that
 * a push reads four predecessors per 128-bit load. */
__global__ void k_round4(int len, const int *in, int *out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
        out[i] = (in[i] + 3) & ~3;
}

__global__ void k_csc_pad(int n_pad, const int *dense_off, const int *pad_off, const int *dense, int *padded)
{
    const int lane = threadIdx.x & 31;
    const long long w0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long u = w0; u < n_pad; u += nw) {
        const int db = dense_off[u], de = dense_off[u + 1], pb = pad_off[u], pe = pad_off[u + 1];
        for (int k = lane; k < pe - pb; k += 32) padded[pb + k] = (db + k < de) ? dense[db + k] : -1;
    }
}

/* ------------------------------------------------------------------ */
/* Heavy vertices cut into edge tasks                                   */
/* ------------------------------------------------------------------ */

__global__ void k_task_count(int heavy_begin, int n_pad, const int *P, int task_pairs, int *count)
{
    const int nh = n_pad - heavy_begin;
    for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h <= nh; h += (long long)gridDim.x * blockDim.x) {
        int c = 0;
        if (h < nh) {
            const int u = heavy_begin + (int)h;
            const int pairs = (P[u + 1] - P[u]) >> 1;
            c = (pairs + task_pairs - 1) / task_pairs;
        }
        count[h] = c;
    }
}

__global__ void k_task_fill(int heavy_begin, int n_pad, const int *P, int task_pairs, const int *toff, ClassTable ct,
                            int4 *tasks)
{
    const int nh = n_pad - heavy_begin;
    for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < nh; h += (long long)gridDim.x * blockDim.x) {
        const int u = heavy_begin + (int)h;
        const int b = P[u] >> 1, e = P[u + 1] >> 1;
        const int nt = toff[h + 1] - toff[h];
        if (nt == 0) continue;
        const int own = ct.owner_of_new(u);
        for (int i = 0; i < nt; i++) {
            const int pb = b + i * task_pairs;
            const int pe = pb + task_pairs < e ? pb + task_pairs : e;
            tasks[toff[h] + i] = make_int4(u, pb, pe, (nt << 1) | own);
        }
    }
}

template <class T>
__global__ void k_task_reset(int heavy_begin, int n_pad, const int *toff, ClassTable ct, T *hacc, int *hrem)
{
    const int nh = n_pad - heavy_begin;
    for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < nh; h += (long long)gridDim.x * blockDim.x) {
        const int u = heavy_begin + (int)h;
        hrem[h] = toff[h + 1] - toff[h];
        hacc[h] = ct.owner_of_new(u) ? (T)0 : credit_traits<T>::top;
    }
}

void launch_task_reset(int bits, int heavy_begin, int n_pad, const int *toff, ClassTable ct, void *hacc, int *hrem,
                       cudaStream_t st)
{
    const long long nh = n_pad - heavy_begin;
    long long g = (nh + 255) / 256;
    g = g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g);
    if (bits == 32) k_task_reset<int32_t><<<(unsigned)g, 256, 0, st>>>(heavy_begin, n_pad, toff, ct, (int32_t *)hacc, hrem);
    else k_task_reset<int64_t><<<(unsigned)g, 256, 0, st>>>(heavy_begin, n_pad, toff, ct, (int64_t *)hacc, hrem);
}

/* Credits back in original vertex order (and width). */
template <class T, class O>
__global__ void k_gather_out(int n, const int *iperm, const T *F, O *out)
{
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const T x = F[iperm[v]];
        out[v] = (x == credit_traits<T>::top) ? credit_traits<O>::top : (O)x;
    }
}

template <class T>
__global__ void k_count_top(int n_pad, const T *F, unsigned long long *out)
{
    unsigned long long c = 0;
    for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n_pad; u += (long long)gridDim.x * blockDim.x)
        c += (F[u] == credit_traits<T>::top);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

static unsigned grid_cap(long long items, int block)
{
    long long g = (items + block - 1) / block;
    return (unsigned)(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

void launch_init_credits(int bits, int n_alloc, void *F, int topv, cudaStream_t st)
{
    if (bits == 32) k_init_credits<int32_t><<<grid_cap(n_alloc, 256), 256, 0, st>>>(n_alloc, (int32_t *)F, topv);
    else k_init_credits<int64_t><<<grid_cap(n_alloc, 256), 256, 0, st>>>(n_alloc, (int64_t *)F, topv);
}

void launch_count_top(int bits, int n_pad, const void *F, unsigned long long *out, cudaStream_t st)
{
    if (bits == 32) k_count_top<int32_t><<<grid_cap(n_pad, 256), 256, 0, st>>>(n_pad, (const int32_t *)F, out);
    else k_count_top<int64_t><<<grid_cap(n_pad, 256), 256, 0, st>>>(n_pad, (const int64_t *)F, out);
}

void launch_gather_out(int in_bits, int out_bits, int n, const int *iperm, const void *F, void *out, cudaStream_t st)
{
    const unsigned g = grid_cap(n, 256);
    if (in_bits == 32 && out_bits == 32) k_gather_out<int32_t, int32_t><<<g, 256, 0, st>>>(n, iperm, (const int32_t *)F, (int32_t *)out);
    else if (in_bits == 32) k_gather_out<int32_t, int64_t><<<g, 256, 0, st>>>(n, iperm, (const int32_t *)F, (int64_t *)out);
    else if (out_bits == 32) k_gather_out<int64_t, int32_t><<<g, 256, 0, st>>>(n, iperm, (const int64_t *)F, (int32_t *)out);
    else k_gather_out<int64_t, int64_t><<<g, 256, 0, st>>>(n, iperm, (const int64_t *)F, (int64_t *)out);
}

/* ------------------------------------------------------------------ */
/* Transpose of an input CSR (values kept): the reference's csr2csc.    */
/* ------------------------------------------------------------------ */

/* One warp per row: key = column, value = edge index; also counts columns. */
__global__ void k_csr_expand(int nrows, const long long *row_ptr, const int *col, int *key, int *val, int *colcount)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = warp0; r < nrows; r += nwarps) {
        for (long long j = row_ptr[r] + lane; j < row_ptr[r + 1]; j += 32) {
            key[j] = col[j];
            val[j] = (int)j;
            atomicAdd(&colcount[col[j]], 1);
        }
    }
}

/* Row of every edge (one warp per row). */
__global__ void k_edge_rows(int nrows, const long long *row_ptr, int *row_of_edge)
{
    const int lane = threadIdx.x & 31;
    const long long warp0 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = warp0; r < nrows; r += nwarps)
        for (long long j = row_ptr[r] + lane; j < row_ptr[r + 1]; j += 32) row_of_edge[j] = (int)r;
}

__global__ void k_csc_gather(long long nnz, const int *sorted_edge, const int *row_of_edge, const int *val,
                             int *csc_row, int *csc_val)
{
    for (long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x; l < nnz; l += (long long)gridDim.x * blockDim.x) {
        const int j = sorted_edge[l];
        csc_row[l] = row_of_edge[j];
        csc_val[l] = val[j];
    }
}

__global__ void k_widen(long long len, const int *in, long long *out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
        out[i] = in[i];
}

}  // namespace eg
