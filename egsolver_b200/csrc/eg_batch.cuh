/*
 * eg_batch.cuh -- the per-game descriptor and launch interface of the
 * batched (CTA-per-game, K thresholds on K lanes) solver, shared by the
 * batch API and the serving loop.
 */
#ifndef EG_BATCH_CUH
#define EG_BATCH_CUH

#include "eg_prep.cuh"

namespace eg {

/* One game to solve at K thresholds.  Vertex ids stored in E and CS are
 * base + local id; P, CP, owner, minw, maxw and F are indexed by the local
 * id (F[local * K + k]). */
struct GameDesc {
    const int *P;              /* n + 1 offsets into E                      */
    const int2 *E;             /* {successor id, weight}                    */
    const int *CP;             /* n + 1 offsets into CS                     */
    const int *CS;             /* predecessor ids                           */
    const unsigned char *owner;
    const int *minw, *maxw;    /* min / max out-weight per vertex           */
    const int *thr;            /* K thresholds p_k                          */
    long long *F;              /* credits, n * K                            */
    long long *rounds;         /* out: rounds run                           */
    int *status;               /* out: eg_status                            */
    long long base;
    int n, K, d, pad;
};

struct BatchCtrl {
    int next_game;
    int pad;
    unsigned long long lifts, edges, num_top;
    unsigned long long t_start;
};

struct BatchParams {
    const GameDesc *games;     /* device array                              */
    const int *order;          /* queue order (largest first), or NULL      */
    BatchCtrl *ctrl;
    int num_games;
    int words_max;             /* shared bitmap words per buffer            */
    long long max_rounds;
    unsigned long long timeout_ns;
};

/* One game uploaded in the batched kernel's layout (local ids, base 0). */
struct GameLayout {
    int *P, *CP, *CS, *minw, *maxw;
    int2 *E;
    unsigned char *owner;
    int n;
    long long m;
    size_t bytes;
};
/* Device bytes a game's layout takes (plus the sort's temporaries while it
 * is built). */
size_t layout_bytes(int n, long long m);
size_t layout_build_bytes(int n, long long m);
/* Uploads the game and builds its CSC on the device (synchronous on st). */
eg_status layout_upload(const eg_game &g, cudaStream_t st, GameLayout *out);
void layout_free(GameLayout *l, cudaStream_t st);
/* A descriptor of a laid-out game for one query. */
GameDesc layout_desc(const GameLayout &l, const int *thr, long long *F, long long *rounds, int *status, int K, int d);

/* Largest game (vertices) the shared-memory frontier of the batched kernel holds. */
constexpr int kBatchMaxGameNodes = 1 << 19;

/* Resets ctrl and launches the batched kernel (lanes = KP, a power of two
 * >= every game's K) with `block` threads per CTA on `st`; *grid gets the
 * number of CTAs. */
eg_status launch_batch(const BatchParams &p, int KP, int block, int num_sms, cudaStream_t st, int *grid);

}  // namespace eg

#endif
