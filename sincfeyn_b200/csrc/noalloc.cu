/* noalloc.cu -- one refinement-level batch that allocates nothing.
 *
 * The usual level pass (sqb_dev_level, reached through sqb_hsum) sizes its per-child work buffers with
 * cudaMalloc and grows them on demand.  Some callers cannot let a library do that: a host program that
 * embeds the level pass in a larger GPU application whose device memory is owned by that application's
 * own pool allocator (an outside cudaMalloc can fail once the pool has taken the memory, and cudaFree
 * waits for the whole device, stalling the application's other streams), or a long-running service that
 * fixes its memory budget at start-up and must not grow it while it runs.  For them,
 * sqb_level_noalloc() runs the same kernels on scratch memory that is part of the library image: a
 * file-scope device array of SQB_NOALLOC_BYTES, which every GPU that loads the library holds until the
 * process exits.  The caller passes the inputs (the cells, on the device) and the outputs (the next
 * level's cells, on the device; sums and counters, on the host).
 *
 * Limits and rules of use:
 *   - at most SQB_NOALLOC_CHILDREN children per call (ncell << D); larger calls are rejected with
 *     SQB_NOALLOC_TOO_BIG and nothing runs: split the cells into several calls;
 *   - every call on a device shares the one array, which keeps the last call's contents; the call
 *     itself clears what must start at zero (the accumulator and the fallback queue);
 *   - calls whose GPU work overlaps (two host threads, or two streams, on one device) race on the array:
 *     issue them one after another;
 *   - the first call on each device looks up the array's device address (cudaGetSymbolAddress) with that
 *     device current; make that first call before any stream capture;
 *   - every call copies the lattice tables from host memory and waits for its stream before it returns
 *     (the sums and counters come back to the caller's host arrays): the host blocks until the call's
 *     GPU work is done.
 * No cudaMalloc, cudaFree or allocating library routine is called. */
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include "sqb_rt.h"
#include "sincfeyn_b200.h"

#define NA_CH SQB_NOALLOC_CHILDREN
/* tiles of the level tail (sqb_level_tail: SQB_TILE children each), one spare */
#define NA_TILES ((NA_CH + SQB_TILE - 1)/SQB_TILE + 1)
#define NA_UP(x) ((((long)(x)) + 255)/256*256)
/* layout of the scratch array: offsets in bytes, each a multiple of 256 */
#define NA_TAB   0L                                  /* X[255], Wt[255] */
#define NA_V     (NA_TAB + 4096L)                    /* double v[NA_CH] */
#define NA_UU    (NA_V + 8L*NA_CH)                   /* double uu[NA_CH] */
#define NA_FB    (NA_UU + 8L*NA_CH)                  /* long fb[NA_CH] */
#define NA_STT   (NA_FB + 8L*NA_CH)                  /* unsigned char stt[NA_CH] */
#define NA_BP    (NA_STT + NA_UP(NA_CH))             /* sqb_part_t per tile */
#define NA_BK    (NA_BP + NA_UP(sizeof(sqb_part_t)*NA_TILES))   /* unsigned keep count per tile */
#define NA_BO    (NA_BK + NA_UP(4L*NA_TILES))        /* unsigned long long offset per tile */
#define NA_ACC   (NA_BO + NA_UP(8L*NA_TILES))        /* sqb_acc_t */
#define NA_MISC  (NA_ACC + NA_UP(sizeof(sqb_acc_t))) /* base, fallback count */
#define NA_END   (NA_MISC + 256L)
static_assert(NA_END <= SQB_NOALLOC_BYTES, "the scratch layout must fit the array the header states");
static_assert(2*255*sizeof(double) <= 4096, "the lattice tables (|k| <= 127) must fit their slot");
static_assert(sizeof(sqb_acc_t) <= 256 && 2*sizeof(unsigned long long) <= 256, "accumulator slots");

static __device__ __align__(256) unsigned char sqb_noalloc_scratch[SQB_NOALLOC_BYTES];

extern "C" int sqb_level_tail(const void *cells, long nchildren, int D, int st, int last, int abskip, double pw, double thr,
                              const double *v, const double *uu, const unsigned char *stt,
                              void *bp, unsigned *bkeep, unsigned long long *boff, sqb_acc_t *acc, unsigned long long *base,
                              void *next, long next_cap, void *stream);
extern "C" size_t sqb_level_tile_bytes(void);
extern "C" long sqb_level_tile_children(void);
extern "C" void sqb_set_error_msg(const char *msg);

#define NA_MAXDEV 64
static unsigned char *na_base[NA_MAXDEV];   /* device address of the array, per device */
static int na_nsm[NA_MAXDEV];

extern "C" int sqb_level_noalloc(const char *graph, double h, int K, const void *cells, long ncell, int st, int last,
                                 double pw, double thr, double abserr, double nearf, double ddslack,
                                 int abskip, int abcheck, int dropunres, void *next, long next_cap,
                                 double *sums, long long *counts, void *stream){
    char msg[256];
    const sqb_graph_t *g = sqb_find_graph(graph);
    if(!g){ snprintf(msg, sizeof msg, "sqb_level_noalloc: no graph %s in this build", graph); sqb_set_error_msg(msg); return SQB_NOALLOC_BAD_ARG; }
    const int D = g->D;
    if(K < 1 || K > 127 || ncell < 0 || st < 1 || (!last && !next)){
        snprintf(msg, sizeof msg, "sqb_level_noalloc: bad arguments (K=%d, ncell=%ld, st=%d)", K, ncell, st);
        sqb_set_error_msg(msg); return SQB_NOALLOC_BAD_ARG;
    }
    const long nch = ncell << D;
    /* the tail kernels' tile size is fixed at build time; the layout above holds NA_TILES of them */
    if(sqb_level_tile_children() != SQB_TILE || sqb_level_tile_bytes() != sizeof(sqb_part_t)){
        sqb_set_error_msg("sqb_level_noalloc: the library's level-tail tiles differ from this file's layout (a build mismatch)");
        return SQB_NOALLOC_SETUP;
    }
    if(nch > NA_CH){
        snprintf(msg, sizeof msg, "sqb_level_noalloc: %ld cells of D=%d give %ld children, more than the fixed scratch holds "
                 "(%ld children per call): split the cells into several calls", ncell, D, nch, (long)NA_CH);
        sqb_set_error_msg(msg); return SQB_NOALLOC_TOO_BIG;
    }
    int dev = 0; cudaError_t e = cudaGetDevice(&dev);
    if(e != cudaSuccess || dev < 0 || dev >= NA_MAXDEV){ sqb_set_error_msg("sqb_level_noalloc: no current CUDA device"); return e ? (int)e : SQB_NOALLOC_BAD_ARG; }
    if(!na_base[dev]){
        void *p = NULL;
        e = cudaGetSymbolAddress(&p, sqb_noalloc_scratch);
        if(e != cudaSuccess || !p){ snprintf(msg, sizeof msg, "sqb_level_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e)); sqb_set_error_msg(msg); return SQB_NOALLOC_SETUP; }
        int nsm = 0; e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if(e != cudaSuccess){ sqb_set_error_msg("sqb_level_noalloc: no SM count"); return SQB_NOALLOC_SETUP; }
        na_nsm[dev] = nsm; na_base[dev] = (unsigned char*)p;
    }
    unsigned char *B = na_base[dev];
    cudaStream_t s = (cudaStream_t)stream;
    double *X = (double*)(B + NA_TAB), *Wt = X + 255;
    sqb_acc_t *acc = (sqb_acc_t*)(B + NA_ACC);
    unsigned long long *base = (unsigned long long*)(B + NA_MISC), *nfb = base + 1;
    /* the lattice tables of driver/lattice.c:18-19, and the zeroed accumulator */
    double tab[2*255];
    for(int k = -K; k <= K; k++){ tab[k + K] = exp(k*h); tab[255 + k + K] = tab[k + K]*h; }
#define NACK(x) do { cudaError_t e_ = (x); if(e_ != cudaSuccess){ snprintf(msg, sizeof msg, "sqb_level_noalloc: %s", cudaGetErrorString(e_)); sqb_set_error_msg(msg); return (int)e_; } } while(0)
    NACK(cudaMemcpyAsync(X, tab, 2*255*sizeof(double), cudaMemcpyHostToDevice, s));
    NACK(cudaMemsetAsync(acc, 0, sizeof(sqb_acc_t), s));
    NACK(cudaMemsetAsync(nfb, 0, sizeof(unsigned long long), s));
    if(nch > 0){
        sqb_eval_t a; memset(&a, 0, sizeof a);
        a.pts = cells; a.n = ncell; a.esize = 1; a.stride = SQB_MAXD; a.flag_at = SQB_PFLAG; a.cells = 1; a.st = st;
        a.X = X; a.Wt = Wt; a.K = K; a.raw = 0; a.abskip = abskip; a.abcheck = abcheck;
        a.abserr = abserr; a.near_thr = nearf*abserr; a.ddslack = ddslack;
        a.v = (double*)(B + NA_V); a.stt = B + NA_STT; a.fb = (long*)(B + NA_FB); a.nfb = nfb; a.fbcap = NA_CH;
        const size_t smem = 2*(2*K + 1)*sizeof(double);
        sqb_kattr_t at; int per = 2;
        if(g->attr(0, 128, smem, &at) && at.blocks_per_sm > 0) per = at.blocks_per_sm;
        long want = (nch + 127)/128, full = (long)na_nsm[dev]*per;
        g->f64(&a, (int)(want < full ? want : full), 128, smem, s);
        NACK(cudaGetLastError());
        sqb_dd_t d; memset(&d, 0, sizeof d);
        d.e = a; d.list = a.fb; d.nlist = nfb; d.listcap = NA_CH; d.all = 0; d.dropunres = dropunres; d.uu = (double*)(B + NA_UU);
        per = 2; if(g->attr(1, 128, smem, &at) && at.blocks_per_sm > 0) per = at.blocks_per_sm;
        g->dd(&d, na_nsm[dev]*per, 128, smem, s);
        NACK(cudaGetLastError());
        int rc = sqb_level_tail(cells, nch, D, st, last, abskip, pw, thr, a.v, d.uu, a.stt,
                                B + NA_BP, (unsigned*)(B + NA_BK), (unsigned long long*)(B + NA_BO), acc, base,
                                next, next_cap, s);
        if(rc){ sqb_set_error_msg("sqb_level_noalloc: kernel launch failed"); return rc; }
    }
    sqb_acc_t r;
    NACK(cudaMemcpyAsync(&r, acc, sizeof r, cudaMemcpyDeviceToHost, s));
    NACK(cudaStreamSynchronize(s));
    const double *src[6] = {r.S, r.A, r.drop, r.b1, r.b2, r.u};
    for(int q = 0; q < 6; q++){ sums[2*q] = src[q][0]; sums[2*q + 1] = src[q][1]; }
    counts[0] = (long long)r.ne; counts[1] = (long long)r.keep; counts[2] = (long long)r.nq;
    counts[3] = (long long)r.unres; counts[4] = (long long)r.skipped; counts[5] = (long long)r.overflow;
    return 0;
}
