/* runtime.cu -- the device layer: device state, node-batch evaluation with the precision fallback, the
 * device-resident refinement level (evaluate, fall back, reduce, keep), and the reference's GPU plug-in
 * ABI (the plain form, driver/gpu.h:12-22).
 *
 * A refinement level (driver/sum.c:652-799) is run on the device in batches of cells:
 *   1. sqb_k_f64 (per graph): every child in FP64 with the per-point tests; points whose |.| bound is
 *      above ABSERR are queued;
 *   2. sqb_k_dd (per graph): the queued points in double-double (qvalue semantics);
 *   3. sqb_k_reduce: per tile of children (in cell order, b ascending), compensated double-double sums of
 *      v*pw, |v|, the dropped weight, the shadow-tier sums and the round column, plus counters and the
 *      number of kept children;
 *   4. sqb_k_finish (one CTA): exclusive scan of the tiles' kept counts and the tiles' sums added in
 *      a fixed order into the level accumulator, so that a run is reproducible;
 *   5. sqb_k_scatter: the kept children written, in order, to the next level's cell list with their
 *      flags (skip bit, shadow tier; driver/sum.c:741-745).
 * Nothing goes back to the host until the level ends: the host reads the accumulator once per level. */
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <omp.h>
#include "sqb_rt.h"
#include "sqdd.cuh"
#include "sqorbit.cuh"
#include <atomic>
#include <vector>
#include "sincfeyn_b200.h"

extern "C" const sqb_graph_t *const SQB_ALL[];
extern "C" const int SQB_NALL;

/* Every piece of state below is per host thread (thread_local): each thread that calls the chosen form
 * has its own stream, events, buffers and error text, so several integrals can run concurrently from
 * a pool of threads (batch.cpp).  The plain form (gpu_setup ... gpu_wait) stays single-threaded, as the
 * reference's driver calls it (driver/eval.c:104-107). */
static thread_local char g_err[512];
#define CKR(x) do { cudaError_t e_ = (x); if(e_ != cudaSuccess){                                    \
    snprintf(g_err, sizeof g_err, "%s at %s:%d: %s", #x, __FILE__, __LINE__, cudaGetErrorString(e_)); \
    return (int)e_; } } while(0)

extern "C" const char *sqb_last_error(void){ return g_err; }
extern "C" void sqb_set_error_msg(const char *msg);        /* the text sqb_error() returns (engine.cpp) */

extern "C" const sqb_graph_t *sqb_find_graph(const char *name){
    for(int i = 0; i < SQB_NALL; i++) if(!strcmp(SQB_ALL[i]->name, name) || !strcmp(SQB_ALL[i]->volkov, name)) return SQB_ALL[i];
    return NULL;
}
extern "C" int sqb_ngraphs(void){ return SQB_NALL; }
extern "C" const sqb_graph_t *sqb_graph_at(int i){ return i >= 0 && i < SQB_NALL ? SQB_ALL[i] : NULL; }

/* ------------------------------------------------------------------------------------------------ */
#define RT 256                    /* threads per reduce / scatter CTA */
#define RPT 16                    /* children per thread (scatter: consecutive; reduce: RT apart) */
#define RTILE (RT*RPT)
#define FT 1024                   /* threads of the one-CTA finish kernel (32 warps) */

typedef sqb_part_t part_t;
static_assert(RTILE == SQB_TILE, "the reduce kernel's tiles are the FP64 kernel's");

/* one integral of a multi-instance level batch, for the tail kernels: its children are the launch's
 * [child0, child0 + n); its kept children go to next (cap cells), its sums to acc, its first kept slot to
 * *base */
typedef struct {
    const signed char *cells; long n, child0;
    int st, last; double pw, thr;
    sqb_pt_t *next; long cap;
    sqb_acc_t *acc; unsigned long long *base;
} lvi_t;
typedef struct {
    const signed char *cells;     /* device pt_t list (12 bytes per cell) */
    long n;                       /* children in this batch */
    int D, st, last, abskip;
    double pw, thr;
    const double *v, *uu;
    const unsigned char *stt;
    sqb_sym_t sym;                /* the symmetry fold (sym.n <= 1: off) */
    const unsigned char *cfl;     /* the predictor's per-child tiers at the last level (NULL: the parent's) */
    int ninst;                    /* > 0: a multi-instance batch, the integrals in inst (the fields above that
                                     describe one batch unused); 0: one batch */
    lvi_t inst[SQB_MAXINST];
    const unsigned char *cw;      /* list mode: every child's orbit weight from the select pass (0: not evaluated) */
} lvl_t;

struct Dev {
    int on, dev, nsm;
    cudaEvent_t t0, t1; void *flush; size_t flushn;
    unsigned long long launches;   /* kernels of this library launched so far */
    cudaEvent_t kev[3*256]; int nkev, kevn;   /* kernel timing: (FP64 start, FP64 end / dd start, dd end) per pass */
    double f64_ms, dd_ms; long f64_n;
    char info[256];
    cudaStream_t s;
    cudaEvent_t e0, e1;
    double *X, *Wt; int tabcap, K;
    long cap;                      /* points per batch */
    double *v, *uu; unsigned char *stt, *cfl, *cw; long *fb; unsigned long long *nfb;
    unsigned long long *sel, *nsel;   /* list mode: the children to evaluate and their number */
    long nbcap; part_t *bp; unsigned *bkeep; unsigned long long *boff; unsigned char *tfb;
    long ttcap; double *tt, *ta;   /* split FP64 pass: running sums per point */
    sqb_acc_t *acc; unsigned long long *base;
    sqb_acc_t *accm; unsigned long long *basem, *queue;   /* multi-instance levels: per integral, tile queue */
    long dcap; sqb_pt_t *dpts; unsigned char *dskip;
    long hcap; sqb_pt_t *hpts; unsigned char *hskip, *hst; double *hv, *huu;
};
static thread_local Dev G;
static int KTIME;                  /* sqb_kernel_timing(): all threads */
static std::atomic<unsigned long long> H2D, D2H;   /* bytes copied by the chosen form's calls, all threads */

/* the timed passes so far: their events are read once the stream has passed them (the callers that wait
 * on the stream anyway), so timing adds no synchronisation between a level's batches */
static void ktime_collect(void){
    if(!G.nkev) return;
    cudaEventSynchronize(G.kev[3*G.nkev - 1]);
    for(int i = 0; i < G.nkev; i++){
        float x = 0, y = 0;
        cudaEventElapsedTime(&x, G.kev[3*i], G.kev[3*i + 1]); cudaEventElapsedTime(&y, G.kev[3*i + 1], G.kev[3*i + 2]);
        G.f64_ms += x; G.dd_ms += y; G.f64_n++;
    }
    G.nkev = 0;
}
/* the event triple of the next timed pass (NULL: timing off or no events) */
static cudaEvent_t *ktime_slot(void){
    if(!KTIME) return NULL;
    const int cap = (int)(sizeof G.kev/sizeof G.kev[0])/3;
    if(G.nkev == cap) ktime_collect();
    if(G.nkev >= G.kevn){
        for(int j = 0; j < 3; j++) if(cudaEventCreate(&G.kev[3*G.nkev + j]) != cudaSuccess) return NULL;
        G.kevn = G.nkev + 1;
    }
    return &G.kev[3*G.nkev++];
}

extern "C" int sqb_dev_init(int device){
    if(G.on) return 0;
    int nd = 0; CKR(cudaGetDeviceCount(&nd));
    if(nd == 0){ snprintf(g_err, sizeof g_err, "no CUDA device"); return -1; }
    if(device < 0 || device >= nd) device = 0;
    CKR(cudaSetDevice(device));
    cudaDeviceProp p; CKR(cudaGetDeviceProperties(&p, device));
    G.dev = device; G.nsm = p.multiProcessorCount;
    snprintf(G.info, sizeof G.info, "%s (sm_%d%d, %d SMs)", p.name, p.major, p.minor, p.multiProcessorCount);
    CKR(cudaStreamCreateWithFlags(&G.s, cudaStreamNonBlocking));
    /* the cell lists and the grow's tables come from the device's stream-ordered pool, which keeps
     * freed memory for the next integral instead of returning it (no cudaFree synchronisation) */
    { cudaMemPool_t pool; CKR(cudaDeviceGetDefaultMemPool(&pool, device));
      unsigned long long keep = ~0ULL; CKR(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)); }
    CKR(cudaEventCreate(&G.e0)); CKR(cudaEventCreate(&G.e1));
    CKR(cudaEventCreate(&G.t0)); CKR(cudaEventCreate(&G.t1));
    CKR(cudaMalloc(&G.acc, sizeof(sqb_acc_t)));
    CKR(cudaMalloc(&G.base, sizeof(unsigned long long)));
    CKR(cudaMalloc(&G.nfb, sizeof(unsigned long long)));
    CKR(cudaMalloc(&G.accm, SQB_MAXINST*sizeof(sqb_acc_t)));
    CKR(cudaMalloc(&G.basem, SQB_MAXINST*sizeof(unsigned long long)));
    CKR(cudaMalloc(&G.queue, sizeof(unsigned long long)));
    CKR(cudaMalloc(&G.nsel, sizeof(unsigned long long)));
    G.on = 1;
    return 0;
}
extern "C" const char *sqb_dev_info(void){ return G.on ? G.info : "off"; }

extern "C" int sqb_dev_tables(const double *X, const double *Wt, int K){
    int nt = 2*K + 1;
    if(nt > G.tabcap){
        if(G.X){ cudaFree(G.X); cudaFree(G.Wt); }
        CKR(cudaMalloc(&G.X, nt*sizeof(double))); CKR(cudaMalloc(&G.Wt, nt*sizeof(double)));
        G.tabcap = nt;
    }
    CKR(cudaMemcpy(G.X, X, nt*sizeof(double), cudaMemcpyHostToDevice));
    CKR(cudaMemcpy(G.Wt, Wt, nt*sizeof(double), cudaMemcpyHostToDevice));
    H2D += 2*nt*sizeof(double);
    G.K = K;
    return 0;
}

static int reserve_points(long n){
    if(n <= G.cap) return 0;
    long c = 1L << 16; while(c < n) c <<= 1;
    if(G.v){ cudaFree(G.v); cudaFree(G.uu); cudaFree(G.stt); cudaFree(G.cfl); cudaFree(G.cw); cudaFree(G.fb); cudaFree(G.sel);
             cudaFree(G.bp); cudaFree(G.bkeep); cudaFree(G.boff); cudaFree(G.tfb); }
    CKR(cudaMalloc(&G.v, c*sizeof(double))); CKR(cudaMalloc(&G.uu, c*sizeof(double)));
    CKR(cudaMalloc(&G.stt, c)); CKR(cudaMalloc(&G.cfl, c)); CKR(cudaMalloc(&G.cw, c)); CKR(cudaMalloc(&G.fb, c*sizeof(long)));
    CKR(cudaMalloc(&G.sel, c*sizeof(unsigned long long)));
    long nb = (c + RTILE - 1)/RTILE;
    CKR(cudaMalloc(&G.bp, nb*sizeof(part_t))); CKR(cudaMalloc(&G.bkeep, nb*sizeof(unsigned))); CKR(cudaMalloc(&G.tfb, nb));
    CKR(cudaMalloc(&G.boff, nb*sizeof(unsigned long long)));
    G.cap = c; G.nbcap = nb;
    return 0;
}

/* the FP64 kernel to run: the contracted one (which 2) when asked for and built, else the exact one */
static inline int f64_which(const sqb_graph_t *g, int fma){ return fma && g->f64_fma ? 2 : 0; }
static inline void launch_f64(const sqb_graph_t *g, int which, const sqb_eval_t *a, int grid, size_t smem, cudaStream_t s){
    if(which == 2) g->f64_fma(a, grid, 128, smem, s); else g->f64(a, grid, 128, smem, s);
}

/* resident CTAs of a graph's kernel on the whole device (which | SQB_ATTR_LEVEL: its level kernel); *fused:
 * the kernel sums level tiles itself; *sweeps: the level kernel's passes over a batch's tiles */
static long grid_cap(const sqb_graph_t *g, int which, size_t smem, int *fused = NULL, int *sweeps = NULL){
    sqb_kattr_t at; memset(&at, 0, sizeof at); int per = 2;
    const int ok = g->attr(which, 128, smem, &at);
    if(ok && at.blocks_per_sm > 0) per = at.blocks_per_sm;
    if(fused) *fused = ok && at.fused;
    if(sweeps) *sweeps = ok && at.sweeps > 1 ? at.sweeps : 1;
    return (long)G.nsm*per;
}

static int grid_for(const sqb_graph_t *g, int which, long npts, size_t smem){
    sqb_kattr_t at; int per = 2;
    if(g->attr(which, 128, smem, &at) && at.blocks_per_sm > 0) per = at.blocks_per_sm;
    long want = (npts + 127)/128, full = (long)G.nsm*per;
    if(want < 1) want = 1;
    return (int)(want < full ? want : full);
}

static void fill_eval(sqb_eval_t *a, const sqb_test_t *t){
    a->X = G.X; a->Wt = G.Wt; a->K = G.K; a->H = 0; a->raw = 0;
    a->abskip = t->abskip; a->abcheck = t->abcheck;
    a->abserr = t->abserr; a->near_thr = t->nearf*t->abserr; a->ddslack = t->ddslack;
    a->v = G.v; a->ab = NULL; a->stt = G.stt; a->fb = G.fb; a->nfb = G.nfb; a->fbcap = G.cap;
}

/* whether a batch's FP64 pass runs in passes (the graph has them, they are asked for, a level batch) */
static inline bool use_split(const sqb_graph_t *g, const sqb_eval_t *a, const sqb_test_t *t){
    return t->split && g->nparts > 0 && a->cells && !t->alldd;
}

/* FP64 pass (or the all-dd pass) and the fallback pass for one batch already described by a */
/* dynamic shared memory of a launch: the tables of its integral(s), 2(2K+1) doubles each */
static size_t table_bytes(const sqb_eval_t *a){
    if(a->ninst <= 0) return 2*(2*(size_t)a->K + 1)*sizeof(double);
    size_t w = 0;
    for(int q = 0; q < a->ninst; q++) w += 2*(2*(size_t)a->inst[q].K + 1);
    return w*sizeof(double);
}

/* SQB_TILE_SUMS (environment, read once): 1 (default) = a level batch's FP64 kernel sums the tiles that
 * need no fallback itself; 0 = the reduce kernel sums every tile */
static int tile_sums(void){
    static int v = -1;
    if(v < 0){ const char *e = getenv("SQB_TILE_SUMS"); v = e && *e ? atoi(e) != 0 : 1; }
    return v;
}

static int eval_batch(const sqb_graph_t *g, sqb_eval_t *a, const sqb_test_t *t, long npts){
    /* the tables, then (level launches) the FP64 kernel's tile-sum columns */
    size_t smem = table_bytes(a) + (a->part ? sizeof(sqb_tile_acc) : 0);
    sqb_dd_t d; memset(&d, 0, sizeof d);
    d.e = *a; d.dropunres = t->dropunres; d.uu = G.uu;
    if(t->alldd){
        d.all = 1;
        g->dd(&d, grid_for(g, 1, npts, smem), 128, smem, G.s);
        CKR(cudaGetLastError());
        G.launches++;
        return 0;
    }
    CKR(cudaMemsetAsync(G.nfb, 0, sizeof(unsigned long long), G.s));
    cudaEvent_t *ev = ktime_slot();
    if(ev) CKR(cudaEventRecord(ev[0], G.s));
    if(use_split(g, a, t)){
        if(npts > G.ttcap){
            if(G.tt){ cudaFree(G.tt); cudaFree(G.ta); }
            long c = 1L << 16; while(c < npts) c <<= 1;
            CKR(cudaMalloc(&G.tt, c*sizeof(double))); CKR(cudaMalloc(&G.ta, c*sizeof(double)));
            G.ttcap = c;
        }
        for(int P = 0; P <= g->nparts; P++){
            sqb_kattr_t at; memset(&at, 0, sizeof at); int per = 2;
            if(g->split_attr(P, t->fma, 128, smem, &at) && at.blocks_per_sm > 0) per = at.blocks_per_sm;
            long want = (npts + 127)/128, full = (long)G.nsm*per;
            g->split(P, t->fma, a, G.tt, G.ta, (int)(want < full ? want : full), 128, smem, G.s);
            CKR(cudaGetLastError());
        }
        G.launches += g->nparts;
    } else {
        const int w = f64_which(g, t->fma);
        if(a->ninst > 0){
            CKR(cudaMemsetAsync(a->queue, 0, sizeof(unsigned long long), G.s));
            int sw = 1;
            const long cap = grid_cap(g, w | (sqb_level_launch(a) ? SQB_ATTR_LEVEL : 0), smem, NULL, &sw);
            const long items = a->ntile*sw;       /* the level kernel may take every tile twice */
            launch_f64(g, w, a, (int)(items < cap ? items : cap), smem, G.s);
        } else launch_f64(g, w, a, grid_for(g, w, npts, smem), smem, G.s);
        CKR(cudaGetLastError());
    }
    if(ev) CKR(cudaEventRecord(ev[1], G.s));
    d.list = G.fb; d.nlist = G.nfb; d.listcap = G.cap; d.all = 0;
    /* the queue length is known only on the device: a persistent grid reads it */
    g->dd(&d, grid_for(g, 1, 1L << 30, smem), 128, smem, G.s);
    CKR(cudaGetLastError());
    G.launches += 2;
    if(ev) CKR(cudaEventRecord(ev[2], G.s));
    return 0;
}

extern "C" int sqb_dev_eval_nodes(const sqb_graph_t *g, long n, const sqb_pt_t *pts, const unsigned char *skip,
                                  const sqb_test_t *t, double *v, unsigned char *near, long *nq, double *u, long *unres){
    if(n <= 0) return 0;
    const long CH = 1L << 22;
    long m0 = n < CH ? n : CH;
    if(reserve_points(m0)) return -1;
    if(m0 > G.dcap){
        if(G.dpts){ cudaFree(G.dpts); cudaFree(G.dskip); cudaFreeHost(G.hpts); cudaFreeHost(G.hskip); cudaFreeHost(G.hv); cudaFreeHost(G.hst); cudaFreeHost(G.huu); }
        long c = 1L << 16; while(c < m0) c <<= 1;
        CKR(cudaMalloc(&G.dpts, c*sizeof(sqb_pt_t))); CKR(cudaMalloc(&G.dskip, c));
        CKR(cudaMallocHost(&G.hpts, c*sizeof(sqb_pt_t))); CKR(cudaMallocHost(&G.hskip, c));
        CKR(cudaMallocHost(&G.hv, c*sizeof(double))); CKR(cudaMallocHost(&G.hst, c)); CKR(cudaMallocHost(&G.huu, c*sizeof(double)));
        G.dcap = c; G.hcap = c;
    }
    long q = 0, nd = 0; double uu = 0;
    for(long i0 = 0; i0 < n; i0 += CH){
        long m = n - i0 < CH ? n - i0 : CH;
        memcpy(G.hpts, pts + i0, m*sizeof(sqb_pt_t));
        CKR(cudaMemcpyAsync(G.dpts, G.hpts, m*sizeof(sqb_pt_t), cudaMemcpyHostToDevice, G.s));
        if(skip){ memcpy(G.hskip, skip + i0, m); CKR(cudaMemcpyAsync(G.dskip, G.hskip, m, cudaMemcpyHostToDevice, G.s)); }
        H2D += m*sizeof(sqb_pt_t) + (skip ? m : 0); D2H += m*(2*sizeof(double) + 1);
        sqb_eval_t a; memset(&a, 0, sizeof a); fill_eval(&a, t);
        a.pts = G.dpts; a.n = m; a.esize = 1; a.stride = SQB_MAXD; a.flag_at = -1; a.cells = 0; a.st = 0;
        a.skip = skip ? G.dskip : NULL;
        if(eval_batch(g, &a, t, m)) return -1;
        CKR(cudaMemcpyAsync(G.hv, G.v, m*sizeof(double), cudaMemcpyDeviceToHost, G.s));
        CKR(cudaMemcpyAsync(G.hst, G.stt, m, cudaMemcpyDeviceToHost, G.s));
        CKR(cudaMemcpyAsync(G.huu, G.uu, m*sizeof(double), cudaMemcpyDeviceToHost, G.s));
        CKR(cudaStreamSynchronize(G.s));
        for(long i = 0; i < m; i++){
            unsigned char s = G.hst[i];
            v[i0 + i] = G.hv[i];
            if(near) near[i0 + i] = (s & SQB_NEAR) ? 1 : 0;
            if(s & SQB_FALLBACK){ q++; uu += G.huu[i]; }
            if(s & SQB_UNRES) nd++;
        }
    }
    *nq += q; *u += uu; *unres += nd;
    return 0;
}

/* n device-resident nodes (pt_t, flags ignored; skip per node on the device or NULL): values and status
 * to the host; the device copies stay valid until the next evaluation (*v_dev, *stt_dev) */
extern "C" int sqb_dev_eval_resident(const sqb_graph_t *g, const sqb_pt_t *pts, long n, const unsigned char *skip,
                                     const sqb_test_t *t, double *v, unsigned char *stt, long *nq, double *u, long *unres,
                                     const double **v_dev, const unsigned char **stt_dev){
    *v_dev = NULL; *stt_dev = NULL;
    if(n <= 0) return 0;
    if(reserve_points(n)) return -1;
    if(n > G.hcap){
        if(G.hv){ cudaFreeHost(G.hv); cudaFreeHost(G.hst); cudaFreeHost(G.huu); cudaFreeHost(G.hpts); cudaFreeHost(G.hskip); }
        long c = 1L << 16; while(c < n) c <<= 1;
        CKR(cudaMallocHost(&G.hv, c*sizeof(double))); CKR(cudaMallocHost(&G.hst, c)); CKR(cudaMallocHost(&G.huu, c*sizeof(double)));
        CKR(cudaMallocHost(&G.hpts, c*sizeof(sqb_pt_t))); CKR(cudaMallocHost(&G.hskip, c));
        G.hcap = c;
    }
    sqb_eval_t a; memset(&a, 0, sizeof a); fill_eval(&a, t);
    a.pts = pts; a.n = n; a.esize = 1; a.stride = SQB_MAXD; a.flag_at = -1; a.cells = 0; a.st = 0; a.skip = skip;
    if(eval_batch(g, &a, t, n)) return -1;
    CKR(cudaMemcpyAsync(G.hv, G.v, n*sizeof(double), cudaMemcpyDeviceToHost, G.s));
    CKR(cudaMemcpyAsync(G.hst, G.stt, n, cudaMemcpyDeviceToHost, G.s));
    CKR(cudaMemcpyAsync(G.huu, G.uu, n*sizeof(double), cudaMemcpyDeviceToHost, G.s));
    CKR(cudaStreamSynchronize(G.s));
    D2H += n*(2*sizeof(double) + 1);
    long q = 0, nd = 0; double uu = 0;
    memcpy(v, G.hv, n*sizeof(double)); memcpy(stt, G.hst, n);
    for(long i = 0; i < n; i++){
        const unsigned char s = G.hst[i];
        if(s & SQB_FALLBACK){ q++; uu += G.huu[i]; }
        if(s & SQB_UNRES) nd++;
    }
    *nq += q; *u += uu; *unres += nd;
    *v_dev = G.v; *stt_dev = G.stt;
    return 0;
}
extern "C" void *sqb_dev_stream(void){ return (void*)G.s; }

/* Load the device code of a graph's kernels now (NULL: every graph).  CUDA loads a kernel's code on
 * its first launch by default (lazy loading); for this library's large per-graph kernels that first
 * launch costs up to a second, so a caller that times integrals, or wants the cost at start-up,
 * preloads.  Returns the number of kernels loaded, or -1. */
extern "C" int sqb_preload(const char *graph){
    if(sqb_dev_init(0)) return -1;
    int n = 0;
    for(int i = 0; i < SQB_NALL; i++){
        const sqb_graph_t *g = SQB_ALL[i];
        if(graph && strcmp(graph, g->name)) continue;
        sqb_kattr_t at;
        for(int which = 0; which < 3; which++) if(g->attr(which, 128, 4096, &at)) n++;
        for(int P = 0; P <= g->nparts && g->nparts > 0; P++)
            for(int fma = 0; fma < 2; fma++) if(g->split_attr(P, fma, 128, 4096, &at)) n++;
    }
    return n;
}
/* instrumentation: kernels launched so far; with ktime on, the FP64 and double-double kernels of every
 * evaluation pass are bracketed by events, read when the host next waits on the stream, and their times
 * summed */
extern "C" unsigned long long sqb_launch_count(void){ return G.launches; }
extern "C" void sqb_kernel_timing(int on){ KTIME = on; }
extern "C" void sqb_kernel_times(double *f64_ms, double *dd_ms, long *f64_launches, int reset){
    ktime_collect();
    *f64_ms = G.f64_ms; *dd_ms = G.dd_ms; *f64_launches = G.f64_n;
    if(reset){ G.f64_ms = G.dd_ms = 0; G.f64_n = 0; }
}

/* ---------------------------------------- level reduce ------------------------------------------ */
__device__ __forceinline__ sqdd shfl_dd(const sqdd &a, int off){
    return sqdd(__shfl_down_sync(0xffffffffu, a.hi, off), __shfl_down_sync(0xffffffffu, a.lo, off));
}
/* the integral of tile b of a batch (one batch: the batch itself, with child0 = 0) */
__device__ __forceinline__ lvi_t lvl_inst(const lvl_t &a, long b){
    lvi_t v;
    if(a.ninst <= 0){
        v.cells = a.cells; v.n = a.n; v.child0 = 0; v.st = a.st; v.last = a.last; v.pw = a.pw; v.thr = a.thr;
        v.next = NULL; v.cap = 0; v.acc = NULL; v.base = NULL;
        return v;
    }
    int k = 0;
    for(int q = 1; q < a.ninst; q++) if(a.inst[q].child0 <= b*(long)RTILE) k = q;
    return a.inst[k];
}
/* child il's coordinates k_d - st bit_d(b) (driver/sum.c:407) */
__device__ __forceinline__ void child_of(const lvl_t &a, const lvi_t &L, long il, int *k){
    const long c = il >> a.D; const int b = (int)(il & ((1L << a.D) - 1));
    const signed char *p = L.cells + c*SQB_MAXD;
    for(int d = 0; d < a.D; d++) k[d] = p[d] - (((b >> d) & 1) ? L.st : 0);
}
/* a present child's multiplicity: its orbit size under a fold, else 1 */
__device__ __forceinline__ int child_weight(const lvl_t &a, const lvi_t &L, long il){
    if(a.cw) return a.cw[il];
    if(a.sym.n <= 1) return 1;
    int k[SQB_MAXD];
    child_of(a, L, il, k);
    return sqb_orbit_n(a.sym, k, a.D);
}

__device__ __forceinline__ int parent_tier(const lvl_t &a, const lvi_t &L, long i, long il){
    if(a.cfl) return (a.cfl[i] >> 1) & 3;
    const long c = il >> a.D;
    return (L.cells[c*SQB_MAXD + SQB_PFLAG] >> 1) & 3;
}

/* per tile of RTILE children: S = sum v*pw and the shadow-tier sums in double-double per thread (they
 * can cancel), sum |v|, the dropped weight and the round column (non-negative) in double per thread,
 * then double-double across threads in a fixed tree.  Thread t of the tile takes children t, t + RT,
 * t + 2 RT, ... (each warp reads 256 contiguous bytes of v per step); the order is fixed, so a run is
 * reproducible. */
__global__ void __launch_bounds__(RT) sqb_k_reduce(const __grid_constant__ lvl_t a, part_t *bp, unsigned *bkeep,
                                                   const unsigned char *tfb){
    if(tfb && !tfb[blockIdx.x]) return;      /* summed by the FP64 pass already (no fallback point in it) */
    const lvi_t L = lvl_inst(a, blockIdx.x);
    const long t0 = blockIdx.x*(long)RTILE + threadIdx.x;
    sqdd S, b1, b2;
    double A = 0, dr = 0, uu = 0;
    unsigned ne = 0, nq = 0, nu = 0, nsk = 0, keep = 0;
    for(int j = 0; j < RPT; j++){
        const long i = t0 + (long)j*RT, il = i - L.child0;
        if(il >= L.n) break;
        const unsigned char s = a.stt[i];
        if(!(s & SQB_PRESENT)) continue;
        /* a folded point stands for its orbit: (mw v) pw and mw |v| (driver/sum.c:734-745) */
        const int mw = child_weight(a, L, il);
        const double m = (double)mw, v = a.v[i], vp = (m*v)*L.pw, av = fabs(v);
        S = sqdd_add_d(S, vp); A += m*av; ne++;
        nsk += (s & SQB_SKIPPED) ? 1 : 0;
        if(s & SQB_FALLBACK){ nq++; uu += a.uu[i]; }
        if(s & SQB_UNRES) nu++;
        if(L.last){
            const int te = parent_tier(a, L, i, il);
            if(te >= 1) b1 = sqdd_add_d(b1, vp);
            if(te >= 2) b2 = sqdd_add_d(b2, vp);
        } else if(av >= L.thr) keep += mw;
        else dr += (m*av)*L.pw;
    }
    sqdd Ad(A), dd(dr), ud(uu);
    for(int off = 16; off; off >>= 1){
        S = S + shfl_dd(S, off); Ad = Ad + shfl_dd(Ad, off); dd = dd + shfl_dd(dd, off);
        b1 = b1 + shfl_dd(b1, off); b2 = b2 + shfl_dd(b2, off); ud = ud + shfl_dd(ud, off);
        ne += __shfl_down_sync(0xffffffffu, ne, off); nq += __shfl_down_sync(0xffffffffu, nq, off);
        nu += __shfl_down_sync(0xffffffffu, nu, off); nsk += __shfl_down_sync(0xffffffffu, nsk, off);
        keep += __shfl_down_sync(0xffffffffu, keep, off);
    }
    __shared__ double wd[RT/32][12];
    __shared__ unsigned wc[RT/32][5];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if(l == 0){
        wd[w][0] = S.hi; wd[w][1] = S.lo; wd[w][2] = Ad.hi; wd[w][3] = Ad.lo; wd[w][4] = dd.hi; wd[w][5] = dd.lo;
        wd[w][6] = b1.hi; wd[w][7] = b1.lo; wd[w][8] = b2.hi; wd[w][9] = b2.lo; wd[w][10] = ud.hi; wd[w][11] = ud.lo;
        wc[w][0] = ne; wc[w][1] = nq; wc[w][2] = nu; wc[w][3] = nsk; wc[w][4] = keep;
    }
    __syncthreads();
    if(w == 0){
        const int nw = RT/32;
        sqdd x[6]; unsigned c[5];
        for(int q = 0; q < 6; q++) x[q] = l < nw ? sqdd(wd[l][2*q], wd[l][2*q + 1]) : sqdd(0.0);
        for(int q = 0; q < 5; q++) c[q] = l < nw ? wc[l][q] : 0;
        for(int off = nw/2; off; off >>= 1){
            for(int q = 0; q < 6; q++) x[q] = x[q] + shfl_dd(x[q], off);
            for(int q = 0; q < 5; q++) c[q] += __shfl_down_sync(0xffffffffu, c[q], off);
        }
        if(l == 0){
            part_t p;
            p.S[0] = x[0].hi; p.S[1] = x[0].lo; p.A[0] = x[1].hi; p.A[1] = x[1].lo; p.drop[0] = x[2].hi; p.drop[1] = x[2].lo;
            p.b1[0] = x[3].hi; p.b1[1] = x[3].lo; p.b2[0] = x[4].hi; p.b2[1] = x[4].lo; p.u[0] = x[5].hi; p.u[1] = x[5].lo;
            p.ne = c[0]; p.nq = c[1]; p.unres = c[2]; p.skipped = c[3];
            bp[blockIdx.x] = p; bkeep[blockIdx.x] = c[4];
        }
    }
}

/* one CTA per integral: the tiles' offsets (exclusive scan of their kept counts) and the batch's sums, in
 * a fixed order (each thread a contiguous run of tiles, then a fixed tree), added into the level
 * accumulator; *base = this batch's first slot in the next list.  One batch (a.ninst = 0): its nb tiles
 * into acc and base; a multi-instance batch: CTA k takes integral k's tiles into its own acc and base */
__global__ void __launch_bounds__(FT) sqb_k_finish(const __grid_constant__ lvl_t a, const part_t *bp, const unsigned *bkeep,
                                                   long nb, unsigned long long *boff, sqb_acc_t *acc,
                                                   unsigned long long *base){
    long tb = 0;
    if(a.ninst > 0){
        const lvi_t &L = a.inst[blockIdx.x];
        tb = L.child0/RTILE; nb = (L.n + RTILE - 1)/RTILE; acc = L.acc; base = L.base;
    }
    bp += tb; bkeep += tb; boff += tb;
    const int t = threadIdx.x, w = t >> 5, l = t & 31;
    const long ch = (nb + FT - 1)/FT, j0 = t*ch, j1 = j0 + ch < nb ? j0 + ch : nb;
    sqdd x[6]; unsigned long long c[5] = {0, 0, 0, 0, 0};
    for(long j = j0; j < j1; j++){
        const part_t &p = bp[j];
        x[0] = x[0] + sqdd(p.S[0], p.S[1]); x[1] = x[1] + sqdd(p.A[0], p.A[1]); x[2] = x[2] + sqdd(p.drop[0], p.drop[1]);
        x[3] = x[3] + sqdd(p.b1[0], p.b1[1]); x[4] = x[4] + sqdd(p.b2[0], p.b2[1]); x[5] = x[5] + sqdd(p.u[0], p.u[1]);
        c[0] += p.ne; c[1] += p.nq; c[2] += p.unres; c[3] += p.skipped; c[4] += bkeep[j];
    }
    /* exclusive scan of the kept counts: warp scan, then across warps */
    __shared__ unsigned long long wsum[FT/32], wpre[FT/32];
    unsigned long long inc = c[4];
    for(int off = 1; off < 32; off <<= 1){ unsigned long long y = __shfl_up_sync(0xffffffffu, inc, off); if(l >= off) inc += y; }
    if(l == 31) wsum[w] = inc;
    /* the sums: warp tree, then the warps' results */
    for(int off = 16; off; off >>= 1){
        for(int q = 0; q < 6; q++) x[q] = x[q] + shfl_dd(x[q], off);
        for(int q = 0; q < 4; q++) c[q] += __shfl_down_sync(0xffffffffu, c[q], off);
    }
    __shared__ double wd[FT/32][12];
    __shared__ unsigned long long wc[FT/32][4];
    if(l == 0){ for(int q = 0; q < 6; q++){ wd[w][2*q] = x[q].hi; wd[w][2*q + 1] = x[q].lo; } for(int q = 0; q < 4; q++) wc[w][q] = c[q]; }
    __syncthreads();
    if(t == 0){ unsigned long long s = 0; for(int q = 0; q < FT/32; q++){ wpre[q] = s; s += wsum[q]; } }
    __syncthreads();
    { unsigned long long o = wpre[w] + inc - c[4]; for(long j = j0; j < j1; j++){ boff[j] = o; o += bkeep[j]; } }
    if(w == 0){
        sqdd y[6]; unsigned long long d[4];
        for(int q = 0; q < 6; q++) y[q] = sqdd(wd[l][2*q], wd[l][2*q + 1]);
        for(int q = 0; q < 4; q++) d[q] = wc[l][q];
        for(int off = 16; off; off >>= 1){
            for(int q = 0; q < 6; q++) y[q] = y[q] + shfl_dd(y[q], off);
            for(int q = 0; q < 4; q++) d[q] += __shfl_down_sync(0xffffffffu, d[q], off);
        }
        if(l == 0){
            const unsigned long long total = wpre[FT/32 - 1] + wsum[FT/32 - 1];
            double *dst[6] = {acc->S, acc->A, acc->drop, acc->b1, acc->b2, acc->u};
            for(int q = 0; q < 6; q++){ sqdd z = sqdd(dst[q][0], dst[q][1]) + y[q]; dst[q][0] = z.hi; dst[q][1] = z.lo; }
            acc->ne += d[0]; acc->nq += d[1]; acc->unres += d[2]; acc->skipped += d[3];
            *base = acc->keep; acc->keep += total;
        }
    }
}

__global__ void __launch_bounds__(RT) sqb_k_scatter(const __grid_constant__ lvl_t a, const unsigned long long *boff,
                                                    const unsigned long long *base, sqb_pt_t *next, long cap,
                                                    unsigned long long *overflow){
    const lvi_t L = lvl_inst(a, blockIdx.x);
    if(a.ninst > 0){ base = L.base; next = L.next; cap = L.cap; overflow = &L.acc->overflow; }
    const long t0 = blockIdx.x*(long)RTILE + threadIdx.x*(long)RPT;
    unsigned mask = 0; int cnt = 0;
    for(int j = 0; j < RPT; j++){
        const long i = t0 + j, il = i - L.child0;
        if(il >= L.n) break;
        if((a.stt[i] & SQB_PRESENT) && fabs(a.v[i]) >= L.thr){ mask |= 1u << j; cnt += child_weight(a, L, il); }
    }
    /* block exclusive scan of cnt */
    __shared__ int ws[RT/32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    int x = cnt;
    for(int off = 1; off < 32; off <<= 1){ int y = __shfl_up_sync(0xffffffffu, x, off); if(l >= off) x += y; }
    if(l == 31) ws[w] = x;
    __syncthreads();
    if(threadIdx.x == 0){ int s = 0; for(int j = 0; j < RT/32; j++){ int y = ws[j]; ws[j] = s; s += y; } }
    __syncthreads();
    unsigned long long o = *base + boff[blockIdx.x] + (unsigned long long)(ws[w] + x - cnt);
    const double thr10 = 10*L.thr, thr100 = 100*L.thr;
    for(int j = 0; j < RPT; j++){
        if(!(mask >> j & 1)) continue;
        const long i = t0 + j, il = i - L.child0;
        const long c = il >> a.D;
        const signed char *p = L.cells + c*SQB_MAXD;
        const unsigned char s = a.stt[i];
        const double av = fabs(a.v[i]);
        const int te = (p[SQB_PFLAG] >> 1) & 3, tv = (av >= thr10) + (av >= thr100);
        const int psk = (s & SQB_SKIPPED) ? 1 : 0, nr = (s & SQB_NEAR) ? 1 : 0;
        const signed char fl = (signed char)((a.abskip && (psk || !nr)) | ((te < tv ? te : tv) << 1));
        int k[SQB_MAXD];
        child_of(a, L, il, k);
        /* the child, then (under a fold) the other members of its orbit in group order, each once
         * (symorbit(), driver/sum.c:38-46), all with the child's flags (driver/sum.c:741-744) */
        const int ng = a.sym.n > 1 ? a.sym.n : 1;
        for(int e = 0; e < ng; e++){
            if(!sqb_image_new(a.sym, k, a.D, e)) continue;
            if((long)o >= cap){ atomicAdd(overflow, 1ULL); o++; continue; }
            union { signed char k[SQB_MAXD]; int w[3]; } q;
            q.w[0] = q.w[1] = q.w[2] = 0;
            int im[SQB_MAXD];
            sqb_image(a.sym, k, a.D, e, im);
            for(int d = 0; d < a.D; d++) q.k[d] = (signed char)im[d];
            q.k[SQB_PFLAG] = fl;
            int *dst = (int*)(next + o);
            dst[0] = q.w[0]; dst[1] = q.w[1]; dst[2] = q.w[2];
            o++;
        }
    }
}

/* list mode: the children of one level batch to evaluate -- in the box, not left out by the predictor and,
 * under a fold, the minimum of their orbit (driver/sum.c:405-416) -- appended to sel as child index | orbit
 * weight << SQB_SEL_SHIFT, in no particular order (each child's value and status go to its own slot, and
 * the reduce kernel sums them in child order).  The other children get value 0 and no status; cw holds
 * every child's weight (0: not evaluated) for the reduce and scatter kernels. */
__global__ void __launch_bounds__(RT) sqb_k_select(const __grid_constant__ lvl_t a, int K, unsigned long long *sel,
                                                   unsigned long long *nsel, double *v, unsigned char *stt,
                                                   unsigned char *cw){
    const lvi_t L = lvl_inst(a, 0);
    const int lane = threadIdx.x & 31;
    for(long b0 = blockIdx.x*(long)RT; b0 < a.n; b0 += (long)gridDim.x*RT){     /* the same trips for a warp */
        const long i = b0 + threadIdx.x;
        int mw = 0;
        if(i < a.n){
            int k[SQB_MAXD]; bool in = true;
            child_of(a, L, i, k);
            for(int d = 0; d < a.D; d++) in = in && k[d] >= -K;
            if(in && !(a.cfl && (a.cfl[i] & 1))) mw = a.sym.n > 1 ? sqb_orbit_n(a.sym, k, a.D) : 1;
            cw[i] = (unsigned char)mw;
            if(!mw){ v[i] = 0; stt[i] = 0; }
        }
        const unsigned m = __ballot_sync(0xffffffffu, mw > 0);
        unsigned long long base = 0;
        if(lane == 0 && m) base = atomicAdd(nsel, (unsigned long long)__popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if(mw > 0) sel[base + __popc(m & ((1u << lane) - 1))] = (unsigned long long)i | ((unsigned long long)mw << SQB_SEL_SHIFT);
    }
}

extern "C" int sqb_dev_level(const sqb_level_t *L, sqb_acc_t *acc, long *next_n, double *ms){
    const sqb_graph_t *g = L->g; const int D = g->D;
    long maxch = L->max_children > 0 ? L->max_children : (1L << 25);
    if(maxch < (1L << D)) maxch = 1L << D;
    long ncb = maxch >> D;
    /* full batches hold whole rounds of tiles: the FP64 kernel's cap resident CTAs take tiles b, b + cap,
     * ..., so with a multiple of cap tiles every CTA takes the same number and none idles while others
     * finish one more */
    {
        int can0 = 0;
        const long cap0 = grid_cap(g, f64_which(g, L->t.fma) | SQB_ATTR_LEVEL, 2*(2*G.K + 1)*sizeof(double), &can0);
        const long round = (cap0*SQB_TILE) >> D;            /* cells per round (SQB_TILE >= 2^D) */
        if(!L->t.alldd && can0 && round > 0 && ncb >= 2*round) ncb = (ncb/round)*round;
    }
    if(reserve_points(ncb << D)) return -1;
    /* the predictor runs at the last level when its table holds values (driver/sum.c:385) */
    bool pon = false;
    if(L->last && L->predict > 0 && L->vt && L->vt->tab){
        long vn = 0, full = 0;
        if(sqb_vtab_counts(L->vt, &vn, &full, G.s)){ snprintf(g_err, sizeof g_err, "%s", sqb_vtab_error()); return -1; }
        pon = vn > 0;
    }
    CKR(cudaMemsetAsync(G.acc, 0, sizeof(sqb_acc_t), G.s));
    CKR(cudaEventRecord(G.e0, G.s));
    for(long c0 = 0; c0 < L->ncell; c0 += ncb){
        const long nc = L->ncell - c0 < ncb ? L->ncell - c0 : ncb, nch = nc << D;
        const sqb_pt_t *cells = L->cells + c0;
        sqb_eval_t a; memset(&a, 0, sizeof a); fill_eval(&a, &L->t);
        a.pts = cells; a.n = nc; a.esize = 1; a.stride = SQB_MAXD; a.flag_at = SQB_PFLAG; a.cells = 1; a.st = L->st;
        if(L->sym && L->sym->n > 1){
            bool ok = L->sym->n <= SQB_SYMG;
            for(int e = 0; ok && e < L->sym->n; e++) for(int i = 0; i < D; i++) ok = ok && L->sym->g[e][i] >= 0 && L->sym->g[e][i] < D;
            if(!ok){ snprintf(g_err, sizeof g_err, "symmetry group: %d elements or an axis outside 0..%d", L->sym->n, D - 1); return -1; }
            a.sym = *L->sym;
        }
        /* level mode: the FP64 pass sums the tiles without fallback points (the all-dd form has no FP64
         * pass: the reduce kernel sums every tile) */
        /* the FP64 pass as a persistent grid taking tiles from the device queue (one integral: ninst = 1);
         * under a fold or the predictor it walks the list of children to evaluate (list mode), and the
         * reduce kernel sums every tile */
        const bool queue = !L->t.alldd && !use_split(g, &a, &L->t);
        /* list mode pays where the orbit test is costly or many children are left out: a group of order
         * 4 or more, or the predictor (measured on four-loop VP integrals: order 8, 1.5x faster; order 2,
         * 16 % slower than testing in place) */
        const bool listm = queue && (a.sym.n >= 4 || pon);
        /* the kernel that runs: the level kernel for a queue batch outside list mode */
        int can = 0;
        const long cap = grid_cap(g, f64_which(g, L->t.fma) | (queue && !listm ? SQB_ATTR_LEVEL : 0),
                                  2*(2*G.K + 1)*sizeof(double), &can);
        const bool fused = tile_sums() && !L->t.alldd && can && !use_split(g, &a, &L->t) && !listm && nch >= 2*SQB_TILE*cap;
        /* the predictor at the last level: which children to leave out, and their tiers */
        if(pon){
            if(sqb_vtab_predict(L->vt, cells, nc, D, L->st, G.K, L->thr, L->predict, L->esok, L->sym, G.cfl,
                                &G.acc->pskip, G.nsm, G.s)){ snprintf(g_err, sizeof g_err, "%s", sqb_vtab_error()); return -1; }
            G.launches++;
            a.cfl = G.cfl;
        }
        if(fused){ a.part = G.bp; a.tkeep = G.bkeep; a.tfb = G.tfb; a.pw = L->pw; a.thr = L->thr; a.last = L->last; }
        if(queue){
            a.part = G.bp; a.tkeep = G.bkeep; a.tfb = G.tfb;     /* every tile summed or flagged for the reduce */
            a.ninst = 1; a.ntile = (nch + SQB_TILE - 1)/SQB_TILE; a.queue = G.queue;
            sqb_inst_t &I = a.inst[0];
            I.pts = cells; I.n = nc; I.child0 = 0; I.st = L->st; I.K = G.K; I.toff = 0; I.fused = fused;
            I.last = L->last; I.pw = L->pw; I.thr = L->thr; I.abserr = L->t.abserr; I.near_thr = L->t.nearf*L->t.abserr;
            I.X = G.X; I.Wt = G.Wt;
        }
        lvl_t r; memset(&r, 0, sizeof r);
        r.cells = (const signed char*)cells; r.n = nch; r.D = D; r.st = L->st; r.last = L->last;
        r.abskip = L->t.abskip; r.pw = L->pw; r.thr = L->thr; r.v = G.v; r.uu = G.uu; r.stt = G.stt;
        r.sym = a.sym; r.cfl = a.cfl;
        const long nb = (nch + RTILE - 1)/RTILE;
        if(listm){
            CKR(cudaMemsetAsync(G.nsel, 0, sizeof(unsigned long long), G.s));
            CKR(cudaMemsetAsync(G.tfb, 1, nb, G.s));
            const long want = (nch + RT - 1)/RT, full = (long)G.nsm*8;
            sqb_k_select<<<(unsigned)(want < full ? want : full), RT, 0, G.s>>>(r, G.K, G.sel, G.nsel, G.v, G.stt, G.cw);
            CKR(cudaGetLastError());
            G.launches++;
            a.sel = G.sel; a.nsel = G.nsel;
            r.cw = G.cw;
        }
        if(eval_batch(g, &a, &L->t, nch)) return -1;
        /* the level before the last stores its values for the predictor */
        if(L->vput && L->vt){
            if(sqb_vtab_put_children(L->vt, cells, nch, D, L->st, G.v, G.stt, L->sym, G.s)){
                snprintf(g_err, sizeof g_err, "%s", sqb_vtab_error()); return -1; }
            G.launches++;
        }
        sqb_k_reduce<<<(unsigned)nb, RT, 0, G.s>>>(r, G.bp, G.bkeep, fused || queue ? G.tfb : NULL);
        CKR(cudaGetLastError());
        sqb_k_finish<<<1, FT, 0, G.s>>>(r, G.bp, G.bkeep, nb, G.boff, G.acc, G.base);
        CKR(cudaGetLastError());
        G.launches += 2;
        if(!L->last){
            sqb_k_scatter<<<(unsigned)nb, RT, 0, G.s>>>(r, G.boff, G.base, L->next, L->next_cap, &G.acc->overflow);
            CKR(cudaGetLastError());
            G.launches++;
        }
    }
    CKR(cudaEventRecord(G.e1, G.s));
    sqb_acc_t h;
    CKR(cudaMemcpyAsync(&h, G.acc, sizeof h, cudaMemcpyDeviceToHost, G.s));
    CKR(cudaStreamSynchronize(G.s));
    D2H += sizeof h;
    float t = 0; cudaEventElapsedTime(&t, G.e0, G.e1); if(ms) *ms = t;
    double *src[6] = {h.S, h.A, h.drop, h.b1, h.b2, h.u}, *dst[6] = {acc->S, acc->A, acc->drop, acc->b1, acc->b2, acc->u};
    for(int q = 0; q < 6; q++){ sqdd x = sqdd(dst[q][0], dst[q][1]) + sqdd(src[q][0], src[q][1]); dst[q][0] = x.hi; dst[q][1] = x.lo; }
    acc->ne += h.ne; acc->nq += h.nq; acc->unres += h.unres; acc->skipped += h.skipped; acc->keep += h.keep; acc->overflow += h.overflow;
    acc->pskip += h.pskip;
    *next_n = (long)h.keep;
    return 0;
}

/* A level of several integrals of one graph at once (see sqb_rt.h).  Each integral keeps the batches,
 * tiles and fused/unfused choice that sqb_dev_level would give it alone; round r launches batch r of every
 * integral that has one, its children numbered integral after integral from tile boundaries. */
extern "C" int sqb_dev_level_multi(const sqb_level_t *Ls, int n, sqb_acc_t *accs, long *next_n, double *ms){
    if(n <= 0) return 0;
    bool one_by_one = n == 1 || n > SQB_MAXINST;
    const sqb_graph_t *g = Ls[0].g; const int D = g->D;
    for(int k = 0; k < n && !one_by_one; k++){
        const sqb_level_t &L = Ls[k];
        one_by_one = L.g != g || L.t.alldd || L.t.split || L.predict > 0 || L.vput || L.st != Ls[0].st ||
                     L.last != Ls[0].last || !L.X || !L.Wt || L.K < 1 || L.K > 127 || L.t.fma != Ls[0].t.fma ||
                     L.t.split != Ls[0].t.split || L.t.abskip != Ls[0].t.abskip || L.t.abcheck != Ls[0].t.abcheck ||
                     L.t.dropunres != Ls[0].t.dropunres || L.t.ddslack != Ls[0].t.ddslack ||
                     ((L.sym && L.sym->n > 1) != (Ls[0].sym && Ls[0].sym->n > 1)) ||
                     (L.sym && Ls[0].sym && L.sym->n > 1 && memcmp(L.sym, Ls[0].sym, sizeof(sqb_sym_t)));
    }
    if(one_by_one){
        /* each integral on its own tables: the thread's current ones are lent the integral's device copy */
        double tot = 0; int rc = 0;
        double *sx = G.X, *sw = G.Wt; const int sk = G.K;
        for(int k = 0; k < n && !rc; k++){
            if(Ls[k].X){ G.X = (double*)Ls[k].X; G.Wt = (double*)Ls[k].Wt; G.K = Ls[k].K; }
            double m = 0;
            rc = sqb_dev_level(&Ls[k], &accs[k], &next_n[k], &m);
            tot += m;
            G.X = sx; G.Wt = sw; G.K = sk;
        }
        if(ms) *ms = tot;
        return rc;
    }
    const sqb_level_t &L0 = Ls[0];
    if(L0.sym && L0.sym->n > 1){
        bool ok = L0.sym->n <= SQB_SYMG;
        for(int e = 0; ok && e < L0.sym->n; e++) for(int i = 0; i < D; i++) ok = ok && L0.sym->g[e][i] >= 0 && L0.sym->g[e][i] < D;
        if(!ok){ snprintf(g_err, sizeof g_err, "symmetry group: %d elements or an axis outside 0..%d", L0.sym->n, D - 1); return -1; }
    }
    /* per integral: cells per batch and the number of batches, as sqb_dev_level chooses them */
    long ncb[SQB_MAXINST], nbat[SQB_MAXINST], capk[SQB_MAXINST]; int cank[SQB_MAXINST]; long rounds = 0;
    const int which = f64_which(g, L0.t.fma);
    for(int k = 0; k < n; k++){
        const sqb_level_t &L = Ls[k];
        long maxch = L.max_children > 0 ? L.max_children : (1L << 25);
        if(maxch < (1L << D)) maxch = 1L << D;
        long c = maxch >> D;
        const size_t sm1 = 2*(2*(size_t)L.K + 1)*sizeof(double);
        int can0 = 0;
        const long cap0 = grid_cap(g, which | SQB_ATTR_LEVEL, sm1, &can0);
        const long round = (cap0*SQB_TILE) >> D;
        if(can0 && round > 0 && c >= 2*round) c = (c/round)*round;
        ncb[k] = c; capk[k] = cap0; cank[k] = can0;
        nbat[k] = (L.ncell + c - 1)/c;
        if(nbat[k] > rounds) rounds = nbat[k];
    }
    /* the largest round's children, each integral's batch from a tile boundary */
    long maxtot = 0;
    for(long r = 0; r < rounds; r++){
        long tot = 0;
        for(int k = 0; k < n; k++) if(r < nbat[k]){
            const long nc = Ls[k].ncell - r*ncb[k] < ncb[k] ? Ls[k].ncell - r*ncb[k] : ncb[k];
            tot += ((nc << D) + SQB_TILE - 1)/SQB_TILE*SQB_TILE;
        }
        if(tot > maxtot) maxtot = tot;
    }
    if(reserve_points(maxtot)) return -1;
    CKR(cudaMemsetAsync(G.accm, 0, n*sizeof(sqb_acc_t), G.s));
    CKR(cudaEventRecord(G.e0, G.s));
    for(long r = 0; r < rounds; r++){
        sqb_eval_t a; memset(&a, 0, sizeof a); fill_eval(&a, &L0.t);
        a.esize = 1; a.stride = SQB_MAXD; a.flag_at = SQB_PFLAG; a.cells = 1;
        if(L0.sym && L0.sym->n > 1) a.sym = *L0.sym;
        a.part = G.bp; a.tkeep = G.bkeep; a.tfb = G.tfb; a.queue = G.queue;
        lvl_t rl; memset(&rl, 0, sizeof rl);
        rl.D = D; rl.abskip = L0.t.abskip; rl.v = G.v; rl.uu = G.uu; rl.stt = G.stt; rl.sym = a.sym;
        long child0 = 0; int m = 0, toff = 0, last = 0, kof[SQB_MAXINST];
        for(int k = 0; k < n; k++){
            if(r >= nbat[k]) continue;
            const sqb_level_t &L = Ls[k];
            const long c0 = r*ncb[k], nc = L.ncell - c0 < ncb[k] ? L.ncell - c0 : ncb[k], nch = nc << D;
            sqb_inst_t &I = a.inst[m];
            I.pts = L.cells + c0; I.n = nc; I.child0 = child0; I.st = L.st; I.K = L.K; I.toff = toff;
            I.fused = tile_sums() && cank[k] && nch >= 2*SQB_TILE*capk[k];
            I.last = L.last; I.pw = L.pw; I.thr = L.thr; I.abserr = L.t.abserr; I.near_thr = L.t.nearf*L.t.abserr;
            I.X = L.X; I.Wt = L.Wt;
            lvi_t &V = rl.inst[m];
            V.cells = (const signed char*)(L.cells + c0); V.n = nch; V.child0 = child0; V.st = L.st; V.last = L.last;
            V.pw = L.pw; V.thr = L.thr; V.next = L.next; V.cap = L.next_cap; V.acc = G.accm + k; V.base = G.basem + k;
            last = L.last; kof[m] = k;
            toff += 2*(2*L.K + 1);
            child0 += (nch + SQB_TILE - 1)/SQB_TILE*SQB_TILE;
            m++;
        }
        (void)kof;
        a.ninst = m; a.ntile = child0/SQB_TILE; rl.ninst = m;
        /* the per-point thresholds of the first integral stand in the launch's own fields (unused by the
         * kernels in a multi-instance launch) */
        if(eval_batch(g, &a, &Ls[0].t, child0)) return -1;
        sqb_k_reduce<<<(unsigned)a.ntile, RT, 0, G.s>>>(rl, G.bp, G.bkeep, G.tfb);
        CKR(cudaGetLastError());
        sqb_k_finish<<<(unsigned)m, FT, 0, G.s>>>(rl, G.bp, G.bkeep, 0, G.boff, NULL, NULL);
        CKR(cudaGetLastError());
        G.launches += 2;
        if(!last){
            sqb_k_scatter<<<(unsigned)a.ntile, RT, 0, G.s>>>(rl, G.boff, NULL, NULL, 0, NULL);
            CKR(cudaGetLastError());
            G.launches++;
        }
    }
    CKR(cudaEventRecord(G.e1, G.s));
    sqb_acc_t h[SQB_MAXINST];
    CKR(cudaMemcpyAsync(h, G.accm, n*sizeof(sqb_acc_t), cudaMemcpyDeviceToHost, G.s));
    CKR(cudaStreamSynchronize(G.s));
    D2H += n*sizeof(sqb_acc_t);
    float t = 0; cudaEventElapsedTime(&t, G.e0, G.e1); if(ms) *ms = t;
    for(int k = 0; k < n; k++){
        sqb_acc_t *acc = &accs[k];
        double *src[6] = {h[k].S, h[k].A, h[k].drop, h[k].b1, h[k].b2, h[k].u}, *dst[6] = {acc->S, acc->A, acc->drop, acc->b1, acc->b2, acc->u};
        for(int q = 0; q < 6; q++){ sqdd x = sqdd(dst[q][0], dst[q][1]) + sqdd(src[q][0], src[q][1]); dst[q][0] = x.hi; dst[q][1] = x.lo; }
        acc->ne += h[k].ne; acc->nq += h[k].nq; acc->unres += h[k].unres; acc->skipped += h[k].skipped;
        acc->keep += h[k].keep; acc->overflow += h[k].overflow; acc->pskip += h[k].pskip;
        next_n[k] = (long)h[k].keep;
    }
    return 0;
}

extern "C" void *sqb_dev_alloc(size_t bytes){ void *p = NULL; if(cudaMallocAsync(&p, bytes ? bytes : 16, G.s) != cudaSuccess){ cudaGetLastError(); return NULL; } return p; }
extern "C" void sqb_dev_free(void *p){ if(p) cudaFreeAsync(p, G.s); }
extern "C" int sqb_dev_upload(void *dst, const void *src, size_t bytes){
    CKR(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, G.s)); CKR(cudaStreamSynchronize(G.s)); H2D += bytes; return 0; }
extern "C" int sqb_dev_download(void *dst, const void *src, size_t bytes){
    CKR(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, G.s)); CKR(cudaStreamSynchronize(G.s)); D2H += bytes; return 0; }
extern "C" void sqb_dev_count_copy(unsigned long long h2d, unsigned long long d2h){ H2D += h2d; D2H += d2h; }

/* measurement helpers: bytes copied between host and device so far; events on the library's stream
 * around a region of work (device milliseconds); an L2 flush (a memset larger than L2) on that stream */
extern "C" void sqb_copy_bytes(unsigned long long *h2d, unsigned long long *d2h){ *h2d = H2D.load(); *d2h = D2H.load(); }
extern "C" int sqb_timer_start(void){ if(sqb_dev_init(0)) return -1; CKR(cudaEventRecord(G.t0, G.s)); return 0; }
extern "C" double sqb_timer_stop(void){
    if(cudaEventRecord(G.t1, G.s) != cudaSuccess || cudaEventSynchronize(G.t1) != cudaSuccess) return -1;
    float t = 0; cudaEventElapsedTime(&t, G.t0, G.t1); return t;
}
extern "C" int sqb_l2_flush(size_t bytes){
    if(sqb_dev_init(0)) return -1;
    if(bytes > G.flushn){ if(G.flush) cudaFree(G.flush); G.flush = NULL; CKR(cudaMalloc(&G.flush, bytes)); G.flushn = bytes; }
    CKR(cudaMemsetAsync(G.flush, G.launches & 255, bytes, G.s));
    return 0;
}
extern "C" size_t sqb_dev_free_bytes(void){ size_t f = 0, t = 0; cudaMemGetInfo(&f, &t); return f; }
extern "C" size_t sqb_dev_total_bytes(void){ size_t f = 0, t = 0; cudaMemGetInfo(&f, &t); return t; }

/* ------------------------------ plain form: the reference's GPU plug-in ABI ---------------------- */
/* Same contract as driver/gpu.cu:1-103: two slots, each with its own stream, event and pinned buffers;
 * gpu_submit* pack the coordinates (here to int8: |k| <= 127, driver/sq.h:117), copy, launch and copy
 * back f*w and |.|*w; gpu_wait waits for the slot.  SINCQED_GPU=0 turns the GPU off, SINCQED_GPU=d
 * picks device d-1.  CUDA errors print and exit(3), as the reference does. */
#define CKX(x) do { cudaError_t e_ = (x); if(e_ != cudaSuccess){ fprintf(stderr, "CUDA error %s at %s:%d: %s\n", #x, __FILE__, __LINE__, cudaGetErrorString(e_)); exit(3); } } while(0)

typedef struct { cudaStream_t st; cudaEvent_t ev; long cap, n; signed char *hK, *dK; unsigned char *hS, *dS; double *hF, *hA, *dF, *dA; } pslot_t;
static pslot_t PS[2];
static int PON = -1, PD, PK; static double PH;
static const sqb_graph_t *PCUR;
static double *PEX; static int PEXN;

static int plain_init(void){
    if(PON >= 0) return PON;
    const char *e = getenv("SINCQED_GPU"); PON = 0;
    if(e && !strcmp(e, "0")) return 0;
    int nd = 0; if(cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0){ cudaGetLastError(); return 0; }
    int dev = e && atoi(e) > 0 ? atoi(e) - 1 : 0; if(dev >= nd) dev = 0;
    if(sqb_dev_init(dev)){ fprintf(stderr, "gpu: %s\n", g_err); exit(3); }
    for(int b = 0; b < 2; b++){ CKX(cudaStreamCreateWithFlags(&PS[b].st, cudaStreamNonBlocking)); CKX(cudaEventCreateWithFlags(&PS[b].ev, cudaEventDisableTiming)); }
    return PON = 1;
}
static void plain_reserve(pslot_t *s, long n){
    if(n <= s->cap) return;
    if(s->cap){ cudaFreeHost(s->hK); cudaFree(s->dK); cudaFreeHost(s->hS); cudaFree(s->dS); cudaFreeHost(s->hF); cudaFree(s->dF); cudaFreeHost(s->hA); cudaFree(s->dA); }
    long c = 1L << 16; while(c < n) c <<= 1; s->cap = c;
    CKX(cudaMallocHost(&s->hK, c*SQB_MAXD)); CKX(cudaMalloc(&s->dK, c*SQB_MAXD));
    CKX(cudaMallocHost(&s->hS, c)); CKX(cudaMalloc(&s->dS, c));
    CKX(cudaMallocHost(&s->hF, c*sizeof(double))); CKX(cudaMalloc(&s->dF, c*sizeof(double)));
    CKX(cudaMallocHost(&s->hA, c*sizeof(double))); CKX(cudaMalloc(&s->dA, c*sizeof(double)));
}

extern "C" const char *gpu_info(void){ return PON == 1 ? G.info : "off"; }

extern "C" int gpu_setup(const char *name, int D, const double *EX, int K, double H){
    PCUR = NULL;
    if(!plain_init()) return 0;
    const sqb_graph_t *g = sqb_find_graph(name);
    if(!g || strcmp(g->name, name)) return 0;
    if(g->D != D){ fprintf(stderr, "gpu: %s has D=%d, expected %d\n", name, g->D, D); exit(3); }
    PCUR = g; PD = D; PK = K; PH = H;
    CKX(cudaDeviceSynchronize());
    if(PEXN < 2*K + 1){ if(PEX) CKX(cudaFree(PEX)); PEXN = 2*K + 1; CKX(cudaMalloc(&PEX, PEXN*sizeof(double))); }
    CKX(cudaMemcpy(PEX, EX, (2*K + 1)*sizeof(double), cudaMemcpyHostToDevice));
    return 1;
}

static void plain_launch(pslot_t *s, long npts, long nrows, int cells, int st, int has_skip){
    sqb_eval_t a; memset(&a, 0, sizeof a);
    a.pts = s->dK; a.n = nrows; a.esize = 1; a.stride = PD; a.flag_at = -1; a.cells = cells; a.st = st;
    a.X = PEX; a.Wt = NULL; a.K = PK; a.H = PH; a.raw = 1; a.skip = has_skip ? s->dS : NULL;
    a.v = s->dF; a.ab = s->dA;
    size_t smem = 2*(2*PK + 1)*sizeof(double);
    PCUR->f64(&a, grid_for(PCUR, 0, npts, smem), 128, smem, s->st);
    CKX(cudaGetLastError());
}

extern "C" void gpu_submit(int slot, long n, const int *k, int stride, const unsigned char *skip){
    pslot_t *s = &PS[slot]; plain_reserve(s, n); s->n = n;
    if(n <= 0) return;
    signed char *hk = s->hK; const int D = PD;
    #pragma omp parallel for schedule(static)
    for(long i = 0; i < n; i++) for(int d = 0; d < D; d++) hk[i*D + d] = (signed char)k[i*stride + d];
    CKX(cudaMemcpyAsync(s->dK, hk, n*D, cudaMemcpyHostToDevice, s->st));
    if(skip){ memcpy(s->hS, skip, n); CKX(cudaMemcpyAsync(s->dS, s->hS, n, cudaMemcpyHostToDevice, s->st)); }
    plain_launch(s, n, n, 0, 0, skip != NULL);
    CKX(cudaMemcpyAsync(s->hF, s->dF, n*sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CKX(cudaMemcpyAsync(s->hA, s->dA, n*sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CKX(cudaEventRecord(s->ev, s->st));
}

extern "C" void gpu_submit_cells(int slot, long nc, const int *cells, int stride, const unsigned char *skip, int st){
    pslot_t *s = &PS[slot]; const long n = nc << PD; plain_reserve(s, n); s->n = n;
    if(nc <= 0) return;
    signed char *hk = s->hK; const int D = PD;
    #pragma omp parallel for schedule(static)
    for(long c = 0; c < nc; c++) for(int d = 0; d < D; d++) hk[c*D + d] = (signed char)cells[c*stride + d];
    CKX(cudaMemcpyAsync(s->dK, hk, nc*D, cudaMemcpyHostToDevice, s->st));
    if(skip){ memcpy(s->hS, skip, nc); CKX(cudaMemcpyAsync(s->dS, s->hS, nc, cudaMemcpyHostToDevice, s->st)); }
    plain_launch(s, n, nc, 1, st, skip != NULL);
    CKX(cudaMemcpyAsync(s->hF, s->dF, n*sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CKX(cudaMemcpyAsync(s->hA, s->dA, n*sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CKX(cudaEventRecord(s->ev, s->st));
}

extern "C" void gpu_wait(int slot, const double **fw, const double **abw){
    pslot_t *s = &PS[slot];
    if(s->n > 0) CKX(cudaEventSynchronize(s->ev));
    *fw = s->hF; *abw = s->hA;
}

/* the reference's per-graph launcher (sq_gpu_launch_t, driver/gpu.h:18-19) on device buffers: int16
 * coordinates, stride D, n points (cells: n = nc << D) */
extern "C" void sqb_gg_launch(const sqb_graph_t *g, void *st, long n, const short *k, const unsigned char *skip,
                              const double *EX, int K, double H, double *of, double *oab, int cmode, int cst){
    if(n <= 0) return;
    if(!G.on && sqb_dev_init(0)){ fprintf(stderr, "gpu: %s\n", g_err); exit(3); }
    sqb_eval_t a; memset(&a, 0, sizeof a);
    a.pts = k; a.n = cmode ? (n >> g->D) : n; a.esize = 2; a.stride = g->D; a.flag_at = -1; a.cells = cmode; a.st = cst;
    a.X = EX; a.Wt = NULL; a.K = K; a.H = H; a.raw = 1; a.skip = skip; a.v = of; a.ab = oab;
    size_t smem = 2*(2*K + 1)*sizeof(double);
    g->f64(&a, grid_for(g, 0, n, smem), 128, smem, st);
}

/* GG_<graph>'s launcher with the FP64 build chosen (0 as written, 2 contracted) */
extern "C" int sqb_plugin_launch(const char *graph, int form, cudaStream_t st, long n, const short *k, const unsigned char *skip,
                                 const double *EX, int K, double H, double *of, double *oab, int cmode, int cst){
    const sqb_graph_t *g = sqb_find_graph(graph);
    if(!g || (form != 0 && form != 2) || (form == 2 && !g->f64_fma) || K < 0 || K > 127){
        snprintf(g_err, sizeof g_err, "sqb_plugin_launch: no graph %s with FP64 build %d (or K %d outside 0..127)", graph, form, K);
        sqb_set_error_msg(g_err);
        return -1;
    }
    if(n <= 0) return 0;
    if(sqb_dev_init(0)){ sqb_set_error_msg(g_err); return -1; }
    sqb_eval_t a; memset(&a, 0, sizeof a);
    a.pts = k; a.n = cmode ? (n >> g->D) : n; a.esize = 2; a.stride = g->D; a.flag_at = -1; a.cells = cmode; a.st = cst;
    a.X = EX; a.Wt = NULL; a.K = K; a.H = H; a.raw = 1; a.skip = skip; a.v = of; a.ab = oab;
    const size_t smem = 2*(2*K + 1)*sizeof(double);
    launch_f64(g, form, &a, grid_for(g, form, n, smem), smem, st);
    const cudaError_t e = cudaGetLastError();
    if(e != cudaSuccess){
        snprintf(g_err, sizeof g_err, "sqb_plugin_launch: %s", cudaGetErrorString(e)); sqb_set_error_msg(g_err); return (int)e; }
    G.launches++;
    return 0;
}

/* pointwise evaluation (parity checks): n points given by their variables, FP64 (SQ_AB = ab) or
 * double-double; f, abs_ hold n values (FP64) or n (hi, lo) pairs (double-double) */
extern "C" int sqb_eval_points_impl(const sqb_graph_t *g, long n, const double *sf, int prec, int ab, double *f, double *abs_){
    if(n <= 0) return 0;
    const int D = g->D;
    /* one stream-ordered block (no device-wide synchronisation, so other threads' work runs on):
     * sf[n D], v, ab, vlo, ablo [n each], X = 1, skip[n] */
    const size_t nd = (size_t)n*D + 4*(size_t)n + 1;
    char *blk = NULL;
    CKR(cudaMallocAsync((void**)&blk, nd*sizeof(double) + (size_t)n, G.s));
    double *dsf = (double*)blk, *dv = dsf + (size_t)n*D, *dab = dv + n, *dvl = dab + n, *dabl = dvl + n, *dX = dabl + n;
    unsigned char *dsk = (unsigned char*)(dX + 1);
    const double one = 1.0;
    CKR(cudaMemcpyAsync(dsf, sf, (size_t)n*D*sizeof(double), cudaMemcpyHostToDevice, G.s));
    CKR(cudaMemcpyAsync(dX, &one, sizeof one, cudaMemcpyHostToDevice, G.s));
    CKR(cudaMemsetAsync(dsk, ab ? 0 : 1, n, G.s));
    sqb_eval_t a; memset(&a, 0, sizeof a);
    a.pts = NULL; a.n = n; a.esize = 1; a.stride = D; a.flag_at = -1; a.cells = 0;
    a.X = dX; a.Wt = dX; a.K = 0; a.raw = 1; a.skip = dsk; a.v = dv; a.ab = dab; a.sfin = dsf; a.vlo = dvl; a.ablo = dabl;
    size_t smem = 2*sizeof(double);
    int rc = 0;
    if(prec == 0 || prec == 2){
        const int w = f64_which(g, prec == 2);
        if(prec == 2 && w != 2){ snprintf(g_err, sizeof g_err, "%s: no contracted FP64 kernel in this library", g->name); rc = -1; }
        else launch_f64(g, w, &a, grid_for(g, w, n, smem), smem, G.s);
    } else { sqb_dd_t d; memset(&d, 0, sizeof d); d.e = a; d.all = 1; d.uu = dvl; g->dd(&d, grid_for(g, 1, n, smem), 128, smem, G.s); }
    if(!rc){
        CKR(cudaGetLastError());
        if(prec == 0 || prec == 2){
            CKR(cudaMemcpyAsync(f, dv, n*sizeof(double), cudaMemcpyDeviceToHost, G.s));
            CKR(cudaMemcpyAsync(abs_, dab, n*sizeof(double), cudaMemcpyDeviceToHost, G.s));
            CKR(cudaStreamSynchronize(G.s));
        } else {
            std::vector<double> h(4*(size_t)n);
            CKR(cudaMemcpyAsync(h.data(), dv, 4*n*sizeof(double), cudaMemcpyDeviceToHost, G.s));   /* v, ab, vlo, ablo */
            CKR(cudaStreamSynchronize(G.s));
            for(long i = 0; i < n; i++){ f[2*i] = h[i]; f[2*i + 1] = h[2*n + i]; abs_[2*i] = h[n + i]; abs_[2*i + 1] = h[3*n + i]; }
        }
    }
    cudaFreeAsync(blk, G.s);
    return rc;
}

/* the scaling test's device part: a->g[3 ndir] for the directions of a, with the factor table xs
 * (3 x (2E+1), host); the values come back to g_host.  Returns 0, 1 if the graph has no raw point
 * function, or -1 */
extern "C" int sqb_dev_scale(const sqb_graph_t *g, sqb_scale_t *a, const double *xs, double *g_host){
    if(!g->scale) return 1;
    const size_t nxs = 3*(size_t)(2*a->E + 1), ng = 3*(size_t)a->ndir;
    double *blk = NULL;
    CKR(cudaMallocAsync((void**)&blk, (nxs + ng)*sizeof(double), G.s));
    a->xs = blk; a->g = blk + nxs;
    CKR(cudaMemcpyAsync(blk, xs, nxs*sizeof(double), cudaMemcpyHostToDevice, G.s));
    long want = ((long)ng + 127)/128, full = (long)G.nsm*4;
    g->scale(a, (int)(want < full ? want : full), 128, G.s);
    CKR(cudaGetLastError());
    G.launches++;
    CKR(cudaMemcpyAsync(g_host, a->g, ng*sizeof(double), cudaMemcpyDeviceToHost, G.s));
    CKR(cudaStreamSynchronize(G.s));
    cudaFreeAsync(blk, G.s);
    return 0;
}

/* FP64 peak probe: independent chains of fused multiply-adds (8 per thread, unrolled) or of adds, on
 * every SM; flops = 2 per FMA, 1 per add.  The measured rate is the denominator of the evaluation
 * kernels' roofline (the device has no vendor FP64 figure in this environment). */
template<int FMA>
__global__ void __launch_bounds__(256) sqb_k_fp64_probe(double *out, long iters, double a, double b){
    double x[8];
#pragma unroll
    for(int j = 0; j < 8; j++) x[j] = threadIdx.x*1e-9 + j;
    for(long i = 0; i < iters; i++){
#pragma unroll
        for(int j = 0; j < 8; j++) x[j] = FMA ? __fma_rn(x[j], a, b) : __dadd_rn(x[j], b);
    }
    double s = 0;
#pragma unroll
    for(int j = 0; j < 8; j++) s += x[j];
    if(s == 1.2345) out[0] = s;      /* keeps the chains alive */
}
/* returns the rate in TFLOP/s (fma = 1: FMA, 2 flops each; fma = 0: adds) */
extern "C" double sqb_probe_fp64(int fma, long iters){
    if(sqb_dev_init(0)) return -1;
    double *o; if(cudaMalloc(&o, sizeof(double)) != cudaSuccess) return -1;
    int per = 0;
    if(fma) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sqb_k_fp64_probe<1>, 256, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sqb_k_fp64_probe<0>, 256, 0);
    const int grid = G.nsm*(per > 0 ? per : 4);
    float best = 1e30f;
    for(int r = 0; r < 4; r++){
        cudaEventRecord(G.e0, G.s);
        if(fma) sqb_k_fp64_probe<1><<<grid, 256, 0, G.s>>>(o, iters, 0.999999, 1e-7);
        else sqb_k_fp64_probe<0><<<grid, 256, 0, G.s>>>(o, iters, 0.999999, 1e-7);
        cudaEventRecord(G.e1, G.s);
        cudaEventSynchronize(G.e1);
        float t = 0; cudaEventElapsedTime(&t, G.e0, G.e1);
        if(r && t < best) best = t;
    }
    cudaFree(o);
    const double ops = (double)grid*256*8*(double)iters*(fma ? 2 : 1);
    return ops/(best*1e-3)/1e12;
}

/* The reduce / finish / scatter sequence of one level batch on buffers the caller names (used by the
 * allocation-free entry point, noalloc.cu): v, uu, stt per child; bp, bkeep, boff per tile; acc and
 * base the accumulator and this batch's first kept slot. */
extern "C" int sqb_level_tail(const void *cells, long nchildren, int D, int st, int last, int abskip, double pw, double thr,
                              const double *v, const double *uu, const unsigned char *stt,
                              void *bp, unsigned *bkeep, unsigned long long *boff, sqb_acc_t *acc, unsigned long long *base,
                              void *next, long next_cap, void *stream){
    lvl_t r; memset(&r, 0, sizeof r);        /* no symmetry fold here (r.sym.n = 0) */
    r.cells = (const signed char*)cells; r.n = nchildren; r.D = D; r.st = st; r.last = last;
    r.abskip = abskip; r.pw = pw; r.thr = thr; r.v = v; r.uu = uu; r.stt = stt;
    const long nb = (nchildren + RTILE - 1)/RTILE;
    cudaStream_t s = (cudaStream_t)stream;
    sqb_k_reduce<<<(unsigned)nb, RT, 0, s>>>(r, (part_t*)bp, bkeep, NULL);
    CKR(cudaGetLastError());
    sqb_k_finish<<<1, FT, 0, s>>>(r, (const part_t*)bp, bkeep, nb, boff, acc, base);
    CKR(cudaGetLastError());
    if(!last){
        sqb_k_scatter<<<(unsigned)nb, RT, 0, s>>>(r, boff, base, (sqb_pt_t*)next, next_cap, &acc->overflow);
        CKR(cudaGetLastError());
    }
    return 0;
}
/* bytes of one tile partial (sizing of caller-provided tile buffers) and children per tile */
extern "C" size_t sqb_level_tile_bytes(void){ return sizeof(part_t); }
extern "C" long sqb_level_tile_children(void){ return RTILE; }
