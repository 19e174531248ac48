/* sqb_rt.h -- the runtime's internal interface between the device layer (runtime.cu) and the host
 * level engine (engine.cpp).  Not part of the public C ABI. */
#pragma once
#include <stddef.h>
#include "sqb_internal.h"
#ifdef __cplusplus
extern "C" {
#endif

#define SQB_MAXD 12                   /* pt_t: signed char k[12], flags in k[11] (driver/sq.h:52,108,116) */
#define SQB_PFLAG (SQB_MAXD - 1)
typedef struct { signed char k[SQB_MAXD]; } sqb_pt_t;

/* the per-point test parameters (driver/eval.c:7-24) */
typedef struct {
    double abserr, nearf, ddslack;
    int abskip, abcheck, dropunres;
    int alldd;                        /* every point in double-double (the plain all-dd form) */
    int fma;                          /* FP64 pass: the contracted kernel (fused multiply-adds) when present */
    int split;                        /* FP64 pass of a level batch in passes, for graphs that have them */
} sqb_test_t;

/* level accumulators, double-double (hi, lo) pairs */
typedef struct {
    double S[2], A[2], drop[2], b1[2], b2[2], u[2];
    unsigned long long ne, keep, nq, unres, skipped, overflow;
    unsigned long long pskip;           /* last level: children the predictor left out */
} sqb_acc_t;

/* the predictor's table of step-2h values (predict.cu): device slots, capacity (a power of two), and
 * two device counters (keys stored, inserts that found the table full) */
typedef struct {
    void *tab; long cap;
    unsigned long long *vn, *full;
} sqb_vtab_t;
int  sqb_vtab_reserve(sqb_vtab_t *t, long more, void *stream);
int  sqb_vtab_put_nodes(sqb_vtab_t *t, const sqb_pt_t *pts, const double *v, long n, int D, void *stream);
int  sqb_vtab_raise_kept(sqb_vtab_t *t, const sqb_pt_t *keep, long m, int D, int st, int K, void *stream);
int  sqb_vtab_put_children(sqb_vtab_t *t, const void *cells, long nch, int D, int st, const double *v,
                           const unsigned char *stt, const sqb_sym_t *sym, void *stream);
int  sqb_vtab_predict(const sqb_vtab_t *t, const void *cells, long ncell, int D, int st, int K, double thr,
                      double alpha, int esok, const sqb_sym_t *sym, unsigned char *cfl,
                      unsigned long long *pskip, int nsm, void *stream);
int  sqb_vtab_counts(const sqb_vtab_t *t, long *vn, long *full, void *stream);
int  sqb_vtab_download(const sqb_vtab_t *t, void *host, void *stream);
int  sqb_vtab_upload(sqb_vtab_t *t, const void *host, long cap, long vn, void *stream);
void sqb_vtab_free(sqb_vtab_t *t, void *stream);
const char *sqb_vtab_error(void);

const sqb_graph_t *sqb_find_graph(const char *name);
int  sqb_ngraphs(void);
const sqb_graph_t *sqb_graph_at(int i);

/* device state: 0 on success, else a CUDA error code (never exits the process) */
int  sqb_dev_init(int device);
const char *sqb_dev_info(void);
const char *sqb_last_error(void);
/* tables X[k+K], Wt[k+K] for the current graph (2K+1 entries each) */
int  sqb_dev_tables(const double *X, const double *Wt, int K);

/* n nodes (host pt_t list, flags ignored) evaluated with the tests and the fallback: values v, near
 * flags (may be NULL); skip (host, may be NULL) per node; counters added to *nq, *u, *unres */
int  sqb_dev_eval_nodes(const sqb_graph_t *g, long n, const sqb_pt_t *pts, const unsigned char *skip,
                        const sqb_test_t *t, double *v, unsigned char *near, long *nq, double *u, long *unres);

/* one refinement level on the device: the children (step st) of the ncell cells in the device list,
 * summed with weight pw; kept children (|v| >= thr, not last) appended to the device list next.
 * Accumulators are added into *acc.  Returns 0, or an error; *next_n is the length of next. */
typedef struct {
    const sqb_graph_t *g;
    const sqb_pt_t *cells; long ncell;  /* device */
    sqb_pt_t *next; long next_cap;      /* device */
    int st, last;
    double pw, thr;
    sqb_test_t t;
    long max_children;                  /* children per batch (0: default) */
    const sqb_sym_t *sym;               /* the symmetry fold (NULL or n <= 1: off) */
    /* the predictor: vput = store this level's values in vt (the level before the last); predict > 0 at
     * the last level = leave out the children whose predicted mean is below predict*thr (esok: and cap
     * their tiers) */
    sqb_vtab_t *vt; int vput; double predict; int esok;
    /* the integral's lattice tables on the device (2K+1 each), for sqb_dev_level_multi; sqb_dev_level uses
     * the thread's current tables (sqb_dev_tables) */
    const double *X, *Wt; int K;
} sqb_level_t;
int  sqb_dev_level(const sqb_level_t *L, sqb_acc_t *acc, long *next_n, double *ms);
/* the same level of n <= SQB_MAXINST integrals of one graph at once (each L[i] as for sqb_dev_level, with
 * its own tables, cells, lists and test thresholds): each launch of the FP64, double-double, reduce, finish
 * and scatter kernels covers batch b of every integral that has one, the FP64 and double-double kernels
 * taking tiles from a device queue.  Batches, tiles and summation order per integral are those of
 * sqb_dev_level, so every result is bit for bit the one sqb_dev_level gives.  Integrals with the predictor
 * or the pass split run one after another through sqb_dev_level. */
int  sqb_dev_level_multi(const sqb_level_t *L, int n, sqb_acc_t *acc, long *next_n, double *ms);

/* the same for n nodes already on the device (pts, skip device pointers); the values and status come
 * back to the host (v, stt) and stay on the device until the next evaluation (*v_dev, *stt_dev) */
int  sqb_dev_eval_resident(const sqb_graph_t *g, const sqb_pt_t *pts, long n, const unsigned char *skip,
                           const sqb_test_t *t, double *v, unsigned char *stt, long *nq, double *u, long *unres,
                           const double **v_dev, const unsigned char **stt_dev);
void *sqb_dev_stream(void);

/* the top level on the device (topgrid.cu): grow frontiers, final threshold, tiers, dilation */
int  sqb_grow_begin(int D, int K, int st, int W, const unsigned long long *P, int gs, int abskip, void *stream);
long sqb_grow_frontier(const sqb_pt_t **pts, const unsigned char **skip);
int  sqb_grow_shells_async(void);
void sqb_grow_shells_take(unsigned char *cls_host);
int  sqb_grow_expand(const double *v_dev, const unsigned char *stt_dev, double thr, long *nkept, long *nnext);
int  sqb_grow_kv(double *kv_host, long n);
int  sqb_grow_finish(double thr, int tiers, long *m);
int  sqb_grow_dilate(int nbits, sqb_pt_t **out, long *n);
void sqb_grow_kept(const sqb_pt_t **keep, long *m);
void sqb_grow_end(void);
const char *sqb_top_error(void);
int  sqb_radix_sort_u64(unsigned long long *keys_dev, long n, int nbits, void *stream);

/* the scaling test on the device (runtime.cu): 0, 1 = the graph has no raw point function, -1 */
int  sqb_dev_scale(const sqb_graph_t *g, sqb_scale_t *a, const double *xs, double *g_host);

/* instrumentation (runtime.cu, topgrid.cu) */
unsigned long long sqb_launch_count(void);
unsigned long long sqb_top_launches(void);
void sqb_kernel_timing(int on);
void sqb_kernel_times(double *f64_ms, double *dd_ms, long *f64_launches, int reset);

/* device memory for level lists */
void *sqb_dev_alloc(size_t bytes);
void  sqb_dev_free(void *p);
int   sqb_dev_upload(void *dst, const void *src, size_t bytes);
int   sqb_dev_download(void *dst, const void *src, size_t bytes);
size_t sqb_dev_free_bytes(void);
size_t sqb_dev_total_bytes(void);

#ifdef __cplusplus
}
#endif
