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
} sqb_test_t;

/* level accumulators, double-double (hi, lo) pairs */
typedef struct {
    double S[2], A[2], drop[2], b1[2], b2[2], u[2];
    unsigned long long ne, keep, nq, unres, skipped, overflow;
} sqb_acc_t;

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
} sqb_level_t;
int  sqb_dev_level(const sqb_level_t *L, sqb_acc_t *acc, long *next_n, double *ms);

/* device memory for level lists */
void *sqb_dev_alloc(size_t bytes);
void  sqb_dev_free(void *p);
int   sqb_dev_upload(void *dst, const void *src, size_t bytes);
int   sqb_dev_download(void *dst, const void *src, size_t bytes);
size_t sqb_dev_free_bytes(void);

#ifdef __cplusplus
}
#endif
