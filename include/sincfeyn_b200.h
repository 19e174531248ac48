/* sincfeyn_b200.h -- the C ABI of the B200 evaluator for sincFeyn's hierarchical Sinc sum.
 *
 * Two forms share one shared library, libsqb200.so:
 *
 * 1. The plain form: the reference's GPU plug-in ABI, unchanged (driver/gpu.h:12-22).  The reference
 *    driver built with -DSQ_GPU (driver/eval.c:97-203, driver/lattice.c:20-22) links against this library
 *    instead of its own driver/gpu.cu and evaluates every batch with this library's sm_100a kernels.
 *
 * 2. The chosen form: one call per integral, sqb_hsum(), which replaces the body of the reference's
 *    hsum() (driver/sum.c:556-814): the top level on the host, every refinement level resident on the
 *    device (FP64 bulk, double-double only for the points the reference's fallback test flags,
 *    double-double level sums), with the same results structure as res_t (driver/sq.h:111).
 *
 * All pointers are host pointers unless a comment says device.  No function here exits the process
 * except where the reference's plug-in contract does (CUDA errors and a D mismatch in the plain form,
 * driver/gpu.cu:16,59); the chosen form returns an error code and sqb_error() says why. */
#pragma once
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------------------------------
 * 1. Plain form: the reference's GPU plug-in (replaces driver/gpu.cu; declarations as driver/gpu.h)
 * ------------------------------------------------------------------------------------------------ */
#ifdef __CUDACC__
typedef cudaStream_t sq_stream_t;
#else
typedef void *sq_stream_t;
#endif
/* launcher of one graph's batch kernel on device buffers (driver/gpu.h:17-19) */
typedef void (*sq_gpu_launch_t)(sq_stream_t st, long n, const short *k, const unsigned char *skip,
                                const double *EX, int K, double H, double *of, double *oab, int cmode, int cst);
typedef struct { const char *name; int D; sq_gpu_launch_t launch; } sq_gpu_t;   /* driver/gpu.h:20 */
extern const sq_gpu_t *GPU_ALL[];            /* NULL-terminated, one GG_<name> per graph (Makefile:231-234) */

/* driver/gpu.h:23: 1 if this graph has a GPU kernel (then D must match, else exit(3)), 0 = CPU path */
int  gpu_setup(const char *name, int D, const double *EX, int K, double H);
/* driver/gpu.h:24: n nodes k[i*stride + d]; skip (may be NULL) per node; returns at once */
void gpu_submit(int slot, long n, const int *k, int stride, const unsigned char *skip);
/* driver/gpu.h:25: waits for the slot; fw = f*w, abw = sum|terms|*w, valid until the slot's next submit */
void gpu_wait(int slot, const double **fw, const double **abw);
/* driver/gpu.h:27: the 2^D children of nc cells at step st; nc << D results in prep() order */
void gpu_submit_cells(int slot, long nc, const int *cells, int stride, const unsigned char *skip, int st);
/* driver/gpu.h:28 */
const char *gpu_info(void);
/* The plug-in launcher of GG_<graph> (sq_gpu_launch_t, same arguments and device buffers) with the build
 * chosen: form 0 = the FP64 kernel rounded as written (what GG_<graph> runs), 2 = the contracted FP64
 * kernel (fused multiply-adds).  Not in the reference's ABI: it lets a caller, or a benchmark that times
 * the reference's own plug-in kernel, run either build on the same nodes.  0, or -1 (no such graph or
 * build; sqb_error() has the message) */
int  sqb_plugin_launch(const char *graph, int form, sq_stream_t st, long n, const short *k, const unsigned char *skip,
                       const double *EX, int K, double H, double *of, double *oab, int cmode, int cst);

/* ------------------------------------------------------------------------------------------------
 * 2. Chosen form
 * ------------------------------------------------------------------------------------------------ */
/* the run parameters that the reference reads from its environment (driver/main.c:176-185,
 * driver/eval.c:7-24); sqb_default_opts() gives the reference's defaults */
typedef struct {
    double abserr0;        /* G2_ABSERR: floor of the per-point fallback threshold (1e-15) */
    double abrel;          /* SINCQED_ABREL: ABSERR = max(abserr0, abrel*eps*Ref) in the levels (1e-3) */
    double nearf;          /* SINCQED_NEARF (1e-3) */
    double ddslack;        /* SINCQED_DDSLACK (1) */
    int abskip;            /* SINCQED_ABSKIP (1) */
    int abcheck;           /* SINCQED_ABCHECK (0) */
    int dropunres;         /* SINCQED_DROPUNRES (1) */
    int growskip;          /* SINCQED_GROWSKIP, top = 0 only (2) */
    int alldd;             /* 1: every point in double-double (the plain all-dd form); 0: FP64 + fallback */
    int device;            /* CUDA device (0) */
    long max_children;     /* children per device batch, 0 = default (2^25) */
    int verbose;           /* 1: timing lines on stderr */
    double ckpt_every;     /* SINCQED_CKPT: > 0 writes a checkpoint at the end of every refinement level but the
                              last and resumes from a matching one (driver/checkpoint.c:1-6); 0 = off (the
                              library's default; the CLI's is the reference's 600) */
    const char *ckpt_dir;  /* SINCQED_CKPT_DIR (NULL: the current directory) */
    int ckpt_stop;         /* test hook: 1 = return SQB_CKPT_STOPPED right after the first checkpoint is written,
                              as a run killed there would stop */
    int fma;               /* SQB_FMA: 1 (default) = the FP64 pass runs the graph's contracted kernel (multiplies
                              and adds fused, as the reference's own CPU build compiles its double half);
                              0 = the kernel that rounds every operation as written, bit for bit the reference's
                              double half built with -ffp-contract=off */
    int split;             /* SQB_SPLIT: 1 = a graph whose point function is a flat sum of independent forest
                              nodes (g3_lbl) runs the FP64 pass of its level batches as passes over groups of
                              nodes (the same operations in the same order: the same values); 0 (default) = one
                              pass, measured faster on the B200 */
    const char *sym;       /* SINCQED_SYM, the symmetry fold (driver/sum.c:21-26, 566-592): NULL, "0" or "off" = no
                              fold (the default, and the reference's GPU build, whose point set is the unfolded
                              tree); "auto" = find the group of axis permutations that leave the integrand
                              invariant; "p0,p1,...[;q0,...]" = these involutions, each checked.  With a group the
                              refinement levels evaluate only the children that are the minimum of their orbit,
                              weight each by the orbit size and keep whole orbits: the kept tree is unchanged, the
                              sums agree to rounding, and the evaluations drop by up to the group's order */
    double predict;        /* SINCQED_PREDICT = alpha (0 = off, the default): at the last level a child whose mean
                              |f| over the corners of its 2h cube (values of the level before, driver/sum.c:64-69)
                              is below alpha*thr is not evaluated; a controlled extra pruning loss */
    int group;             /* sqb_hsum_batch: 1 = the integrals of one graph (up to SQB_GROUP_MAX, e.g. the graph at
                              several h) run as one group (sqb_hsum_group), their refinement levels in shared
                              launches that take tiles of every integral from a device queue; 0 (default) = each
                              integral alone.  The results are the same bit for bit */
} sqb_opts_t;
#define SQB_GROUP_MAX 8
#define SQB_CKPT_STOPPED 2 /* sqb_hsum's return code under ckpt_stop */

/* res_t of the reference (driver/sq.h:111) and the per-graph log counters (driver/main.c:58-65) */
typedef struct {
    double S[3];           /* S_h, S_2h, S_4h (NaN where the run had no such level) */
    double Ah, ref, prune, trunc, unres, t;
    long nev, nq, kept_top;
    double es1, es2;       /* shadow-tier sums at the last level (eps*10, eps*100 runs) */
    int esok;
    long abskipped, unresdrop;
    int zero;              /* the integrand vanished at every probe node (driver/sum.c:346-359) */
    /* timing: host seconds for the top level (grow + dilate), device milliseconds per level */
    double t_top, t_levels;
    int nlev;
    long lev_evals[16];
    double lev_ms[16];
    /* with sqb_kernel_timing(1): milliseconds in the FP64 and double-double evaluation kernels, and the
     * number of FP64 launches; always: kernels of this library launched by the call */
    double f64_ms, dd_ms;
    long f64_launches, launches;
    /* the symmetry fold: group order (1 = none), its generators as the reference prints them
     * ("0,2,1,4,3; ..."), their largest deviation max|f(k) - f(k sigma)|/sum|terms| over 200 nodes, and
     * the refused SINCQED_SYM entries (one per line) */
    int sym_order;
    char sym_desc[256];
    double sym_worst;
    char sym_msg[512];
    long pskip;            /* final-level points the predictor left out (PSKIP, driver/sum.c:806) */
} sqb_result_t;

void sqb_default_opts(sqb_opts_t *o);
/* the hierarchical Sinc sum of one graph at (h, N, eps, top); top < 0 picks the reference's default
 * (driver/main.c:211-215).  Returns 0, or a nonzero error code (sqb_error() has the message). */
int  sqb_hsum(const char *graph, double h, int N, double eps, int top, const sqb_opts_t *o, sqb_result_t *r);
const char *sqb_error(void);

/* Many integrals at once (no counterpart in the reference, whose driver runs one graph after another,
 * driver/main.c:220-247): each job is one sqb_hsum(); `workers` host threads, each with its own CUDA
 * stream and device buffers, take the jobs in descending `cost` (ties in list order) so that one
 * integral's latency-bound top-level grow overlaps another's FP64 level passes.  Results and return
 * codes per job (res[j], rcs[j]); *device_ms = device time of the whole batch (CUDA events: every worker
 * stream waits on a start event of the caller's stream, which waits on every worker's end event).
 * Returns 0, or the number of failed jobs (sqb_error() names the first). */
typedef struct {
    const char *graph;
    double h; int N; double eps; int top;   /* as sqb_hsum; top < 0: the reference's default */
    double cost;                            /* scheduling estimate (e.g. expected evaluations); 0: list order */
} sqb_job_t;
int  sqb_hsum_batch(const sqb_job_t *jobs, int n, const sqb_opts_t *o, int workers, sqb_result_t *res, int *rcs,
                    double *device_ms);
/* Several integrals of ONE graph (n <= SQB_GROUP_MAX; e.g. the graph at several h) as one group: their
 * top levels one after another, then every refinement level as one sequence of launches over all the
 * integrals that have it (the FP64 and double-double kernels take tiles of every integral from a device
 * queue; one reduce, one finish with one block per integral, one scatter).  Each result (res[j], rcs[j]) is
 * bit for bit the one sqb_hsum gives alone.  No counterpart in the reference.  A group with a checkpoint
 * (ckpt_every > 0), the predictor, the all-dd form or the pass split runs its integrals one after another.
 * Returns 0, or the number of failed jobs (sqb_error() names the first). */
int  sqb_hsum_group(const sqb_job_t *jobs, int n, const sqb_opts_t *o, sqb_result_t *res, int *rcs);
/* the batch tuner: runs the calibration jobs twice per candidate worker count, the candidates in turn, rate[c]
 * = the better of the two runs' evaluated points per second of device time (the first run of a worker count
 * also pays its workers' first allocations); *best = the fastest candidate.  Returns 0 or a batch error. */
int  sqb_batch_tune(const sqb_job_t *jobs, int n, const sqb_opts_t *o, const int *cand, int ncand, double *rate,
                    int *best);

/* The symmetry fold's group search on its own (the part of driver/sum.c:464-592 that picks the group),
 * with the caller's evaluator: fn(ctx, n, k, f, ab) puts f and the |.| sum of the integrand at the n
 * lattice nodes k[i*D + d] (Sinc variables EX[k + K]) into f[i], ab[i] and returns 0.  spec as
 * sqb_opts_t.sym.  Out: elems[e*12 + i] = image axis i of element e (element 0 the identity), desc,
 * worst and msg as in sqb_result_t.  Returns the group order (1: no fold) or -1 if fn failed. */
typedef int (*sqb_sym_eval_fn)(void *ctx, long n, const int *k, double *f, double *ab);
int  sqb_sym_find(int D, sqb_sym_eval_fn fn, void *ctx, const char *spec, int *elems, char *desc, int ndesc,
                  double *worst, char *msg, int nmsg);

/* The scaling test (`sincqed scale GRAPH [kappa] [seed]`, driver/main.c:76-115) with the raw
 * double-double point function on the device: every direction e in {-E..E}^(n-1) \ {0} of the Schwinger
 * parameters (E = SCALE_E, 1 by default) about random x0 (srand(seed)), |ptq(x) prod x| at kappa/3,
 * 2 kappa/3 and kappa; a direction is slow if ratio = g(kappa)/g(2 kappa/3) > 0.3 and g(kappa) > 1e-30.
 * Returns 0, 1 if the graph has no raw point function (VP graphs: the reference prints "no scale test"),
 * or -1 (sqb_error()). */
typedef struct {
    int n, fixed;              /* Schwinger parameters, the fixed one */
    long ndir;                 /* directions tested: (2E+1)^(n-1) - 1 */
    int slow;                  /* slow directions */
    double worst;              /* the largest ratio, its direction (index and exponents) and g there */
    long worst_dir; int worst_e[16]; double worst_g[3];
    int listed_e[12][16]; double listed_g[12][3];   /* the first min(slow, 12) slow directions */
} sqb_scale_result_t;
int  sqb_scale_test(const char *graph, double kappa, unsigned seed, int E, sqb_scale_result_t *r);
/* its host halves, for a caller that evaluates the point function itself: the base point x0[n] and the
 * factor table xs[3 (2E+1)] (xs[q (2E+1) + e + E] = exp(-kappa (q+1)/3 e)); and the summary of the values
 * g[3 d + q] over the (2E+1)^(n-1) directions d */
void sqb_scale_setup(int n, int fixed, double kappa, unsigned seed, int E, double *x0, double *xs);
void sqb_scale_summary(int n, int fixed, int E, long ndir, const double *g, sqb_scale_result_t *r);

/* sizeof of a structure of this interface by its name ("sqb_opts_t", "sqb_result_t", "sqb_job_t",
 * "sqb_ckpt_t", "sqb_scale_result_t"; and the internal level interface "sqb_level_t", "sqb_acc_t",
 * "sqb_test_t", "sqb_scale_t"), so that a binding can check its copies; -1 if unknown */
long sqb_struct_size(const char *name);

/* the graphs compiled into this library: name, Volkov string, L, D, mirror weight */
int  sqb_graph_count(void);
const char *sqb_graph_name(int i);
/* info[0..5] = L, D, weight, n, fixed, zlattice; returns 0 if unknown */
int  sqb_graph_info(const char *name, int *info);
const char *sqb_graph_volkov(const char *name);
/* algorithmic FP64 flops per point of the graph's double path, with (ab=1) or without (ab=0) the |.|
 * sums: + - * / counted 1 each (scripts/plot5_cost.py:11); 0 if unknown */
double sqb_graph_flops(const char *name, int ab);

/* pointwise evaluation of the graph kernels on the device, for parity checks: n points sf[i*D + d]
 * (the Sinc variables), outputs f and the |.| sum; prec 0 = FP64 (ab: SQ_AB), 2 = FP64 contracted,
 * 1 = double-double, returned as (hi, lo) pairs in f2 and ab2 (2n entries each) */
int  sqb_eval_points(const char *graph, long n, const double *sf, int prec, int ab, double *f, double *abs_);

/* the device the library runs on ("off" before the first call) */
const char *sqb_device_info(void);
/* load the device code of a graph's kernels now (graph NULL: all graphs); CUDA otherwise loads each
 * kernel on its first launch, up to about a second for the largest graphs.  Returns the number of
 * kernels loaded, or -1 */
int  sqb_preload(const char *graph);

/* instrumentation: bracket every FP64 and double-double evaluation launch with events (read when the
 * call next waits on its stream, no extra synchronisation) so that sqb_result_t carries their times; and
 * the measured FP64 rate of this device in TFLOP/s (fma = 1: fused multiply-adds, 2 flops each; 0: adds),
 * the roofline denominator of the evaluation kernels */
void sqb_kernel_timing(int on);
double sqb_probe_fp64(int fma, long iters);
/* bytes copied host->device and device->host by the chosen form so far */
void sqb_copy_bytes(unsigned long long *h2d, unsigned long long *d2h);
/* CUDA events on the library's stream around a region of calls: device milliseconds */
int  sqb_timer_start(void);
double sqb_timer_stop(void);
/* overwrite `bytes` of device memory on the library's stream (an L2 flush between timed steps) */
int  sqb_l2_flush(size_t bytes);

/* ------------------------------------------------------------------------------------------------
 * 3. One refinement-level batch without allocation.  This entry point has no counterpart in the
 *    reference: it exists for callers that cannot let the library call cudaMalloc, such as a program
 *    that owns the device memory through its own pool allocator, or a service whose memory budget is
 *    fixed when it starts.  It runs the level pass of sqb_hsum (the 2^D children of ncell cells at step
 *    st: FP64 evaluation, double-double fallback, compensated sums, kept children appended in order) on
 *    a scratch array built into the library (SQB_NOALLOC_BYTES of device memory per GPU, held until the
 *    process exits) and calls no cudaMalloc, cudaFree or allocating library routine.
 *    - cells: device pt_t list (12 bytes per cell: k[0..D-1], flags in byte 11); next: device list for the
 *      kept children (unused when last != 0), next_cap entries;
 *    - h, K: the lattice (z = k h, |k| <= K); pw, thr: the level's weight step^D and keep threshold;
 *      abserr .. dropunres: the per-point test parameters (sqb_opts_t);
 *    - sums (host, 12 doubles): S, sum|v|, dropped weight, the two shadow-tier sums and the round column,
 *      each as (hi, lo); counts (host, 6): evaluated, kept, fallback, unresolved, skipped |.| sums,
 *      kept children that did not fit next_cap;
 *    - at most SQB_NOALLOC_CHILDREN children (ncell << D) per call, else SQB_NOALLOC_TOO_BIG and nothing
 *      runs; calls share the scratch, so calls whose GPU work overlaps race: issue them one at a time;
 *      the first call on a device looks up the scratch address, so make it before any stream capture;
 *    - each call waits for its stream before it returns (the sums and counters are host arrays): the host
 *      blocks until the call's GPU work is done;
 *    - the scratch is SQB_NOALLOC_BYTES of device memory on every GPU that loads the library, held until
 *      the process exits (the layout is checked against this size when the library is compiled).
 *    Returns 0, a negative SQB_NOALLOC_* code or a CUDA error code; sqb_error() has the message. */
#define SQB_NOALLOC_CHILDREN (1L << 18)
#define SQB_NOALLOC_BYTES (6700000L)
#define SQB_NOALLOC_BAD_ARG (-1)
#define SQB_NOALLOC_TOO_BIG (-2)
#define SQB_NOALLOC_SETUP (-3)
int  sqb_level_noalloc(const char *graph, double h, int K, const void *cells, long ncell, int st, int last,
                       double pw, double thr, double abserr, double nearf, double ddslack,
                       int abskip, int abcheck, int dropunres, void *next, long next_cap,
                       double *sums, long long *counts, void *stream);

/* ------------------------------------------------------------------------------------------------
 * 4. Checkpoints in the reference's format SQCK4 (driver/checkpoint.c:59-120, ckpt_t at driver/sq.h:84-93):
 *    the file sincqed_<graph>.ckpt that the reference writes and resumes from, field for field, so that
 *    either program resumes the other's run.  sqb_hsum writes one at the end of every level but the last
 *    (opts ckpt_every > 0): the next level's cells, streamed from the device in cell order, and the run's
 *    sums; it resumes from a file whose header matches (name, h, eps, N, top, dim, K) and removes it when
 *    the graph finishes.  The predictor table is written empty (vcap = 0: the predictor is off). */
typedef struct {
    char name[32]; double h, eps; int N, top, dim, k;    /* header ckhead_t (magic "SQCK4") */
    int lev; long next;                                  /* level to refine next, first unprocessed cell */
    double s, a, drop, u; long ne, q;                    /* sums of the level in progress (or just finished) */
    double Slev[16]; int nl;
    double S[3], Ah, ref, prune, trunc, unres, t;        /* res_t */
    long nev, nq, kept_top;
    long ncur; signed char *cur;                         /* cells, 12 bytes each (pt_t) */
    long nnxt; signed char *nxt;
    double es[5]; long cnt[3]; int esok;                 /* shadow sums and predictor check; counters */
    int vsz; long vcap, vn; void *vs;                    /* the predictor's table: vcap slots of vsz bytes */
} sqb_ckpt_t;
#define SQB_CKPT_VSLOT 16  /* sizeof(vslot_t) of the reference (driver/sum.c:85) */
/* write c to path atomically (path.tmp, then rename); 0 or -1 */
int  sqb_ckpt_save(const char *path, const sqb_ckpt_t *c);
/* read path into c (cur, nxt, vs allocated; free them with sqb_ckpt_free): 1 read, 0 absent, -1 damaged or
 * another format */
int  sqb_ckpt_load(const char *path, sqb_ckpt_t *c);
void sqb_ckpt_free(sqb_ckpt_t *c);
/* the file name the reference uses: <dir or .>/sincqed_<graph>.ckpt (driver/checkpoint.c:67-69) */
void sqb_ckpt_name(char *buf, size_t n, const char *dir, const char *graph);

#ifdef __cplusplus
}
#endif
