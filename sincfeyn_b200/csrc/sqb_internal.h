/* sqb_internal.h -- what the generated per-graph translation units and the runtime share: the launch
 * arguments of the evaluation kernels and the graph descriptor with its launchers.  Not part of the
 * public C ABI (include/sincfeyn_b200.h). */
#pragma once
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* status bits of one evaluated point (test mode) */
enum {
    SQB_PRESENT = 1,      /* a lattice node (not a child below the box) */
    SQB_NEAR = 2,         /* |.| bound above NEARF*ABSERR: its children must check (driver/eval.c:37) */
    SQB_FALLBACK = 4,     /* |.| bound above ABSERR: recomputed in double-double (driver/eval.c:38) */
    SQB_UNRES = 8,        /* unresolved even in double-double (driver/eval.c:28) */
    SQB_SKIPPED = 16      /* evaluated without the |.| sums (driver/eval.c:35) */
};

/* A group of axis permutations under which the integrand is invariant (the symmetry fold of
 * driver/sum.c:21-46): n elements, g[0] the identity, image of k under element e: k'_i = k[g[e][i]].
 * n <= 1: no fold.  With a group, a level batch evaluates only the children that are the lexicographic
 * minimum of their orbit, weights each by the orbit size and keeps the whole orbit. */
#define SQB_SYMG 64
typedef struct {
    int n;
    signed char g[SQB_SYMG][12];
} sqb_sym_t;

/* One launch of the FP64 evaluation kernel over nodes, or over the 2^D children of cells.
 * Coordinates are integers k (|k| <= K) of esize bytes (1: the pt_t layout of the level lists and
 * checkpoints, 2: the int16 layout of the reference's GPU plug-in), stride elements per node or
 * cell; the per-node flags byte (pt_t slot PFLAG) sits at element flag_at, or flag_at < 0. */
/* the sums of one tile of SQB_TILE consecutive children of a level batch, double-double (hi, lo) */
#define SQB_TILE 4096
/* the FP64 kernel's running tile sums in level mode, one column per thread of its SQB_TILE_THREADS:
 * dynamic shared memory after the launch's tables (the host adds its size to such launches) */
#define SQB_TILE_THREADS 128
typedef struct {
    double S[2][SQB_TILE_THREADS], A[SQB_TILE_THREADS], dr[SQB_TILE_THREADS], b1[2][SQB_TILE_THREADS], b2[2][SQB_TILE_THREADS];
    unsigned ne[SQB_TILE_THREADS], nsk[SQB_TILE_THREADS], keep[SQB_TILE_THREADS];
    int fb;
} sqb_tile_acc;
typedef struct {
    double S[2], A[2], drop[2], b1[2], b2[2], u[2];
    unsigned long long ne, nq, unres, skipped;
} sqb_part_t;

/* One integral of a multi-instance level launch: the instances of one graph at several h (or several
 * integrals of it) share a launch, the launch's children numbered instance after instance, each instance's
 * range starting at a multiple of SQB_TILE so that no tile straddles two instances. */
#define SQB_MAXINST 8
typedef struct {
    const void *pts;              /* its cells (device), pt_t layout */
    long n;                       /* its cells in this launch */
    long child0;                  /* its first child in the launch's numbering (a multiple of SQB_TILE) */
    int st, K, toff, fused;       /* step; lattice half-width; offset of its tables in the launch's shared
                                     table area (X then Wt, 2K+1 each); the FP64 kernel sums its tiles */
    int last;
    double pw, thr;               /* its level's weight step^D and keep threshold */
    double abserr, near_thr;      /* its per-point test thresholds (ABSERR depends on the integral's Ref) */
    const double *X, *Wt;         /* its tables (device, 2K+1 each) */
} sqb_inst_t;

typedef struct {
    const void *pts;
    long n;                       /* nodes, or cells */
    int esize, stride, flag_at;
    int cells, st;                /* cells: child b of cell c is k_d - st*bit_d(b) (driver/sum.c:407) */
    const double *X, *Wt;         /* 2K+1 entries: integration variable and weight factor per k;
                                     Wt == NULL: the factor is X*H (driver/lattice.c:33) */
    int K;
    double H;
    int raw;                      /* 1: plain form, v = f w and ab = ab w, no tests */
    const unsigned char *skip;    /* per node or cell: evaluate without the |.| sums (may be NULL) */
    int abskip, abcheck;          /* with flag_at >= 0: skip = abskip && (flags & 1) */
    double abserr, near_thr, ddslack;
    double *v, *ab;               /* value per point (raw: f w); raw only: ab w */
    const double *sfin;           /* raw only, pointwise checks: the D variables of point i at sfin[i*D], w = 1 */
    double *vlo, *ablo;           /* raw double-double pass: the low parts of f and ab */
    unsigned char *stt;           /* test mode: status per point */
    long *fb;                     /* test mode: points that need the fallback (unordered) */
    unsigned long long *nfb;
    long fbcap;
    /* level mode (test mode over cells, part != NULL): the FP64 pass also sums every tile of SQB_TILE
     * children that needs no fallback (part, tkeep: kept count), and flags the others (tfb = 1) for the
     * reduce kernel, which sums them after the double-double pass */
    sqb_part_t *part;
    unsigned *tkeep;
    unsigned char *tfb;
    double pw, thr;               /* the level's weight step^D and keep threshold */
    int last;                     /* the last level: shadow-tier sums, no kept children */
    sqb_sym_t sym;                /* cells only: the symmetry fold (sym.n <= 1: off) */
    const unsigned char *cfl;     /* cells only, the predictor at the last level (NULL: off): per child, bit 0 =
                                     not evaluated, bits 1-2 = its shadow tier */
    /* multi-instance level launch (ninst >= 1, cells, level mode): the instances' own fields above are
     * unused; the CTAs take tiles of SQB_TILE children from the device counter queue in turn, children
     * numbered as sqb_inst_t says (ntile tiles in all).  ninst = 0: one batch described by the fields above */
    int ninst;
    long ntile;
    unsigned long long *queue;
    sqb_inst_t inst[SQB_MAXINST];
    /* list mode (one integral's level batch under a fold or the predictor): the children to evaluate, as
     * child index | orbit weight << 56, *nsel of them, written by the select pass, which also zeroed the
     * others; the FP64 kernel walks the list (tiles of SQB_TILE entries from the queue) and leaves every
     * tile's sums to the reduce kernel */
    const unsigned long long *sel, *nsel;
} sqb_eval_t;
#define SQB_SEL_SHIFT 56

/* The double-double kernel over a list of points of the same launch geometry (fb/nfb from the FP64
 * pass), or over every point (all = 1: the all-double-double form). */
typedef struct {
    sqb_eval_t e;                 /* geometry, tables, outputs v and stt */
    const long *list;             /* NULL with all = 1 */
    const unsigned long long *nlist;
    long listcap;
    int all;
    int dropunres;
    double *uu;                   /* per point: e^2 of the round column (driver/eval.c:26) */
} sqb_dd_t;

/* The scaling test (sincqed scale, driver/main.c:79-115): for direction d (exponent e_i in -E..E of each
 * Schwinger parameter but the fixed one, base-(2E+1) digits of d) and q = 0, 1, 2 the parameters
 * x_i = x0_i * xs[q][e_i + E] (xs[q][j] = exp(-kappa (q+1)/3 (j - E)), double-double products),
 * meas = prod_{i != fixed} x_i, and g[3 d + q] = |(double)(ptq(x, 0) meas)|; 0 for d = 0 */
#define SQB_SCALE_MAXN 16
typedef struct {
    int n, fixed, E;
    long ndir;
    double x0[SQB_SCALE_MAXN];
    const double *xs;             /* device: 3 x (2E+1) */
    double *g;                    /* device: 3 ndir */
} sqb_scale_t;

typedef struct {
    int regs, local_bytes, max_threads, blocks_per_sm;
    int fused;                    /* FP64 kernel: sums level tiles itself (level mode available) */
    int sweeps;                   /* level kernel: passes over a batch's tiles (1, or 2: see SQB_SWEEPS) */
} sqb_kattr_t;
#define SQB_ATTR_LEVEL 4          /* attr(which | SQB_ATTR_LEVEL, ...): the FP64 level kernel's attributes */
/* a launch that the FP64 level kernel runs: a level batch of cells (int8 coordinates) whose tiles come from
 * the device queue, not in list mode */
static inline bool sqb_level_launch(const sqb_eval_t *a){
    return a->ninst > 0 && a->cells && a->esize == 1 && a->part && !a->sel && !a->sfin && !a->raw;
}

typedef struct {
    const char *name, *volkov;
    int L, D, weight, n, fixed;
    int zlattice;                              /* 1: the variable is z itself (synthetic integrand) */
    void (*f64)(const sqb_eval_t *a, int grid, int block, size_t smem, void *stream);
    void (*dd)(const sqb_dd_t *a, int grid, int block, size_t smem, void *stream);
    /* which: 0 FP64 kernel, 1 dd kernel, 2 contracted FP64 kernel, with SQB_ATTR_LEVEL added: the FP64
     * level kernel of that build; blocks_per_sm for this block size and dynamic shared memory; 0 if that
     * kernel is not in the library */
    int (*attr)(int which, int block, size_t smem, sqb_kattr_t *out);
    /* the FP64 kernel compiled with contraction (-fmad=true: fused multiply-adds), from the graph's second
     * translation unit; NULL if the library was built without it */
    void (*f64_fma)(const sqb_eval_t *a, int grid, int block, size_t smem, void *stream);
    /* nparts > 0: the FP64 pass of a level batch may run as nparts passes (P = 0 .. nparts-1), each adding
     * a group of the point function's nodes to the point's running sums tt[i], ta[i], and a final pass
     * (P = nparts) with the tests; fma: the contracted build */
    int nparts;
    void (*split)(int P, int fma, const sqb_eval_t *a, double *tt, double *ta, int grid, int block, size_t smem,
                  void *stream);
    int (*split_attr)(int P, int fma, int block, size_t smem, sqb_kattr_t *out);
    /* the scaling test on the raw double-double point function ptq; NULL for graphs without one (VP) */
    void (*scale)(const sqb_scale_t *a, int grid, int block, void *stream);
} sqb_graph_t;

#ifdef __cplusplus
}
#endif
