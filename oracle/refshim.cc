/* Test infrastructure (oracle build only): a C entry point into the reference's own kernels, for the
 * pointwise parity tests.  Linked into oracle/_ref/libsqref.so together with the reference kernels
 * (compiled by oracle/Makefile with -ffp-contract=off), driver/graphs.c and the generated registry.
 *
 * The reference calls its kernels through graph_t (driver/common.h:26-38): fd(sf, &ab) in double with
 * the thread-local SQ_AB flag gating the |.| sums, fq(sq, &abq) in QREAL (double-double here), and the
 * packed fv(n, sf, ld, out, ab).  Nothing here changes how they compute. */
#include "sq.h"

__thread int SQ_AB = 1;      /* defined by driver/eval.c in the reference binary */
static int ready = 0;
static void init(void){ if(!ready){ register_graphs(); ready = 1; } }

extern "C" {
int sqref_count(void){ init(); return NALL; }
const char *sqref_name(int i){ init(); return i >= 0 && i < NALL ? ALL[i]->name : NULL; }
/* L, D, weight, n (Schwinger parameters), fixed, has_fv; returns 0 if the graph is unknown */
int sqref_info(const char *name, int *info){
    init(); const graph_t *g = find(name); if(!g) return 0;
    info[0] = g->L; info[1] = g->D; info[2] = g->weight; info[3] = g->n; info[4] = g->fixed; info[5] = g->fv != NULL;
    return 1;
}
const char *sqref_volkov(const char *name){ init(); const graph_t *g = find(name); return g ? g->volkov : NULL; }
/* fd at n points sf[i*D + d]; sqab = SQ_AB during the call (driver/eval.c:57-58) */
int sqref_fd(const char *name, long n, const double *sf, int sqab, double *f, double *ab){
    init(); const graph_t *g = find(name); if(!g) return 0;
    int D = g->D;
    for(long i = 0; i < n; i++){ SQ_AB = sqab; f[i] = g->fd(sf + i*D, &ab[i]); SQ_AB = 1; }
    return 1;
}
/* the packed fv (driver/eval.c:66-73): all n points in one call */
int sqref_fv(const char *name, long n, const double *sf, int sqab, double *f, double *ab){
    init(); const graph_t *g = find(name); if(!g || !g->fv) return 0;
    SQ_AB = sqab; g->fv(n, sf, g->D, f, ab); SQ_AB = 1;
    return 1;
}
/* fq in double-double: value and |.| sum as (hi, lo) pairs (driver/eval.c:43-44) */
int sqref_fq(const char *name, long n, const double *sf, double *f2, double *ab2){
    init(); const graph_t *g = find(name); if(!g) return 0;
    int D = g->D;
    for(long i = 0; i < n; i++){
        QREAL sq[MAXD], abq; for(int d = 0; d < D; d++) sq[d] = (QREAL)sf[i*D + d];
        QREAL v = g->fq(sq, &abq);
        f2[2*i] = v.hi; f2[2*i + 1] = v.lo; ab2[2*i] = abq.hi; ab2[2*i + 1] = abq.lo;
    }
    return 1;
}
}
