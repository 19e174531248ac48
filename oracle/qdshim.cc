/* Test infrastructure (oracle build only): a quad-double oracle of the two-loop kernels.  The reference's
 * kernels/g2 sources compile unchanged over its own quad-double type (pslq/quad/qd.h, ~64 digits, every
 * operation an exact expansion cut to four doubles) when pslq/quad/common.h stands in for driver/common.h
 * (pslq/quad/Makefile builds its extended-precision sums that way).  This shim evaluates their QREAL half
 * at given Sinc variables, for the tests that state the double-double kernels' error against it. */
#include <string.h>
#include "common.h"              /* pslq/quad/common.h: -I order of oracle/Makefile */

__thread int SQ_AB = 1;
extern const graph_t G_g2_00, G_g2_01, G_g2_02, G_g2_03, G_v2_00;
static const graph_t *const ALLQ[] = {&G_g2_00, &G_g2_01, &G_g2_02, &G_g2_03, &G_v2_00};

/* n points sf[i*D + d]; f and ab get the four components of each value (4n doubles each); returns D or -1 */
extern "C" int sqqd_fq(const char *name, long n, const double *sf, double *f, double *ab){
    for(const graph_t *g : ALLQ){
        if(strcmp(g->name, name)) continue;
        const int D = g->D;
        for(long i = 0; i < n; i++){
            qd s[16], a;
            for(int d = 0; d < D; d++) s[d] = qd(sf[i*D + d]);
            qd v = g->fq(s, &a);
            for(int c = 0; c < 4; c++){ f[4*i + c] = v.x[c]; ab[4*i + c] = a.x[c]; }
        }
        return D;
    }
    return -1;
}
