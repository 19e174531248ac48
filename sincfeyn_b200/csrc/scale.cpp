/* scale.cpp -- the scaling test (`sincqed scale GRAPH [kappa] [seed]`, driver/main.c:76-115) with the
 * graph's raw double-double point function evaluated on the device.
 *
 * With x0_i = exp(4 rand()/RAND_MAX - 2) after srand(seed) (x0 = 1 at the fixed parameter), every
 * direction e in {-E..E}^(n-1) \ {0} (SCALE_E, default 1) scales x_i = x0_i exp(-kappa' e_i) and
 * measures g(kappa') = |ptq(x) prod_{i != fixed} x_i| at kappa' = kappa/3, 2 kappa/3, kappa: the
 * integrand times the measure must vanish along every direction as kappa' grows, so
 * ratio = g(kappa)/g(2 kappa/3) above 0.3 (with g(kappa) > 1e-30) marks a slow direction.  The device
 * computes the 3 (2E+1)^(n-1) values in double-double exactly as the reference's QREAL code does; the
 * host takes the directions in order (the reference's with one thread) for the worst ratio and the
 * first twelve slow directions. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <vector>
#include "sqb_rt.h"
#include "sqb_rand.h"
#include "sincfeyn_b200.h"

extern "C" void sqb_set_error_msg(const char *msg);

/* the host half: the random base point and factor table of driver/main.c:80-96 */
extern "C" void sqb_scale_setup(int n, int fixed, double kappa, unsigned seed, int E, double *x0, double *xs){
    SqbRand rng(seed);
    for(int i = 0; i < n; i++) x0[i] = exp(4.0*rng.next()/RAND_MAX - 2.0);
    x0[fixed] = 1;
    const int B = 2*E + 1;
    for(int q = 0; q < 3; q++){
        const double kk = kappa*(q + 1)/3.0;
        for(int e = -E; e <= E; e++) xs[q*B + e + E] = exp(-kk*e);
    }
}
/* ... and the directions in order over the values g[3 d + q] (driver/main.c:98-108, one thread) */
extern "C" void sqb_scale_summary(int n, int fixed, int E, long ndir, const double *gv, sqb_scale_result_t *r){
    const int B = 2*E + 1;
    r->n = n; r->fixed = fixed; r->ndir = ndir - 1; r->slow = 0; r->worst = 0; r->worst_dir = -1;
    for(long d = 0; d < ndir; d++){
        int e[SQB_SCALE_MAXN] = {0}, nz = 0; long q = d;
        for(int i = 0; i < n; i++){ if(i == fixed){ e[i] = 0; continue; } e[i] = (int)(q % B) - E; q /= B; nz += e[i] != 0; }
        if(!nz) continue;
        const double *gd = &gv[3*d];
        const double ratio = gd[1] > 0 ? gd[2]/gd[1] : 0;
        if(ratio > r->worst){
            r->worst = ratio; r->worst_dir = d;
            memcpy(r->worst_g, gd, sizeof r->worst_g); memcpy(r->worst_e, e, sizeof e);
        }
        if(ratio > 0.3 && gd[2] > 1e-30){
            if(r->slow < 12){ memcpy(r->listed_e[r->slow], e, sizeof e); memcpy(r->listed_g[r->slow], gd, sizeof r->listed_g[0]); }
            r->slow++;
        }
    }
}

extern "C" int sqb_scale_test(const char *graph, double kappa, unsigned seed, int E, sqb_scale_result_t *r){
    char msg[256];
    memset(r, 0, sizeof *r);
    r->worst_dir = -1;
    const sqb_graph_t *g = sqb_find_graph(graph);
    if(!g){ snprintf(msg, sizeof msg, "no graph %s in this build", graph); sqb_set_error_msg(msg); return -1; }
    r->n = g->n; r->fixed = g->fixed;
    if(!g->scale) return 1;                              /* VP graphs: no raw point function */
    if(E < 1 || g->n < 2 || g->n > SQB_SCALE_MAXN || g->fixed < 0 || g->fixed >= g->n){
        snprintf(msg, sizeof msg, "%s: scale test needs E >= 1 and 2 <= n <= %d (n = %d)", graph, SQB_SCALE_MAXN, g->n);
        sqb_set_error_msg(msg); return -1;
    }
    const int n = g->n, fixed = g->fixed, B = 2*E + 1;
    long ndir = 1;
    for(int i = 0; i < n - 1; i++){
        if(ndir > (1L << 26)/B){ snprintf(msg, sizeof msg, "%s: (2E+1)^(n-1) directions exceed 2^26", graph); sqb_set_error_msg(msg); return -1; }
        ndir *= B;
    }
    if(sqb_dev_init(0)){ snprintf(msg, sizeof msg, "device: %s", sqb_last_error()); sqb_set_error_msg(msg); return -1; }
    sqb_scale_t a; memset(&a, 0, sizeof a);
    a.n = n; a.fixed = fixed; a.E = E; a.ndir = ndir;
    std::vector<double> xs(3*(size_t)B), gv(3*(size_t)ndir);
    sqb_scale_setup(n, fixed, kappa, seed, E, a.x0, xs.data());
    const int rc = sqb_dev_scale(g, &a, xs.data(), gv.data());
    if(rc < 0){ snprintf(msg, sizeof msg, "device: %s", sqb_last_error()); sqb_set_error_msg(msg); return -1; }
    sqb_scale_summary(n, fixed, E, ndir, gv.data(), r);
    return 0;
}
