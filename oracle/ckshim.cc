/* Test infrastructure (oracle build only): C entry points to the reference's own checkpoint reader and
 * writer (driver/checkpoint.c:59-120, ckpt_save / ckpt_load), so that the tests can exchange checkpoint
 * files between the reference and the evaluator without running a sum.  Built into _ref/libsqck.so
 * together with the reference's checkpoint.c, io.c and lattice.c. */
#include "sq.h"

static void setup(const char *dir, const char *name, int dim, int k, graph_t *g){
    memset(g, 0, sizeof *g); g->name = name; g->volkov = name;
    setenv("SINCQED_CKPT_DIR", dir, 1);
    DIM = dim; K = k; CKPT_EVERY = 600;
}
extern "C" int ref_ckpt_save(const char *dir, const char *name, double h, int N, double eps, int top, int dim, int k, ckpt_t *c){
    graph_t g; setup(dir, name, dim, k, &g);
    return ckpt_save(&g, h, N, eps, top, c);
}
/* 1 if a matching checkpoint was read into c (cell lists malloc'ed by the reference), else 0 */
extern "C" int ref_ckpt_load(const char *dir, const char *name, double h, int N, double eps, int top, int dim, int k, ckpt_t *c){
    graph_t g; setup(dir, name, dim, k, &g);
    memset(c, 0, sizeof *c); c->vsz = 16;
    return ckpt_load(&g, h, N, eps, top, c);
}
extern "C" void ref_ckpt_free(ckpt_t *c){ free(c->cur.p); free(c->nxt.p); free(c->vs); memset(c, 0, sizeof *c); }
extern "C" int ref_ckpt_sizeof(void){ return (int)sizeof(ckpt_t); }
