/* engine.cpp -- the host side of the chosen form: sqb_hsum(), the hierarchical Sinc sum of one graph
 * (driver/sum.c:556-814), with every refinement level resident on the device.
 *
 *   lattice      K rounded up to a multiple of 2^(top+1); EX[k+K] = e^{kh}, weight factor EX*h
 *                (driver/lattice.c:13-34);
 *   box_zero     4097 fixed probe nodes; an integrand that is 0 at all of them is reported as zero
 *                (driver/sum.c:346-359);
 *   grow         the support-following top level (driver/sumkey.h:126-461): breadth-first from z = 0
 *                over axis neighbours at step 2^top h; a frontier is evaluated as one device batch,
 *                its values come to the host for the order-dependent sums (Neumaier S, the running
 *                sum|f w| whose threshold eps_rel * a decides what is kept, the outer shells, the
 *                dropped weight), and the device builds the next frontier: every not-yet-seen
 *                neighbour of a kept point, in (kept point, axis, sign) order -- the order the
 *                reference's parallel lowest-id claims produce (topgrid.cu); then the final
 *                re-threshold and the shadow-tier flood fill on the device.  One table holds every
 *                evaluated point, which is the reference's result whenever it reports no candidate
 *                below its freed boundary tables (BTUNS = 0, driver/sum.c:631);
 *   dilate       on the device: the kept cells and their axis neighbours, deduplicated (skip bit AND,
 *                tier max) and radix-sorted by mixed-radix key, i.e. lexicographically in k
 *                (driver/sumkey.h:20-90);
 *   levels       sqb_dev_level() for lev = top-1 .. 0 (driver/sum.c:652-799), the cell lists staying
 *                in device memory.
 * Sums of the grow are Neumaier sums in point order as the reference's kadd (driver/sum.c:18-20);
 * the levels' sums are double-double on the device. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdint.h>
#include <vector>
#include <algorithm>
#include <omp.h>
#include <chrono>
#include <future>
#include "sqb_rt.h"
#include "sincfeyn_b200.h"

static thread_local char E_[512];
static thread_local double MEMSHARE = 1.0;    /* share of device memory for this thread's cell lists */
extern "C" void sqb_set_mem_share(double f){ MEMSHARE = f > 0 && f <= 1 ? f : 1.0; }
extern "C" const char *sqb_error(void){ return E_; }
extern "C" void sqb_set_error_msg(const char *msg){ snprintf(E_, sizeof E_, "%s", msg); }
#define FAIL(...) do { snprintf(E_, sizeof E_, __VA_ARGS__); return -1; } while(0)

static double now(void){ return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

extern "C" void sqb_default_opts(sqb_opts_t *o){
    memset(o, 0, sizeof *o);
    o->abserr0 = 1e-15; o->abrel = 1e-3; o->nearf = 1e-3; o->ddslack = 1;
    o->abskip = 1; o->abcheck = 0; o->dropunres = 1; o->growskip = 2;
    o->alldd = 0; o->device = 0; o->max_children = 0; o->verbose = 0;
    o->fma = 1; o->split = 0;
}

/* sizeof of the structures a binding mirrors (the public ones and the level interface), so that a
 * binding can check its copies; -1 for an unknown name */
extern "C" long sqb_struct_size(const char *name){
    static const struct { const char *n; long s; } T[] = {
        {"sqb_opts_t", sizeof(sqb_opts_t)}, {"sqb_result_t", sizeof(sqb_result_t)}, {"sqb_job_t", sizeof(sqb_job_t)},
        {"sqb_ckpt_t", sizeof(sqb_ckpt_t)}, {"sqb_scale_result_t", sizeof(sqb_scale_result_t)},
        {"sqb_level_t", sizeof(sqb_level_t)}, {"sqb_acc_t", sizeof(sqb_acc_t)}, {"sqb_test_t", sizeof(sqb_test_t)},
        {"sqb_scale_t", sizeof(sqb_scale_t)}};
    for(const auto &e : T) if(name && !strcmp(name, e.n)) return e.s;
    return -1;
}

extern "C" int sqb_graph_count(void){ return sqb_ngraphs(); }
extern "C" const char *sqb_graph_name(int i){ const sqb_graph_t *g = sqb_graph_at(i); return g ? g->name : NULL; }
extern "C" const char *sqb_graph_volkov(const char *name){ const sqb_graph_t *g = sqb_find_graph(name); return g ? g->volkov : NULL; }
extern "C" int sqb_graph_info(const char *name, int *info){
    const sqb_graph_t *g = sqb_find_graph(name); if(!g) return 0;
    info[0] = g->L; info[1] = g->D; info[2] = g->weight; info[3] = g->n; info[4] = g->fixed; info[5] = g->zlattice;
    return 1;
}
extern "C" const char *sqb_device_info(void){ return sqb_dev_info(); }

/* Neumaier sum, driver/sum.c:18-20 */
struct ksum { double s = 0, c = 0;
    void add(double x){ double t = s + x; if(fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s; s = t; }
    double val() const { return s + c; } };

/* ---------------------------------------------------------------------------------------------- */
/* the run of one graph */
struct Run {
    const sqb_graph_t *g; int D, K, top; double h, eps;
    sqb_opts_t o; sqb_test_t t;
    std::vector<double> X, Wt;
    long nq = 0, unresdrop = 0; double u = 0;
    sqb_vtab_t *vt = NULL;          /* the predictor's table (opts.predict > 0), else NULL */
};
/* releases the predictor's table on every return of sqb_hsum */
struct VtabGuard { sqb_vtab_t t; VtabGuard(){ memset(&t, 0, sizeof t); } ~VtabGuard(){ sqb_vtab_free(&t, sqb_dev_stream()); } };
/* the predictor's table must not have overflowed */
static int vt_check(Run &R, char *err, size_t n){
    if(!R.vt) return 0;
    long vn = 0, full = 0;
    if(sqb_vtab_counts(R.vt, &vn, &full, sqb_dev_stream())){ snprintf(err, n, "predictor: %s", sqb_vtab_error()); return -1; }
    if(full){ snprintf(err, n, "predictor: %ld values found its table full", full); return -1; }
    return 0;
}

static void set_test(Run &R, double abserr){
    R.t.abserr = abserr; R.t.nearf = R.o.nearf; R.t.ddslack = R.o.ddslack;
    R.t.abskip = R.o.abskip; R.t.abcheck = R.o.abcheck; R.t.dropunres = R.o.dropunres; R.t.alldd = R.o.alldd;
    R.t.fma = R.o.fma; R.t.split = R.o.split;
}

static int eval(Run &R, const std::vector<sqb_pt_t> &p, const unsigned char *skip, std::vector<double> &v, std::vector<unsigned char> &nr){
    v.resize(p.size()); nr.resize(p.size());
    if(p.empty()) return 0;
    if(sqb_dev_eval_nodes(R.g, (long)p.size(), p.data(), skip, &R.t, v.data(), nr.data(), &R.nq, &R.u, &R.unresdrop))
        FAIL("device: %s", sqb_last_error());
    return 0;
}

/* driver/sum.c:346-359 */
static int box_zero(Run &R, int lev, long *nev, int *zero){
    const int st = 1 << lev, W = 2*(R.K/st) + 1, NP = 4096;
    std::vector<sqb_pt_t> p(NP + 1);
    for(long i = 0; i <= NP; i++){
        memset(&p[i], 0, sizeof p[i]);
        unsigned long long y = 0x9E3779B97F4A7C15ULL*(unsigned long long)(i + 1);
        if(i) for(int d = 0; d < R.D; d++){ y ^= y >> 29; y *= 0xBF58476D1CE4E5B9ULL; y ^= y >> 32; p[i].k[d] = (signed char)(((int)(y % (unsigned long long)W) - R.K/st)*st); }
    }
    std::vector<double> v; std::vector<unsigned char> nr;
    long nq0 = R.nq; double u0 = R.u;
    if(eval(R, p, NULL, v, nr)) return -1;
    R.nq = nq0; R.u = u0;        /* the probe's fallback count and round column are its own; its
                                    unresolved points are counted, as the global UNRESDROP does */
    *zero = 1;
    for(double x : v) if(x != 0){ *zero = 0; break; }
    if(*zero) *nev += NP + 1;
    return 0;
}

/* mixed-radix key (driver/sumkey.h:7-18): 1 c_0 ... c_{D-1} in base W, c_i = k_i/st + K/st; W = 0 if
 * the keys would not fit 63 bits; *nbits = bit length of the largest key */
static int keyradix(const Run &R, int st, uint64_t *P, int *nbits){
    const uint64_t W = 2*(R.K/st) + 1, TOP = 1ULL << 63; uint64_t p = 1;
    for(int i = R.D - 1; i >= 0; i--){ P[i] = p; if(p > TOP/W) return 0; p *= W; }
    *nbits = 64 - __builtin_clzll(p) + 1;             /* keys < 2 W^D */
    return (int)W;
}

struct GrowOut { double S, A, e1, e2, drop, gshs; long gshn, nev; };

/* driver/sumkey.h:126-461 (see the file comment); the kept cells, dilated at the same step when
 * dilate_out is given, stay on the device */
static int grow(Run &R, int lev, double eps_rel, GrowOut *go, sqb_pt_t **dilated, long *ndil){
    const int st = 1 << lev; uint64_t P[SQB_MAXD]; int nbits = 0;
    const int W = keyradix(R, st, P, &nbits);
    if(!W) FAIL("lattice too wide for 64-bit grid keys (D=%d, N=%d, step %dh)", R.D, 2*R.K + 1, st);
    const double pw = pow(st, R.D);
    const int store = lev > 0, gs = lev == 0 && R.o.abskip ? R.o.growskip : 0;
    if(sqb_grow_begin(R.D, R.K, st, W, (const unsigned long long*)P, gs, R.o.abskip, sqb_dev_stream()))
        FAIL("device grow: %s", sqb_top_error());
    /* the grow's device tables are released on every return, an error included, so that a failed
     * integral leaves its memory to the next one */
    struct End { ~End(){ sqb_grow_end(); } } end_of_grow;
    std::vector<unsigned char> stt;
    ksum ks; double a = 0, x1 = 0, x2 = 0, dr = 0, gshs = 0; long ne = 0, gshn = 0, nkeep = 0;
    double te = 0, th = 0, tx = 0; int nfr = 0; const double tg0 = now();    /* phase times (verbose) */
    /* A frontier's order-dependent sums that its expansion does not need (the Neumaier S, the shell, drop
     * and shadow sums) run on a helper task while the device expands the frontier and evaluates the next;
     * the tasks run one frontier after another (each waits for its predecessor), each over its frontier in
     * point order, so every sum is the in-line one bit for bit.  Only the |v| sum that sets the threshold
     * stays in line.  Values and shell classes alternate between two buffers; every return joins the
     * tasks first. */
    std::vector<double> vb[2]; std::vector<unsigned char> cb[2];
    std::shared_future<void> fut[2], last;
    struct Join { std::shared_future<void> &f; ~Join(){ if(f.valid()) f.wait(); } } join{last};
    for(;;){
        const sqb_pt_t *pts; const unsigned char *skip;
        const long n = sqb_grow_frontier(&pts, &skip);
        if(n <= 0) break;
        const int b = nfr & 1;
        if(fut[b].valid()) fut[b].wait();          /* the task two frontiers back read this buffer */
        std::vector<double> &v = vb[b]; std::vector<unsigned char> &cls = cb[b];
        v.resize(n); stt.resize(n); cls.resize(n);
        const double *vd; const unsigned char *sd;
        const double t0 = now();
        if(sqb_grow_shells_async()) FAIL("device grow: %s", sqb_top_error());
        if(sqb_dev_eval_resident(R.g, pts, n, skip, &R.t, v.data(), stt.data(), &R.nq, &R.u, &R.unresdrop, &vd, &sd))
            FAIL("device: %s", sqb_last_error());
        sqb_grow_shells_take(cls.data());
        /* the predictor stores every grow value (driver/sumkey.h:219-222) */
        if(R.vt && (sqb_vtab_reserve(R.vt, n, sqb_dev_stream()) || sqb_vtab_put_nodes(R.vt, pts, vd, n, R.D, sqb_dev_stream())))
            FAIL("predictor: %s", sqb_vtab_error());
        const double t1 = now(); te += t1 - t0; nfr++;
        ne += n;
        /* the frontier's sums in point order, then its threshold (driver/sumkey.h:225-245) */
        for(long i = 0; i < n; i++) a += fabs(v[i])*pw;
        const double thr = eps_rel*a;
        {
            const std::shared_future<void> prev = last;
            last = fut[b] = std::async(std::launch::async, [&, b, n, thr, prev]{
                if(prev.valid()) prev.wait();
                const double *vv = vb[b].data(); const unsigned char *cc = cb[b].data();
                for(long i = 0; i < n; i++) ks.add(vv[i]*pw);
                for(long i = 0; i < n; i++){
                    const double w = fabs(vv[i])*pw;
                    if(cc[i] & 2) x1 += w; else if(cc[i] & 4) x2 += w;
                    if(!(fabs(vv[i]) >= thr)){ dr += w; gshs += vv[i]*pw; gshn++; }
                }
            }).share();
        }
        long nk = 0, nn = 0;
        const double t2 = now(); th += t2 - t1;
        if(sqb_grow_expand(vd, sd, thr, &nk, &nn)) FAIL("device grow: %s", sqb_top_error());
        tx += now() - t2;
        nkeep += nk;
    }
    if(last.valid()) last.wait();                  /* every frontier's sums are in */
    const double tg1 = now();
    /* the final threshold, driver/sumkey.h:399-401 */
    const double thr = eps_rel*a;
    { std::vector<double> kv(nkeep);
      if(nkeep && sqb_grow_kv(kv.data(), nkeep)) FAIL("device grow: %s", sqb_top_error());
      for(long i = 0; i < nkeep; i++) if(!(kv[i] >= thr)) dr += kv[i]*pw; }
    long m = 0;
    if(sqb_grow_finish(thr, store && R.D < SQB_MAXD, &m)) FAIL("device grow: %s", sqb_top_error());
    /* ... and what the eps*10^t grows evaluated (driver/sumkey.h:445-451) */
    if(R.vt && store && R.D < SQB_MAXD && m){
        const sqb_pt_t *kp; long km;
        sqb_grow_kept(&kp, &km);
        if(sqb_vtab_raise_kept(R.vt, kp, km, R.D, st, R.K, sqb_dev_stream())) FAIL("predictor: %s", sqb_vtab_error());
    }
    const double tg2 = now();
    *dilated = NULL; *ndil = 0;
    if(store && sqb_grow_dilate(nbits, dilated, ndil)) FAIL("device dilate: %s", sqb_top_error());
    if(R.o.verbose)
        fprintf(stderr, "# %s grow: %d frontiers, %ld points, %ld kept: eval %.1f ms, host sums %.1f ms, expand %.1f ms; "
                "final threshold + tiers %.1f ms; dilate %.1f ms (%ld cells)\n", R.g->name, nfr, ne, nkeep,
                1e3*te, 1e3*th, 1e3*tx, 1e3*(tg2 - tg1), 1e3*(now() - tg2), *ndil);
    (void)tg0;
    go->S = ks.val(); go->A = a; go->e1 = x1; go->e2 = x2; go->drop = dr; go->gshs = gshs; go->gshn = gshn; go->nev = ne;
    return 0;
}

static inline double ddv(const double *x){ return x[0] + x[1]; }

/* the fold's evaluator: f and the |.| sum at lattice nodes (lattice_node(), driver/lattice.c:30-34:
 * sf = EX[k + K]) with the FP64 kernel that rounds as written (the reference's fd); nodes outside the
 * lattice are clamped to its edge */
extern "C" int sqb_eval_points_impl(const sqb_graph_t *g, long n, const double *sf, int prec, int ab, double *f, double *abs_);
static int sym_nodes(void *ctx, long n, const int *k, double *f, double *ab){
    const Run &R = *(const Run*)ctx;
    std::vector<double> sf((size_t)n*R.D);
    for(long i = 0; i < n*R.D; i++){ const int kk = k[i] < -R.K ? -R.K : (k[i] > R.K ? R.K : k[i]); sf[i] = R.X[kk + R.K]; }
    return sqb_eval_points_impl(R.g, n, sf.data(), 0, 1, f, ab);
}

/* One integral's run, in phases: begin() (lattice, symmetry group, checkpoint, box_zero, grow and dilate,
 * or the resumed state), then per refinement level prep() (the level's sqb_level_t and next list) and
 * done() (the level's sums, its checkpoint, the lists swapped), then end() (the result).  sqb_hsum runs
 * them for one integral; sqb_hsum_group runs several integrals of one graph with their levels in shared
 * launches.  Every early return releases the device lists and the checkpoint (destructor). */
struct Integral {
    Run R; sqb_result_t *res = NULL; sqb_sym_t sym; VtabGuard vtg;
    int N = 0, top = 0, K = 0;
    double t0 = 0, tl0 = 0; unsigned long long l0 = 0;
    char ckfn[4096] = ""; sqb_ckpt_t ck; int resumed = 0;
    sqb_pt_t *dcur = NULL, *dnext = NULL; long ncur = 0, next_cap = 0;
    double Slev[16]; int nl = 0, esok = 0, lev0 = -1; long cnext = 0;
    sqb_acc_t acc0;
    double es1 = 0, es2 = 0, ah = 0, uu = 0;
    long nkeep0 = 0;
    double *dtab = NULL;                       /* this integral's tables on the device (group levels) */
    Integral(){ memset(&sym, 0, sizeof sym); memset(&ck, 0, sizeof ck); memset(&acc0, 0, sizeof acc0); }
    ~Integral(){ sqb_dev_free(dcur); sqb_dev_free(dnext); sqb_dev_free(dtab); sqb_ckpt_free(&ck); }
    Integral(const Integral &) = delete;
    Integral &operator=(const Integral &) = delete;

    /* 0: the levels follow; 1: finished at the top (zero integrand, or nothing to sum); -1: error */
    int begin(const char *graph, double h, int N_, double eps, int top_, const sqb_opts_t *opts, sqb_result_t *res_, int tables){
        res = res_; N = N_;
        memset(res, 0, sizeof *res);
        R.g = sqb_find_graph(graph);
        if(!R.g) FAIL("no graph %s in this build", graph);
        if(opts) R.o = *opts; else sqb_default_opts(&R.o);
        if(sqb_dev_init(R.o.device)) FAIL("device: %s", sqb_last_error());
        top = top_;
        if(top < 0){ top = 1; while(top < 2 && (1 << (top + 1))*h <= 3.0*(1 + 1e-9)) top++; }   /* driver/main.c:211-215 */
        R.D = R.g->D; R.h = h; R.eps = eps; R.top = top;
        if(R.D >= SQB_MAXD) FAIL("D=%d needs MAXD > 12", R.D);
        const int m = 1 << (top + 1); K = (N - 1)/2; K = ((K + m - 1)/m)*m;   /* driver/lattice.c:16 */
        if(K > 127) FAIL("N = %d gives K = %d; points are stored in 8 bits, so K <= 127 (N <= 255)", N, K);
        R.K = K;
        R.X.resize(2*K + 1); R.Wt.resize(2*K + 1);
        for(int k = -K; k <= K; k++){
            if(R.g->zlattice){ R.X[k + K] = k*h; R.Wt[k + K] = h; }
            else { R.X[k + K] = exp(k*h); R.Wt[k + K] = R.X[k + K]*h; }
        }
        if(sqb_dev_tables(R.X.data(), R.Wt.data(), K)) FAIL("device: %s", sqb_last_error());
        if(tables){
            dtab = (double*)sqb_dev_alloc(2*(2*K + 1)*sizeof(double));
            if(!dtab || sqb_dev_upload(dtab, R.X.data(), (2*K + 1)*sizeof(double)) ||
               sqb_dev_upload(dtab + 2*K + 1, R.Wt.data(), (2*K + 1)*sizeof(double))) FAIL("device copy of the lattice tables failed");
        }
        /* the symmetry fold's group (driver/sum.c:566-592), before the run's clock starts as there */
        sym.n = 1;
        res->sym_order = 1;
        if(R.o.predict > 0) R.vt = &vtg.t;
        if(R.o.sym && *R.o.sym){
            static thread_local int el[SQB_SYMG*SQB_MAXD];
            const int n = sqb_sym_find(R.D, sym_nodes, &R, R.o.sym, el, res->sym_desc, sizeof res->sym_desc, &res->sym_worst,
                                       res->sym_msg, sizeof res->sym_msg);
            if(n < 0) FAIL("symmetry search: device: %s", sqb_last_error());
            sym.n = n; res->sym_order = n;
            for(int e = 0; e < n; e++) for(int i = 0; i < SQB_MAXD; i++) sym.g[e][i] = (signed char)el[e*SQB_MAXD + i];
        }
        t0 = now();
        l0 = sqb_launch_count() + sqb_top_launches();
        { double a, b; long c; sqb_kernel_times(&a, &b, &c, 1); }
        /* a checkpoint of this run (same graph, h, eps, N, top, D, K) resumes it (driver/sum.c:596-606) */
        if(R.o.ckpt_every > 0){
            sqb_ckpt_name(ckfn, sizeof ckfn, R.o.ckpt_dir, R.g->name);
            const int lr = sqb_ckpt_load(ckfn, &ck);
            if(lr == 1 && !strcmp(ck.name, R.g->name) && ck.h == h && ck.eps == eps && ck.N == N && ck.top == top &&
               ck.dim == R.D && ck.k == K && ck.lev >= 0 && ck.lev < top && ck.next >= 0 && ck.next <= ck.ncur && ck.nl >= 1) resumed = 1;
            else {
                if(lr == 1) sqb_ckpt_free(&ck);
                memset(&ck, 0, sizeof ck);
                if(lr && R.o.verbose) fprintf(stderr, "# checkpoint %s is for a different run or damaged: ignored\n", ckfn);
            }
        }
        lev0 = top - 1;
        if(resumed){
            for(int i = 0; i < 3; i++) res->S[i] = NAN;
            res->nev = ck.nev; res->ref = ck.ref; res->prune = ck.prune; res->trunc = ck.trunc; res->kept_top = ck.kept_top;
            R.nq = ck.nq; res->abskipped = ck.cnt[1]; res->pskip = ck.cnt[0];
            if(R.vt && ck.vcap > 0 && ck.vs && sqb_vtab_upload(R.vt, ck.vs, ck.vcap, ck.vn, sqb_dev_stream()))
                FAIL("predictor: %s", sqb_vtab_error());
            nl = ck.nl; for(int i = 0; i < nl; i++) Slev[i] = ck.Slev[i];
            esok = ck.esok; lev0 = ck.lev; cnext = ck.next; t0 -= ck.t;
            ncur = ck.ncur;
            dcur = (sqb_pt_t*)sqb_dev_alloc((size_t)(ncur ? ncur : 1)*sizeof(sqb_pt_t));
            if(!dcur || (ncur && sqb_dev_upload(dcur, ck.cur, (size_t)ncur*sizeof(sqb_pt_t))))
                FAIL("device copy of the checkpoint's %ld cells failed", ncur);
            if(cnext > 0){         /* a level in progress: its partial sums carry on */
                acc0.S[0] = ck.s; acc0.A[0] = ck.a; acc0.drop[0] = ck.drop; acc0.u[0] = ck.u;
                acc0.b1[0] = ck.es[0]; acc0.b2[0] = ck.es[1]; acc0.ne = ck.ne; acc0.nq = ck.q;
            }
            if(R.o.verbose) fprintf(stderr, "# resuming %s from checkpoint: refine to step %dh, cell %ld of %ld\n",
                                    R.g->name, 1 << ck.lev, ck.next, ck.ncur);
            res->t_top = 0;
        } else {
            set_test(R, R.o.abserr0);
            int zero = 0;
            if(box_zero(R, top, &res->nev, &zero)) return -1;
            if(zero){ res->zero = 1; res->t = now() - t0; return 1; }
            GrowOut go;
            if(grow(R, top, eps*1e-3, &go, &dcur, &ncur)) return -1;
            if(vt_check(R, E_, sizeof E_)) return -1;
            res->nev += go.nev; res->ref = go.A; res->prune = go.drop;
            if(top == 0 && go.gshn) res->prune = fabs(go.gshs);
            if(go.A == 0){ res->t = now() - t0; res->nq = R.nq; res->unresdrop = R.unresdrop; return 1; }
            { double r = go.e2 > 0 ? go.e1/go.e2 : 0; res->trunc = (r > 0 && r < 1) ? go.e1*r/(1 - r) : go.e1; }
            for(int i = 0; i < 3; i++) res->S[i] = NAN;
            Slev[nl++] = go.S;
            res->kept_top = ncur;
            res->t_top = now() - t0;
            esok = R.D < SQB_MAXD && top > 0;
        }
        /* the levels on the device */
        set_test(R, fmax(R.o.abserr0, R.o.abrel*eps*res->ref));    /* driver/sum.c:651 */
        tl0 = now();
        return 0;
    }

    /* the level lev (lev0 >= lev >= 0): its sqb_level_t, the next level's list allocated */
    int prep(int lev, sqb_level_t *L, sqb_acc_t *acc){
        const int st = 1 << lev, last = lev == 0;
        /* resumed in mid-level: cells [cnext, ncur) remain, and the checkpoint's kept cells come first */
        nkeep0 = lev == lev0 ? ck.nnxt : 0;
        const long c0 = lev == lev0 ? cnext : 0;
        memset(L, 0, sizeof *L);
        L->g = R.g; L->cells = dcur + c0; L->ncell = ncur - c0; L->st = st; L->last = last;
        L->pw = pow(st, R.D); L->thr = R.eps*res->ref*1e-2; L->t = R.t; L->max_children = R.o.max_children;
        L->sym = &sym;
        L->X = dtab; L->Wt = dtab ? dtab + 2*K + 1 : NULL; L->K = K;
        /* the predictor: the level before the last stores its values, the last level uses them
         * (driver/sum.c:385, 739) */
        if(R.vt){
            L->vt = R.vt; L->vput = lev == 1; L->esok = esok;
            if(last) L->predict = R.o.predict;
            if(L->vput && sqb_vtab_reserve(R.vt, (ncur - c0) << R.D, sqb_dev_stream())) FAIL("predictor: %s", sqb_vtab_error());
        }
        if(!last){
            double want = (double)(ncur - c0)*(double)(1L << R.D) + nkeep0;
            double room = 0.35*MEMSHARE*(double)sqb_dev_total_bytes()/sizeof(sqb_pt_t);
            next_cap = (long)(want < room ? want : room) + 1;
            dnext = (sqb_pt_t*)sqb_dev_alloc(next_cap*sizeof(sqb_pt_t));
            if(!dnext) FAIL("device allocation of the next level (%ld cells) failed", next_cap);
            if(nkeep0 && (nkeep0 >= next_cap || sqb_dev_upload(dnext, ck.nxt, (size_t)nkeep0*sizeof(sqb_pt_t))))
                FAIL("device copy of the checkpoint's kept cells failed");
            L->next = dnext + nkeep0; L->next_cap = next_cap - nkeep0;
        }
        if(lev == lev0) *acc = acc0; else memset(acc, 0, sizeof *acc);
        return 0;
    }

    /* after the level's sums acc (nn kept children, ms device milliseconds): 0, -1, or SQB_CKPT_STOPPED */
    int done(int lev, const sqb_acc_t &acc, long nn, double ms){
        const int st = 1 << lev, last = lev == 0;
        if(acc.overflow) FAIL("level %d: %ld kept cells exceed the device list (%ld)", lev, nn, next_cap);
        nn += nkeep0;
        Slev[nl++] = ddv(acc.S);
        res->prune += ddv(acc.drop); res->nev += (long)acc.ne; R.nq += (long)acc.nq; R.unresdrop += (long)acc.unres;
        res->abskipped += (long)acc.skipped; res->pskip += (long)acc.pskip;
        if(vt_check(R, E_, sizeof E_)) return -1;
        if(res->nlev < 16){ res->lev_evals[res->nlev] = (long)acc.ne; res->lev_ms[res->nlev] = ms; res->nlev++; }
        if(last){ ah = ddv(acc.A); uu = ddv(acc.u); es1 = ddv(acc.b1); es2 = ddv(acc.b2); }
        if(R.o.verbose) fprintf(stderr, "# %s level step %dh: %ld cells, %llu evals, %llu fallback, %ld kept, %.1f ms\n",
                                R.g->name, st, ncur, acc.ne, acc.nq, nn, ms);
        if(R.o.ckpt_every > 0 && !last){
            /* the state between this level and the next, as the reference saves it (driver/sum.c:797-799) */
            std::vector<sqb_pt_t> host((size_t)nn);
            if(nn && sqb_dev_download(host.data(), dnext, (size_t)nn*sizeof(sqb_pt_t))) FAIL("device: %s", sqb_last_error());
            sqb_ckpt_t c; memset(&c, 0, sizeof c);
            snprintf(c.name, sizeof c.name, "%s", R.g->name);
            c.h = R.h; c.eps = R.eps; c.N = N; c.top = top; c.dim = R.D; c.k = K;
            c.lev = lev - 1; c.next = 0;
            c.s = Slev[nl - 1]; c.a = ddv(acc.A); c.drop = ddv(acc.drop); c.u = ddv(acc.u);
            c.ne = (long)acc.ne; c.q = (long)acc.nq;
            for(int i = 0; i < nl; i++) c.Slev[i] = Slev[i];
            c.nl = nl;
            c.ref = res->ref; c.prune = res->prune; c.trunc = res->trunc; c.t = now() - t0;
            c.nev = res->nev; c.nq = R.nq; c.kept_top = res->kept_top;
            c.ncur = nn; c.cur = (signed char*)host.data();
            c.cnt[0] = res->pskip; c.cnt[1] = res->abskipped; c.esok = esok;
            c.vsz = SQB_CKPT_VSLOT;
            /* the predictor's table goes with the checkpoint, so that a resumed run predicts as an unbroken
             * one (driver/sum.c:68-69) */
            std::vector<char> vs;
            if(R.vt && R.vt->tab){
                long vn = 0, full = 0;
                vs.resize((size_t)R.vt->cap*SQB_CKPT_VSLOT);
                if(sqb_vtab_counts(R.vt, &vn, &full, sqb_dev_stream()) || sqb_vtab_download(R.vt, vs.data(), sqb_dev_stream()))
                    FAIL("predictor: %s", sqb_vtab_error());
                c.vs = vs.data(); c.vcap = R.vt->cap; c.vn = vn;
            }
            if(sqb_ckpt_save(ckfn, &c) && R.o.verbose) fprintf(stderr, "# warning: could not write checkpoint %s\n", ckfn);
            if(R.o.ckpt_stop){
                snprintf(E_, sizeof E_, "stopped after the checkpoint %s (ckpt_stop)", ckfn);
                return SQB_CKPT_STOPPED;
            }
        }
        sqb_dev_free(dcur); dcur = dnext; dnext = NULL; ncur = last ? 0 : nn;
        return 0;
    }

    void end(){
        sqb_dev_free(dcur); dcur = NULL;
        if(R.o.ckpt_every > 0) remove(ckfn);          /* the graph is finished (driver/sum.c:804) */
        res->t_levels = now() - tl0;
        if(top > 0){ res->unres = sqrt(uu); res->Ah = ah; }
        else res->unres = R.u;            /* top = 0: the grow's sum of squares as it stands (driver/sum.c:795) */
        res->S[0] = Slev[nl - 1]; res->S[1] = nl > 1 ? Slev[nl - 2] : NAN; res->S[2] = nl > 2 ? Slev[nl - 3] : NAN;
        res->es1 = es1; res->es2 = es2; res->esok = esok;
        res->nq = R.nq; res->unresdrop = R.unresdrop;
        sqb_kernel_times(&res->f64_ms, &res->dd_ms, &res->f64_launches, 1);
        res->launches = (long)(sqb_launch_count() + sqb_top_launches() - l0);
        res->t = now() - t0;
    }
};

extern "C" int sqb_hsum(const char *graph, double h, int N, double eps, int top, const sqb_opts_t *opts, sqb_result_t *res){
    Integral I;
    const int b = I.begin(graph, h, N, eps, top, opts, res, 0);
    if(b) return b < 0 ? -1 : 0;
    for(int lev = I.lev0; lev >= 0; lev--){
        sqb_level_t L; sqb_acc_t acc;
        if(I.prep(lev, &L, &acc)) return -1;
        long nn = 0; double ms = 0;
        if(sqb_dev_level(&L, &acc, &nn, &ms)) FAIL("device: %s", sqb_last_error());
        const int rc = I.done(lev, acc, nn, ms);
        if(rc) return rc;
    }
    I.end();
    return 0;
}

/* Several integrals of one graph (e.g. one graph at several h), their refinement levels in shared launches:
 * the integrals' top levels run one after another on this thread's stream, then for lev from the highest
 * down to 0 one sqb_dev_level_multi over the integrals that have that level.  Each result is bit for bit
 * the one sqb_hsum gives alone; the level times (lev_ms) are those of the shared launches.  A group with a
 * checkpoint or the predictor runs its integrals one after another. */
extern "C" int sqb_hsum_group(const sqb_job_t *jobs, int n, const sqb_opts_t *opts, sqb_result_t *res, int *rcs){
    sqb_opts_t o; if(opts) o = *opts; else sqb_default_opts(&o);
    if(n <= 0) return 0;
    int fails = 0;
    bool seq = n == 1 || n > SQB_MAXINST || o.ckpt_every > 0 || o.predict > 0 || o.alldd || o.split == 1;
    for(int j = 1; j < n && !seq; j++) seq = strcmp(jobs[j].graph, jobs[0].graph) != 0;
    if(seq){
        for(int j = 0; j < n; j++){ rcs[j] = sqb_hsum(jobs[j].graph, jobs[j].h, jobs[j].N, jobs[j].eps, jobs[j].top, &o, &res[j]); fails += rcs[j] != 0; }
        return fails;
    }
    std::vector<Integral> I(n);
    std::vector<int> live(n, 0);
    int maxlev = -1;
    for(int j = 0; j < n; j++){
        rcs[j] = 0;
        const int b = I[j].begin(jobs[j].graph, jobs[j].h, jobs[j].N, jobs[j].eps, jobs[j].top, &o, &res[j], 1);
        if(b < 0){ rcs[j] = -1; fails++; continue; }
        if(b == 0){ live[j] = 1; if(I[j].lev0 > maxlev) maxlev = I[j].lev0; }
    }
    char err[512] = "";
    for(int lev = maxlev; lev >= 0; lev--){
        sqb_level_t L[SQB_MAXINST]; sqb_acc_t acc[SQB_MAXINST]; long nn[SQB_MAXINST]; int who[SQB_MAXINST], m = 0;
        for(int j = 0; j < n; j++){
            if(!live[j] || lev > I[j].lev0) continue;
            if(I[j].prep(lev, &L[m], &acc[m])){ rcs[j] = -1; fails++; live[j] = 0; if(!*err) snprintf(err, sizeof err, "%s: %s", jobs[j].graph, E_); continue; }
            who[m++] = j;
        }
        if(!m) continue;
        double ms = 0;
        if(sqb_dev_level_multi(L, m, acc, nn, &ms)){
            snprintf(E_, sizeof E_, "device: %s", sqb_last_error());
            for(int q = 0; q < m; q++){ rcs[who[q]] = -1; live[who[q]] = 0; fails++; }
            if(!*err) snprintf(err, sizeof err, "%s", E_);
            continue;
        }
        for(int q = 0; q < m; q++){
            const int j = who[q];
            const int rc = I[j].done(lev, acc[q], nn[q], ms);
            if(rc){ rcs[j] = rc; live[j] = 0; fails++; if(!*err) snprintf(err, sizeof err, "%s: %s", jobs[j].graph, E_); }
        }
    }
    for(int j = 0; j < n; j++) if(live[j]) I[j].end();
    if(fails && *err) snprintf(E_, sizeof E_, "%s", err);
    return fails;
}

/* pointwise kernel evaluation for parity checks */
extern "C" int sqb_eval_points(const char *graph, long n, const double *sf, int prec, int ab, double *f, double *abs_){
    const sqb_graph_t *g = sqb_find_graph(graph);
    if(!g) FAIL("no graph %s in this build", graph);
    if(sqb_dev_init(0)) FAIL("device: %s", sqb_last_error());
    if(sqb_eval_points_impl(g, n, sf, prec, ab, f, abs_)) FAIL("device: %s", sqb_last_error());
    return 0;
}
