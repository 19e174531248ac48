/* sym.cpp -- the group of the symmetry fold (driver/sum.c:21-46, 464-546, 566-592).
 *
 * A group G of axis permutations with f(k o g) = f(k): found automatically (symfind(): axes with the
 * same profile along lines through (1, ..., 1), the involutions that pair only such axes tried at one
 * generic node, the passing ones checked at 200 nodes and closed under composition, most axes moved
 * first) or given as involutions "p0,p1,...[;q0,...]" and checked the same way.  The reference's
 * searches evaluate one node at a time; here every phase is one batch of nodes handed to the caller's
 * evaluator (the device kernels), and the decisions are then taken in the reference's order, so the
 * group, its element order (which fixes the order of a kept orbit in the next level's list), the
 * description and the worst deviation are the reference's.
 *
 * The random nodes come from the C library's rand() stream after srand(12345) and srand(4242)
 * (driver/sum.c:468, 528), reproduced per call by sqb_rand.h. */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <string>
#include <vector>
#include "sqb_rt.h"
#include "sqb_rand.h"
#include "sincfeyn_b200.h"

namespace {

typedef SqbRand Rng;

struct Finder {
    int D;
    sqb_sym_eval_fn fn; void *ctx;
    int n = 1;                                  /* group order; g[0] the identity */
    int g[SQB_SYMG][SQB_MAXD];
    std::vector<int> k200;                      /* symcheck()'s 200 nodes (driver/sum.c:468-471) */
    std::vector<double> f200;
    bool have200 = false;
    std::string msg;

    Finder(int D_, sqb_sym_eval_fn f, void *c) : D(D_), fn(f), ctx(c) {
        memset(g, 0, sizeof g);
        for(int i = 0; i < SQB_MAXD; i++) g[0][i] = i;
    }
    int eval(const std::vector<int> &k, std::vector<double> &f, std::vector<double> &ab){
        const long m = (long)k.size()/D;
        f.assign(m, 0.0); ab.assign(m, 0.0);
        return m ? fn(ctx, m, k.data(), f.data(), ab.data()) : 0;
    }
    /* the 200 nodes and f there, once */
    int nodes200(){
        if(have200) return 0;
        Rng r(12345);
        k200.resize(200*D);
        for(int t = 0; t < 200; t++) for(int d = 0; d < D; d++) k200[t*D + d] = (r.next() % 9) - 4;
        std::vector<double> ab;
        if(eval(k200, f200, ab)) return -1;
        have200 = true;
        return 0;
    }
    /* symcheck() for several permutations at once: worst |f(k) - f(k o p)| / sum|terms|(k o p) */
    int check(const std::vector<std::vector<int>> &ps, std::vector<double> &worst){
        if(nodes200()) return -1;
        std::vector<int> ks(ps.size()*200*D);
        for(size_t c = 0; c < ps.size(); c++)
            for(int t = 0; t < 200; t++) for(int d = 0; d < D; d++) ks[(c*200 + t)*D + d] = k200[t*D + ps[c][d]];
        std::vector<double> f2, ab;
        if(eval(ks, f2, ab)) return -1;
        worst.assign(ps.size(), 0.0);
        for(size_t c = 0; c < ps.size(); c++)
            for(int t = 0; t < 200; t++){
                const double b = ab[c*200 + t];
                const double r = fabs(f200[t] - f2[c*200 + t])/(b > 0 ? b : 1);
                if(r > worst[c]) worst[c] = r;
            }
        return 0;
    }
    bool same(const int *a, const int *b) const { for(int i = 0; i < D; i++) if(a[i] != b[i]) return false; return true; }
    bool member(const int *p) const { for(int e = 0; e < n; e++) if(same(g[e], p)) return true; return false; }
    /* symadd(): add p and close under composition (products a o b with both indices running over the
     * growing list); false if p is already there or the group would pass SQB_SYMG elements */
    bool add(const int *p){
        if(member(p)) return false;
        static thread_local int G[SQB_SYMG][SQB_MAXD];
        memcpy(G, g, sizeof G);
        int m = n;
        memcpy(G[m++], p, sizeof G[0]);
        for(int a = 0; a < m; a++) for(int b = 0; b < m; b++){
            int c[SQB_MAXD] = {0};
            for(int i = 0; i < D; i++) c[i] = G[a][G[b][i]];
            bool dup = false;
            for(int e = 0; e < m && !dup; e++) dup = same(G[e], c);
            if(dup) continue;
            if(m == SQB_SYMG) return false;
            memcpy(G[m++], c, sizeof G[0]);
        }
        memcpy(g, G, sizeof g); n = m;
        return true;
    }
};

/* symenum()'s leaves in its order: involutions p pairing only axes of equal profile, p != identity;
 * at most 20001 of them (the reference stops after its 20001st try) */
struct Enum {
    int D; const int *grp; int tries = 0;
    std::vector<std::vector<int>> out; std::vector<int> moved;
    void run(int *p, int i, int mv){
        if(tries > 20000) return;
        while(i < D && p[i] >= 0) i++;
        if(i == D){
            if(!mv) return;
            tries++;
            out.emplace_back(p, p + D); moved.push_back(mv);
            return;
        }
        p[i] = i; run(p, i + 1, mv); p[i] = -1;
        for(int j = i + 1; j < D; j++) if(p[j] < 0 && grp[j] == grp[i]){
            p[i] = j; p[j] = i; run(p, i + 1, mv + 2); p[i] = p[j] = -1; }
    }
};

void appendf(char *desc, int nd, const char *fmt, ...) __attribute__((format(printf, 3, 4)));
void appendf(char *desc, int nd, const char *fmt, ...){
    const int o = (int)strlen(desc); if(o >= nd - 1) return;
    va_list ap; va_start(ap, fmt); vsnprintf(desc + o, nd - o, fmt, ap); va_end(ap);
}

/* symfind(), driver/sum.c:520-546 */
int find_auto(Finder &F, char *desc, int nd, double *worst){
    const int D = F.D;
    static const int T[3] = {-3, 2, 5};
    std::vector<int> k(3*D*D);
    for(int i = 0; i < D; i++) for(int t = 0; t < 3; t++){
        int *q = &k[(i*3 + t)*D];
        for(int d = 0; d < D; d++) q[d] = 1;
        q[i] += T[t];
    }
    std::vector<double> sig, ab;
    if(F.eval(k, sig, ab)) return -1;
    double amax = 0;
    for(double a : ab) if(a > amax) amax = a;
    if(!(amax > 0)) return 0;
    int grp[SQB_MAXD], ng = 0;
    for(int i = 0; i < D; i++){
        grp[i] = -1;
        for(int j = 0; j < i && grp[i] < 0; j++){
            bool same = true;
            for(int t = 0; t < 3; t++) if(fabs(sig[i*3 + t] - sig[j*3 + t]) > 1e-11*amax) same = false;
            if(same) grp[i] = grp[j];
        }
        if(grp[i] < 0) grp[i] = ng++;
    }
    if(ng == D) return 0;                               /* no two axes alike */
    /* the generic node and the candidates' images of it */
    Rng r(4242);
    int k1[SQB_MAXD];
    for(int d = 0; d < D; d++) k1[d] = (r.next() % 9) - 4;
    Enum E; E.D = D; E.grp = grp;
    int p[SQB_MAXD]; for(int i = 0; i < D; i++) p[i] = -1;
    E.run(p, 0, 0);
    std::vector<int> ks((E.out.size() + 1)*D);
    for(int d = 0; d < D; d++) ks[d] = k1[d];
    for(size_t c = 0; c < E.out.size(); c++) for(int d = 0; d < D; d++) ks[(c + 1)*D + d] = k1[E.out[c][d]];
    std::vector<double> fk, abk;
    if(F.eval(ks, fk, abk)) return -1;
    const double f0 = fk[0], ab0 = abk[0];
    std::vector<std::vector<int>> cand; std::vector<int> cm;
    for(size_t c = 0; c < E.out.size() && cand.size() < 64; c++)
        if(fabs(fk[c + 1] - f0) <= 1e-11*ab0){ cand.push_back(E.out[c]); cm.push_back(E.moved[c]); }
    if(cand.empty()) return 0;
    std::vector<double> w;
    if(F.check(cand, w)) return -1;
    for(int m = D; m > 0; m--) for(size_t c = 0; c < cand.size(); c++){
        if(cm[c] != m || F.member(cand[c].data())) continue;
        if(w[c] >= 1e-10) continue;
        if(!F.add(cand[c].data())) continue;
        if(w[c] > *worst) *worst = w[c];
        for(int i = 0; i < D && (int)strlen(desc) < nd - 8; i++)
            appendf(desc, nd, "%s%d", i ? "," : (desc[0] ? "; " : ""), cand[c][i]);
    }
    return 0;
}

/* SINCQED_SYM="p0,p1,...[;q0,...]": involutions, each checked (driver/sum.c:573-586) */
int find_manual(Finder &F, const char *spec, char *desc, int nd, double *worst){
    const int D = F.D;
    const char *q = spec;
    while(*q){
        int P[SQB_MAXD] = {0}, n = 0; const char *q0 = q; char *r;
        while(n < D){ long v = strtol(q, &r, 10); if(r == q) break; P[n++] = (int)v; q = r; while(*q == ',' || *q == ' ') q++; }
        bool ok = n == D && (!*q || *q == ';'), id = true;
        for(int i = 0; ok && i < D; i++){ if(P[i] < 0 || P[i] >= D || P[P[i]] != i) ok = false; if(P[i] != i) id = false; }
        const int len = (int)(q - q0);
        char line[512];
        if(!ok || id){
            snprintf(line, sizeof line, "SINCQED_SYM entry \"%.*s\" is not a non-trivial involution of the %d axes; ignored", len, q0, D);
            F.msg += line; F.msg += "\n";
            while(*q && *q != ';') q++;
        } else {
            std::vector<std::vector<int>> one(1, std::vector<int>(P, P + D)); std::vector<double> w;
            if(F.check(one, w)) return -1;
            if(w[0] >= 1e-10){
                snprintf(line, sizeof line, "SINCQED_SYM entry \"%.*s\": max |f(k)-f(k sigma)|/sum|terms| %.1e, NOT SYMMETRIC: ignored", len, q0, w[0]);
                F.msg += line; F.msg += "\n";
            } else if(F.add(P)){
                if(w[0] > *worst) *worst = w[0];
                appendf(desc, nd, "%s%.*s", desc[0] ? "; " : "", len, q0);
            }
        }
        while(*q == ';' || *q == ' ') q++;
    }
    return 0;
}

}  // namespace

/* The fold's group for a graph of D axes; fn(ctx, n, k, f, ab) evaluates f and the |.| sum at n lattice
 * nodes k[i*D + d] (Sinc variables EX[k + K]).  spec: NULL, "", "0" or "off" = no fold; "auto" = search;
 * else the involutions to check.  On return: elems[e*12 + i] for e < order (element 0 the identity),
 * desc the generators accepted ("0,2,1,4,3; ..."), *worst their largest deviation, msg the entries that
 * were refused (one per line).  Returns the order (1: no fold) or -1 if the evaluator failed. */
extern "C" int sqb_sym_find(int D, sqb_sym_eval_fn fn, void *ctx, const char *spec, int *elems, char *desc, int ndesc,
                            double *worst, char *msg, int nmsg){
    if(desc && ndesc > 0) desc[0] = 0;
    if(msg && nmsg > 0) msg[0] = 0;
    *worst = 0;
    if(D < 1 || D > SQB_MAXD) return -1;
    for(int e = 0; e < SQB_SYMG; e++) for(int i = 0; i < SQB_MAXD; i++) elems[e*SQB_MAXD + i] = e ? 0 : i;
    if(!spec || !*spec || !strcmp(spec, "0") || !strcmp(spec, "off")) return 1;
    Finder F(D, fn, ctx);
    char dbuf[1024] = "";
    const int rc = strcmp(spec, "auto") ? find_manual(F, spec, dbuf, sizeof dbuf, worst) : find_auto(F, dbuf, sizeof dbuf, worst);
    if(rc) return -1;
    for(int e = 0; e < F.n; e++) for(int i = 0; i < SQB_MAXD; i++) elems[e*SQB_MAXD + i] = i < D ? F.g[e][i] : 0;
    if(desc && ndesc > 0) snprintf(desc, ndesc, "%s", dbuf);
    if(msg && nmsg > 0) snprintf(msg, nmsg, "%s", F.msg.c_str());
    return F.n;
}
