/* Test infrastructure: a serial CPU restatement of the reference's hierarchical Sinc sum, the checker
 * of the evaluator's host logic (never part of it).  It calls the reference's own kernels (graph_t, built
 * by oracle/Makefile without FP contraction) and restates, one function per reference routine, what the
 * reference does around them, in the order the reference sums:
 *
 *   lattice        driver/lattice.c:13-34
 *   finish/qvalue  driver/eval.c:25-61      (per-point tests, double-double fallback)
 *   box_zero       driver/sum.c:346-359
 *   grow           driver/sumkey.h:126-461  (serially: one table of every evaluated point, the next
 *                                            frontier in (kept point, axis, sign) order, final
 *                                            threshold, shadow-tier flood fill)
 *   dilate         driver/sumkey.h:20-90    (axis neighbours, flags merged, key order)
 *   levels         driver/sum.c:642-799     (children in cell order, Neumaier block sums over blocks of
 *                                            2^18 >> D cells, kept children with their flags)
 * Symmetry fold, predictor, checkpoints, histograms and dumps are not restated (the evaluator's point
 * set is the unfolded one, as the reference's GPU build, driver/sum.c:571).
 *
 *   sq_oracle h N eps top GRAPH...   ->  one line per graph: name value S_2h evals quad kept_top prune
 */
#include "sq.h"
#include <vector>
#include <algorithm>
#include <unordered_set>
#include <unordered_map>
#include <stdint.h>

__thread int SQ_AB = 1;

static const graph_t *G; static int D, KK; static double HH;   /* graph, dimension, half-width, step */
static std::vector<double> EXT;
static double ABS_ERR = 1e-15;
static const double ABSERR0_ = 1e-15, ABREL_ = 1e-3, NEARF_ = 1e-3, DDSLACK_ = 1;
static long NQ, UNRES; static double U;

/* driver/lattice.c:13-19 */
static void lattice(double h, int N, int top){
    HH = h; D = G->D; int m = 1 << (top + 1); KK = (N - 1)/2; KK = ((KK + m - 1)/m)*m;
    EXT.assign(2*KK + 1, 0); for(int k = -KK; k <= KK; k++) EXT[k + KK] = exp(k*HH);
}
/* driver/lattice.c:30-34 */
static void node(const int *k, double *sf, double *w){ double ww = 1; for(int i = 0; i < D; i++){ sf[i] = EXT[k[i] + KK]; ww *= sf[i]*HH; } *w = ww; }
/* driver/eval.c:25-30 */
static double qvalue(double vq, double abq, double w, double *u){
    double e = abq*w*QEPS; if(!(e*16 <= ABS_ERR)) *u += isfinite(e) ? e*e : 0;
    double v = isfinite(vq) ? vq*w : 0;
    if(!(e <= fabs(v))){ UNRES++; return 0; }
    return v;
}
/* driver/eval.c:33-61 (leafx + finish) */
static double leaf(const int *k, int skip, int *near, double *u){
    double sf[MAXD], w, ab; node(k, sf, &w);
    if(skip) SQ_AB = 0;
    double v = G->fd(sf, &ab); SQ_AB = 1;
    *near = 0;
    if(skip){ v *= w; return isfinite(v) ? v : 0; }
    double bnd = ab*w*16*DBL_EPSILON/DDSLACK_;
    if(!(bnd <= NEARF_*ABS_ERR)) *near = 1;
    if(!(bnd <= ABS_ERR)){
        QREAL sq[MAXD], abq; for(int i = 0; i < D; i++) sq[i] = (QREAL)sf[i];
        QREAL vq = G->fq(sq, &abq); NQ++;
        return qvalue((double)vq, (double)abq, w, u);
    }
    v *= w; return isfinite(v) ? v : 0;
}
/* driver/sum.c:18-20 */
struct ks_t { double s = 0, c = 0; void add(double x){ double t = s + x; if(fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s; s = t; } double val() const { return s + c; } };

struct pt { int k[MAXD]; int fl; };
static uint64_t keyof(const int *k, int st, uint64_t W){ uint64_t y = 1; for(int i = 0; i < D; i++) y = y*W + (uint64_t)(k[i]/st + KK/st); return y; }

/* driver/sum.c:346-359 */
static int box_zero(int lev){
    int st = 1 << lev, W = 2*(KK/st) + 1; double u = 0;
    for(long i = 0; i <= 4096; i++){
        int k[MAXD] = {0}; unsigned long long y = 0x9E3779B97F4A7C15ULL*(unsigned long long)(i + 1);
        if(i) for(int d = 0; d < D; d++){ y ^= y >> 29; y *= 0xBF58476D1CE4E5B9ULL; y ^= y >> 32; k[d] = ((int)(y % (unsigned long long)W) - KK/st)*st; }
        int nr; long nq0 = NQ; double v = leaf(k, 0, &nr, &u); NQ = nq0;
        if(v != 0) return 0;
    }
    return 1;
}

struct res { double S0, S1, prune, ref; long nev, nq, kept; };

int run(double h, int N, double eps, int top, res *R){
    memset(R, 0, sizeof *R); NQ = 0; UNRES = 0; U = 0;
    lattice(h, N, top); ABS_ERR = ABSERR0_;
    if(box_zero(top)){ R->nev = 4097; return 0; }
    /* ---- grow at step 2^top, driver/sumkey.h:130-461 ---- */
    const int st = 1 << top; const uint64_t W = 2*(KK/st) + 1; const double pw = pow(st, D), eps_rel = eps*1e-3;
    std::vector<uint64_t> P(D); { uint64_t p = 1; for(int i = D - 1; i >= 0; i--){ P[i] = p; p *= W; } }
    std::unordered_set<uint64_t> seen;
    std::vector<pt> fr(1), nx, keep; memset(&fr[0], 0, sizeof fr[0]); seen.insert(keyof(fr[0].k, st, W));
    std::vector<double> kv; ks_t ks; double a = 0, dr = 0, u = 0; long ne = 0;
    while(!fr.empty()){
        std::vector<double> v(fr.size()); std::vector<int> nr(fr.size());
        for(size_t i = 0; i < fr.size(); i++) v[i] = leaf(fr[i].k, 0, &nr[i], &u);
        ne += fr.size();
        for(size_t i = 0; i < fr.size(); i++){ ks.add(v[i]*pw); a += fabs(v[i])*pw; }
        const double thr = eps_rel*a;
        std::vector<size_t> kj;
        for(size_t i = 0; i < fr.size(); i++){
            if(fabs(v[i]) >= thr){ kj.push_back(i); kv.push_back(fabs(v[i])); pt p = fr[i]; p.fl = !nr[i]; keep.push_back(p); }
            else dr += fabs(v[i])*pw;
        }
        nx.clear();
        for(size_t j : kj) for(int d = 0; d < D; d++) for(int sg = -1; sg <= 1; sg += 2){
            pt p = fr[j]; p.k[d] += st*sg; p.fl = 0;
            if(p.k[d] > KK || p.k[d] < -KK) continue;
            if(seen.insert(keyof(p.k, st, W)).second) nx.push_back(p);
        }
        fr.swap(nx);
    }
    const double thr0 = eps_rel*a;
    { size_t m = 0; for(size_t i = 0; i < keep.size(); i++){ if(kv[i] >= thr0){ kv[m] = kv[i]; keep[m++] = keep[i]; } else dr += kv[i]*pw; }
      keep.resize(m); kv.resize(m); }
    /* shadow tiers, driver/sumkey.h:402-444 */
    { std::unordered_map<uint64_t, size_t> idx; for(size_t i = 0; i < keep.size(); i++) idx[keyof(keep[i].k, st, W)] = i;
      std::vector<int> tr(keep.size(), 0);
      for(int t = 1; t <= 2; t++){
          const double lim = (t == 1 ? 10 : 100)*thr0; std::vector<size_t> cu, nw;
          for(size_t i = 0; i < keep.size(); i++){ int z = 1; for(int d = 0; d < D; d++) if(keep[i].k[d]) z = 0; if(z && kv[i] >= lim){ tr[i] = t; cu.push_back(i); } }
          while(!cu.empty()){
              nw.clear();
              for(size_t i : cu) for(int d = 0; d < D; d++) for(int sg = -1; sg <= 1; sg += 2){
                  int k2[MAXD]; memcpy(k2, keep[i].k, sizeof k2); k2[d] += st*sg; if(k2[d] > KK || k2[d] < -KK) continue;
                  auto f = idx.find(keyof(k2, st, W)); if(f == idx.end()) continue;
                  size_t j = f->second; if(kv[j] >= lim && tr[j] < t){ tr[j] = t; nw.push_back(j); } }
              cu.swap(nw);
          }
      }
      for(size_t i = 0; i < keep.size(); i++) keep[i].fl = (keep[i].fl & 1) | (tr[i] << 1); }
    R->ref = a; R->prune = dr; R->nev = ne;
    double Slev[16]; int nl = 0; Slev[nl++] = ks.val();
    /* ---- dilate, driver/sumkey.h:20-90 ---- */
    std::vector<pt> cur;
    { std::unordered_map<uint64_t, int> fl;
      for(const pt &c : keep) for(int j = -1; j < D; j++) for(int sg = -1; sg <= 1; sg += 2){
          if(j < 0 && sg > 0) continue;
          pt p = c; if(j >= 0){ p.k[j] += st*sg; if(p.k[j] > KK || p.k[j] < -KK) continue; }
          uint64_t y = keyof(p.k, st, W); auto f = fl.find(y);
          if(f == fl.end()) fl[y] = c.fl;
          else f->second = ((f->second & c.fl) & 1) | (std::max(f->second >> 1, c.fl >> 1) << 1); }
      std::vector<uint64_t> ys; for(auto &e : fl) ys.push_back(e.first); std::sort(ys.begin(), ys.end());
      for(uint64_t y0 : ys){ pt p; memset(&p, 0, sizeof p); uint64_t y = y0;
          for(int i = D - 1; i >= 0; i--){ p.k[i] = ((int)(y % W) - KK/st)*st; y /= W; }
          p.fl = fl[y0]; cur.push_back(p); } }
    R->kept = cur.size();
    /* ---- levels, driver/sum.c:642-799 ---- */
    ABS_ERR = fmax(ABSERR0_, ABREL_*eps*R->ref);
    const long B = ((1L << 18) >> D) < 1 ? 1 : ((1L << 18) >> D);
    for(int lev = top - 1; lev >= 0; lev--){
        const int s = 1 << lev, last = lev == 0; const double pwl = pow(s, D), thr = eps*R->ref*1e-2;
        double Ss = 0, KC = 0, drop = 0, ul = 0; long nel = 0;
        std::vector<pt> nxt;
        for(size_t c0 = 0; c0 < cur.size(); c0 += B){
            ks_t bs;
            for(size_t c = c0; c < cur.size() && c < c0 + B; c++){
                const int psk = cur[c].fl & 1, te = cur[c].fl >> 1;
                for(int b = 0; b < (1 << D); b++){
                    pt q; memset(&q, 0, sizeof q); int ok = 1;
                    for(int i = 0; i < D; i++){ q.k[i] = cur[c].k[i] - (((b >> i) & 1) ? s : 0); if(q.k[i] < -KK) ok = 0; }
                    if(!ok) continue;
                    int nr; double v = leaf(q.k, psk, &nr, &ul); nel++;
                    bs.add(v*pwl);
                    if(!last){ if(fabs(v) >= thr){ int tv = (fabs(v) >= 10*thr) + (fabs(v) >= 100*thr);
                            q.fl = (psk || !nr) | ((te < tv ? te : tv) << 1); nxt.push_back(q); }
                        else drop += fabs(v)*pwl; }
                }
            }
            ks_t t; t.s = Ss; t.c = KC; t.add(bs.val()); Ss = t.s; KC = t.c;   /* kblock, driver/sum.c:77-81 */
        }
        Ss += KC;
        Slev[nl++] = Ss; R->prune += drop; R->nev += nel;
        if(last) U = ul;
        cur.swap(nxt);
    }
    R->S0 = Slev[nl - 1]; R->S1 = nl > 1 ? Slev[nl - 2] : NAN; R->nq = NQ;
    return 0;
}

int main(int argc, char **argv){
    if(argc < 6){ fprintf(stderr, "usage: sq_oracle h N eps top GRAPH...\n"); return 1; }
    register_graphs();
    double h = atof(argv[1]), eps = atof(argv[3]); int N = atoi(argv[2]), top = atoi(argv[4]);
    for(int a = 5; a < argc; a++){
        G = find(argv[a]); if(!G){ fprintf(stderr, "no graph %s\n", argv[a]); return 2; }
        res R; run(h, N, eps, top, &R);
        printf("%s %+.17e %+.17e %ld %ld %ld %.6e\n", G->name, G->weight*R.S0, G->weight*R.S1, R.nev, R.nq, R.kept, G->weight*R.prune);
    }
    return 0;
}
