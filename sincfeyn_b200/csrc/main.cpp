/* main.cpp -- the `sincqed` command line of the evaluator, the drop-in for the reference's
 * `sincqed list | run h N [eps] [top] GRAPH...` (driver/main.c:174-253).
 *
 * Graph selection (names, Volkov strings, groups), the default top, the N adjustment note, the
 * per-graph line, the results file (same columns, driver/main.c:66-73 and :226) and the environment
 * settings that reach the hot path follow the reference.  SQB_ALLDD=1 runs the all-double-double form;
 * SQB_DEVICE picks the CUDA device. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <time.h>
#include <stdarg.h>
#include <vector>
#include <string>
#include "sincfeyn_b200.h"

/* exact and known values of the reference's registry (driver/graphs.c:31-41), keyed by Volkov string */
struct ref_t { const char *volkov; double val, err; const char *src; };
static const ref_t REFS[] = {
    {"3; 1-4, 2-5", -0.46764544609361365, 0, "exact 1/6+13pi^2/36-5pi^2ln2/6+5z3/4 (crossed)"},
    {"3; 1-5, 2-4",  0.77747802228274215, 0, "exact 11/48+pi^2/18 (ladder)"},
    {"2; 1-4, 3-5", -0.064020941344682816, 0, "exact -55/24+pi^2/18+pi^2ln2/3-z3/2 (corner, PSLQ)"},
    {"2; 1-5, 3-4", -0.58997802228274215, 0, "exact -1/24-pi^2/18 (SE, PSLQ)"},
    {"3; 1-6, 2-5, 4-7", -0.334695, 5e-7, "analytic, 6 digits"},
    {"VP: 1-loop vertex + Pi2", 0.015687421859103, 0, "exact 119/36-pi^2/3"},
    {"VP: 2; 1-3 +Pi2(1-3)+Pi2(1-3)+Pi2(1-3)", 0.000876865858890, 0, "1D integral (mpmath)"},
    {"LbL (6 orderings)", 0.3710052921, 1e-10, "analytic (electron loop)"},
    {NULL, 0, 0, NULL}
};
static const ref_t *findref(const char *v){ for(int i = 0; REFS[i].volkov; i++) if(!strcmp(REFS[i].volkov, v)) return &REFS[i]; return NULL; }

/* group selectors, driver/graphs.c:15-29 */
static int selected(const char *name, const char *volkov, int L, const char *s){
    if(!strcmp(s, name) || !strcmp(s, volkov)) return 1;
    if(!strcmp(s, "all2")) return L == 2;
    if(!strcmp(s, "all3")) return L == 3 && strncmp(name, "w3_", 3);
    if(!strcmp(s, "all4")) return L == 4;
    if(!strcmp(s, "q3"))   return !strncmp(name, "g3_", 3) && strcmp(name, "g3_lbl");
    if(!strcmp(s, "vp3"))  return !strncmp(name, "v3_", 3);
    if(!strcmp(s, "vp4"))  return !strncmp(name, "v4_", 3) || !strncmp(name, "w4_", 3);
    if(!strcmp(s, "lbl4")) return !strncmp(name, "l4_", 3);
    if(!strcmp(s, "pi6"))  return !strncmp(name, "w4_p6", 5);
    if(!strcmp(s, "lbl"))  return !strcmp(name, "g3_lbl");
    if(!strcmp(s, "synth")) return !strncmp(name, "syn_", 4);   /* the seeded synthetic integrands (no graph) */
    return 0;
}
static int isnum(const char *s){ char *e; strtod(s, &e); return e != s && *e == 0; }

static FILE *LOGF, *RESF;
static void say(const char *fmt, ...){
    va_list ap; va_start(ap, fmt); vprintf(fmt, ap); va_end(ap); fflush(stdout);
    if(LOGF){ va_start(ap, fmt); vfprintf(LOGF, fmt, ap); va_end(ap); fflush(LOGF); }
}

int main(int argc, char **argv){
    sqb_opts_t o; sqb_default_opts(&o);
    const char *e;
    if((e = getenv("G2_ABSERR"))) o.abserr0 = atof(e);
    if((e = getenv("SINCQED_ABREL"))) o.abrel = atof(e);
    if((e = getenv("SINCQED_ABSKIP"))) o.abskip = atoi(e);
    if((e = getenv("SINCQED_ABCHECK"))) o.abcheck = atoi(e);
    if((e = getenv("SINCQED_NEARF"))) o.nearf = atof(e);
    if((e = getenv("SINCQED_DDSLACK"))) o.ddslack = atof(e);
    if((e = getenv("SINCQED_DROPUNRES"))) o.dropunres = atoi(e);
    if((e = getenv("SINCQED_GROWSKIP"))) o.growskip = atoi(e);
    if((e = getenv("SQB_ALLDD"))) o.alldd = atoi(e);
    if((e = getenv("SQB_DEVICE"))) o.device = atoi(e);
    if((e = getenv("SQB_VERBOSE"))) o.verbose = atoi(e);
    if((e = getenv("SQB_FMA"))) o.fma = atoi(e);
    if((e = getenv("SQB_SPLIT"))) o.split = atoi(e);
    o.sym = getenv("SINCQED_SYM");     /* unset: no fold, as the reference's GPU build (driver/sum.c:571) */
    if((e = getenv("SINCQED_PREDICT"))) o.predict = atof(e);
    /* checkpoints at every level end, on by default as in the reference (driver/main.c:28,184) */
    o.ckpt_every = 600;
    if((e = getenv("SINCQED_CKPT"))) o.ckpt_every = atof(e);
    o.ckpt_dir = getenv("SINCQED_CKPT_DIR");
    const int NG = sqb_graph_count();
    if(argc < 2 || !strcmp(argv[1], "list")){
        printf("%d graphs (one per mirror pair; w = mirror weight), precision fallback double-double on the GPU\n", NG);
        for(int i = 0; i < NG; i++){ int info[6]; const char *n = sqb_graph_name(i); sqb_graph_info(n, info);
            printf("  %-8s L=%d  %-22s D=%d w=%d\n", n, info[0], sqb_graph_volkov(n), info[1], info[2]); }
        printf("usage: %s run h N [eps] [top] GRAPH... | scale GRAPH [kappa] [seed]\n", argv[0]);
        return 0;
    }
    /* the scaling test (driver/main.c:192-199), on the device */
    if(!strcmp(argv[1], "scale")){
        if(argc < 3) return 1;
        const double kap = argc > 3 ? atof(argv[3]) : 24; const unsigned seed = argc > 4 ? atoi(argv[4]) : 1;
        const int E = getenv("SCALE_E") ? atoi(getenv("SCALE_E")) : 1;
        int rc = 0;
        for(int i = 0; i < NG; i++){
            int info[6]; const char *n = sqb_graph_name(i); sqb_graph_info(n, info);
            const char *volkov = sqb_graph_volkov(n);
            if(!selected(n, volkov, info[0], argv[2])) continue;
            sqb_scale_result_t r;
            const int k = sqb_scale_test(n, kap, seed, E, &r);
            if(k == 1){ printf("%-6s %-22s (no scale test for VP graphs)\n", n, volkov); continue; }
            if(k < 0){ fprintf(stderr, "sincqed: %s\n", sqb_error()); rc = 2; continue; }
            for(int j = 0; j < r.slow && j < 12; j++){
                printf("  slow direction e=(");
                for(int q = 0; q < r.n; q++) if(q != r.fixed) printf("%+d", r.listed_e[j][q]);
                printf(")  |g| at kappa/3,2/3,1: %.3e %.3e %.3e\n", r.listed_g[j][0], r.listed_g[j][1], r.listed_g[j][2]);
            }
            printf("%-6s %-22s scale test kappa=%g: %ld directions, %d slow (ratio>0.3), worst ratio %.3g (dir %ld: e=(",
                   n, volkov, kap, r.ndir, r.slow, r.worst, r.worst_dir);
            for(int q = 0; q < r.n; q++) if(q != r.fixed) printf("%+d", r.worst_e[q]);
            printf(") |g| %.2e %.2e %.2e)\n", r.worst_g[0], r.worst_g[1], r.worst_g[2]);
            fflush(stdout);
        }
        return rc;
    }
    if(strcmp(argv[1], "run")){ fprintf(stderr, "unknown command %s\n", argv[1]); return 1; }
    if(argc < 5){ fprintf(stderr, "run h N [eps] [top] GRAPH...\n"); return 1; }
    const double h = atof(argv[2]); const int N = atoi(argv[3]); int a = 4;
    double eps = 1e-11; int top = -1;
    if(a < argc && isnum(argv[a])) eps = atof(argv[a++]);
    if(a < argc && isnum(argv[a])) top = atoi(argv[a++]);
    if(top < 0){
        const double ts = getenv("SINCQED_TOPSTEP") ? atof(getenv("SINCQED_TOPSTEP")) : 3.0;
        top = 1; while(top < 2 && (1 << (top + 1))*h <= ts*(1 + 1e-9)) top++;
    }
    const char *lf = getenv("SINCQED_LOG") ? getenv("SINCQED_LOG") : "sincqed.log";
    const char *rf = getenv("SINCQED_RESULTS") ? getenv("SINCQED_RESULTS") : "sincqed_results.txt";
    if(*lf && strcmp(lf, "-")) LOGF = fopen(lf, "a");
    if(*rf && strcmp(rf, "-")){
        FILE *t = fopen(rf, "r"); int fresh = !t; if(t) fclose(t);
        RESF = fopen(rf, "a");
        if(RESF && fresh) fprintf(RESF, "# name     volkov                       L D w      h    N      eps top  value                  err       disc     prune    trunc    round    S_2h            evals        time_s  ref                    diff\n");
    }
    /* selection in command-line order, without repeats (driver/main.c:156-168) */
    std::vector<std::string> sel;
    for(int b = a; b < argc; b++){
        int hit = 0;
        for(int i = 0; i < NG; i++){
            int info[6]; const char *n = sqb_graph_name(i); sqb_graph_info(n, info);
            if(!selected(n, sqb_graph_volkov(n), info[0], argv[b])) continue;
            hit = 1; int dup = 0; for(auto &s : sel) dup |= s == n;
            if(!dup) sel.push_back(n);
        }
        if(!hit) fprintf(stderr, "# no graph matches %s in this build\n", argv[b]);
    }
    time_t now = time(NULL); char tb[32]; strftime(tb, sizeof tb, "%Y-%m-%d %H:%M:%S", localtime(&now));
    std::string cmd; for(int i = 0; i < argc; i++){ cmd += argv[i]; cmd += ' '; }
    say("# sincqed %s: %s\n", tb, cmd.c_str());
    say("# h=%g N=%d eps=%g top=%d precision=%s  graphs=%d  device=%s\n", h, N, eps, top,
        o.alldd ? "double-double (all points)" : "FP64 + double-double fallback", (int)sel.size(), "cuda");
    { int m = 1 << (top + 1), K0 = (N - 1)/2, K1 = ((K0 + m - 1)/m)*m;
      if(K1 != K0) say("# note: N=%d adjusted to N=%d (half-width must be a multiple of 2^(top+1)=%d); range |z| <= %g\n", N, 2*K1 + 1, m, K1*h);
      else say("# range |z| <= %g\n", K1*h);
      if(RESF) fprintf(RESF, "# %s  %s\n# window |z| <= %g\n", tb, cmd.c_str(), K1*h); }
    double tot = 0, toterr = 0, toterr2 = 0; int rc = 0;
    for(size_t j = 0; j < sel.size(); j++){
        const char *name = sel[j].c_str(); int info[6]; sqb_graph_info(name, info);
        const int L = info[0], D = info[1], w = info[2]; const char *volkov = sqb_graph_volkov(name);
        sqb_result_t R;
        if(sqb_hsum(name, h, N, eps, top, &o, &R)){ fprintf(stderr, "sincqed: %s: %s\n", name, sqb_error()); rc = 2; continue; }
        for(const char *m = R.sym_msg; *m; ){
            const char *nl = strchr(m, '\n'); const int len = nl ? (int)(nl - m) : (int)strlen(m);
            say("# %s: %.*s\n", name, len, m); m += len + (nl ? 1 : 0);
        }
        if(R.sym_order > 1)
            say("# %s: symmetry fold sigma=%s (group of order %d), max |f(k)-f(k sigma)|/sum|terms| over 200 nodes %.1e\n",
                name, R.sym_desc, R.sym_order, R.sym_worst);
        if(R.zero) say("# %s: integrand is exactly zero at 4097 probe nodes; reported as zero without a scan\n", name);
        const double v = w*R.S[0], d2 = fabs(R.S[1] - R.S[0]);
        const double disc = R.Ah > 0 ? 2*d2*d2/R.Ah : 0;
        const double err = w*(disc + R.prune + R.trunc + R.unres);
        char lv[64] = "";
        if(isfinite(R.S[1])) snprintf(lv, sizeof lv, "  |S2h-Sh| %.1e", w*d2);
        if(isfinite(R.S[2])) snprintf(lv + strlen(lv), sizeof lv - strlen(lv), "  S_4h %+.6f", w*R.S[2]);
        say("%-7s %-22s D=%d w=%d  %+.12f  err %.2e (disc %.1e prune %.1e trunc %.1e round %.1e)%s  evals %ld quad %ld kept %ld  %.1fs",
            name, volkov, D, w, v, err, w*disc, w*R.prune, w*R.trunc, w*R.unres, lv, R.nev, R.nq, R.kept_top, R.t);
        const ref_t *r = findref(volkov);
        if(r) say("  ref %+.12f (%s) diff %+.2e", r->val, r->src, v - r->val);
        say("\n");
        if(o.abskip) say("# %s: %ld of %ld evaluations skipped the |.| sums (no fallback check)\n", name, R.abskipped, R.nev);
        if(R.unresdrop) say("# WARNING %s: %ld points unresolved even in double-double (eps*sum|terms| > |value|, not one digit left) %s; their bound is in the round column\n",
                            name, R.unresdrop, o.dropunres ? "counted as 0 (SINCQED_DROPUNRES=0 keeps them)" : "kept as they came out");
        if(R.esok){ double d1 = w*(R.S[0] - R.es1), dd2 = w*(R.es1 - R.es2), rr = d1 != 0 ? dd2/d1 : 0;
            say("# %s eps extrapolation: eps*10 would change the value by %+.3e, eps*100 by a further %+.3e (ratio %.2f)", name, -d1, -dd2, rr);
            if(rr > 1.5) say("; pruning loss left at eps ~ %+.2e (add to the value)\n", d1/(rr - 1)); else say("\n"); }
        if(o.predict > 0) say("# %s predictor alpha %g: skipped %ld final-level points\n", name, o.predict, R.pskip);
        say("# %s timing: top level %.2fs on the host, levels %.2fs", name, R.t_top, R.t_levels);
        for(int l = 0; l < R.nlev; l++) say("%s%ld evals %.1f ms", l ? ", " : " (", R.lev_evals[l], R.lev_ms[l]);
        say("%s\n", R.nlev ? ")" : "");
        if(RESF){
            fprintf(RESF, "%-8s %-28s %d %d %d %5.3f %4d %8.1e %d %+.15e %.3e %.2e %.2e %.2e %.2e ",
                    name, volkov, L, D, w, h, 2*(((N - 1)/2 + (1 << (top + 1)) - 1)/(1 << (top + 1))*(1 << (top + 1))) + 1,
                    eps, top, v, err, w*disc, w*R.prune, w*R.trunc, w*R.unres);
            if(isfinite(R.S[1])) fprintf(RESF, "%+.8e", w*R.S[1]); else fprintf(RESF, "%15s", "-");
            fprintf(RESF, " %12ld %9.1f", R.nev, R.t);
            if(r) fprintf(RESF, " %+.15e %+.3e", r->val, v - r->val); else fprintf(RESF, " %22s %10s", "-", "-");
            fprintf(RESF, "\n"); fflush(RESF);
        }
        tot += v; toterr += err; toterr2 += err*err;
    }
    if(sel.size() > 1){
        say("# sum of %d graphs: %+.12f  err %.2e (linear sum)  %.2e (in quadrature)\n", (int)sel.size(), tot, toterr, sqrt(toterr2));
        if(RESF) fprintf(RESF, "# SUM %d graphs  %+.15e  err %.3e (linear)  %.3e (quadrature)\n", (int)sel.size(), tot, toterr, sqrt(toterr2));
    }
    if(LOGF) fclose(LOGF);
    if(RESF) fclose(RESF);
    return rc;
}
