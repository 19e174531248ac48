/* sqkern.cuh -- the evaluation kernels, instantiated once per graph by the generated translation
 * unit (kgen output included after this header, then SQ_GRAPH(...) below).
 *
 * One thread per lattice point.  A point is a node (k given) or child b of a cell (k_d - st*bit_d(b),
 * in the order of prep() in the reference, driver/sum.c:405-408; children below the box, k_d < -K,
 * are not points).  The per-coordinate tables X[k+K] (the integration variable, s = e^{kh}) and
 * Wt[k+K] (its weight factor s*h) sit in shared memory; the weight is accumulated in coordinate order
 * as lattice_node() does (driver/lattice.c:30-34), so it rounds identically.
 *
 * FP64 pass (sqb_k_f64): f and the |.| sum in double.  Raw mode returns f*w and ab*w (the reference's
 * GPU plug-in contract, driver/gpu_kernel.h:22-36).  Test mode applies the reference's per-point tests
 * (finish(), driver/eval.c:33-53): skipped points keep f*w; otherwise the bound ab*w*16*eps/DDSLACK sets
 * the near flag and, above ABSERR, queues the point for the double-double pass.
 * DD pass (sqb_k_dd): the queued points (or all of them) in double-double, with qvalue()'s round
 * column and unresolved-point rule (driver/eval.c:25-30). */
#pragma once
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include "sqdd.cuh"
#include "sqb_internal.h"
#include "sqscale.cuh"
#include "sqorbit.cuh"

#ifndef SQG_NS
#define SQG_NS(n) sqg_##n                    /* the graph's namespace (sqgf_<name> in the contracted unit) */
#endif
#define SQ_TABLE static __constant__ const
#define SQ_FUNC __device__
#ifndef SQ_FUNC_K
#define SQ_FUNC_K __device__                    /* FP64 class: point functions (pt_, vp_, helpers); a graph's
                                                   unit may define it __forceinline__ */
#endif
#define SQ_CHUNK __device__ __forceinline__      /* FP64: chunk arguments stay in registers */
#define SQ_CHUNK_DD __device__ __noinline__     /* double-double: real calls bound the compile */
#define RABS(x) sq_rabs(x)
#define SQ_EXP(x) sq_exp(x)
#define SQ_LOG(x) sq_log(x)

#ifndef SQB_BLOCK
#define SQB_BLOCK 128
#endif
#ifndef SQB_MINB
#define SQB_MINB 1            /* FP64 kernel: resident blocks per SM the register allocation must allow */
#endif
#ifndef SQB_LEVEL_KERNEL
#ifdef SQB_FMA_TU
#define SQB_LEVEL_KERNEL 1    /* the contracted unit: a level kernel beside the general one, both calling the point
                                 function (sqb_fcall); the exact unit keeps one kernel with the function inlined */
#else
#define SQB_LEVEL_KERNEL 0
#endif
#endif
#ifndef SQB_SWEEPS
#define SQB_SWEEPS 1          /* level kernel: 2 = two sweeps over a batch's tiles, the children of cells that skip
                                 the |.| sums first, then the others, so that the CTAs on an SM run one form of a
                                 point function at a time (a large integrand's two forms do not fit the
                                 instruction caches together); the reduce kernel then sums every tile */
#endif
#ifndef SQB_FUSE
#define SQB_FUSE 1            /* FP64 kernel: level mode (tile sums in shared memory) compiled in; a kernel
                                 that spills its registers is built without it, keeping L1 for its stack */
#endif
#define SQB_QEPS 4.93e-32   /* double-double epsilon of the fallback's error model (driver/common.h:8) */
#ifndef SQB_TABLE_GLOBAL
#define SQB_TABLE_GLOBAL 0    /* FP64 pass: 1 = the lattice tables read through the read-only data cache instead of
                                 from the CTA's shared-memory copy */
#endif
#if SQB_TABLE_GLOBAL
#define SQB_TAB(p, j) __ldg((p) + (j))
#else
#define SQB_TAB(p, j) (p)[j]
#endif

/* The per-integral fields of a launch (sqb_inst_t) sit in shared memory: every thread of a CTA works on
 * one integral at a time.  A launch over one batch (ninst = 0) has one record, made from its own fields;
 * a multi-instance launch (ninst >= 1) has one per integral, with their tables side by side. */
__device__ __forceinline__ void sqb_inst_of(const sqb_eval_t &a, sqb_inst_t *I){
    I->pts = a.pts; I->n = a.n; I->child0 = 0; I->st = a.st; I->K = a.K; I->toff = 0; I->fused = 1;
    I->last = a.last; I->pw = a.pw; I->thr = a.thr; I->abserr = a.abserr; I->near_thr = a.near_thr;
    I->X = a.X; I->Wt = a.Wt;
}
/* the instance of global child index i (ninst >= 1): the last one whose range starts at or before i */
__device__ __forceinline__ int sqb_inst_at(const sqb_eval_t &a, long i){
    int k = 0;
    for(int q = 1; q < a.ninst; q++) if(a.inst[q].child0 <= i) k = q;
    return k;
}
/* shared-memory words of the tables of a launch: 2(2K+1) per integral */
__host__ __device__ __forceinline__ int sqb_table_words(const sqb_eval_t &a){
    if(a.ninst <= 0) return 2*(2*a.K + 1);
    int w = 0;
    for(int q = 0; q < a.ninst; q++) w += 2*(2*a.inst[q].K + 1);
    return w;
}

/* coordinates and weight of point il of integral I (ig: its index in the launch, the same for one batch);
 * returns 0 for a child below the box, a child the predictor leaves out or, under a symmetry fold, a child
 * that is not the minimum of its orbit (driver/sum.c:405-416), else the point's multiplicity (the orbit
 * size; 1 without a fold) */
template<int D, bool ORB = true, int LV = 0>
__device__ __forceinline__ int sqb_point(const sqb_eval_t &a, const sqb_inst_t &I, const double *sX, const double *sW,
                                         long il, long ig, long *cell, double *sf, double *w){
    long c; int b;
    const bool cells = LV || a.cells;           /* the level kernel: cells of int8 coordinates */
    if(cells){ c = il >> D; b = (int)(il & ((1L << D) - 1)); } else { c = il; b = 0; }
    *cell = c;
    if(!LV && a.sfin){
#pragma unroll
        for(int d = 0; d < D; d++) sf[d] = a.sfin[ig*D + d];
        *w = 1.0;
        return 1;
    }
    double ww = 1.0; bool in = true;
    int kk[D];
    const int K = I.K, st = I.st;
    if(LV || a.esize == 1){
        const signed char *p = (const signed char*)I.pts + c*(long)a.stride;
#pragma unroll
        for(int d = 0; d < D; d++){
            int kd = p[d] - (((b >> d) & 1) ? st : 0);
            kk[d] = kd;
            if(kd < -K){ in = false; kd = -K; }
            sf[d] = SQB_TAB(sX, kd + K); ww = ww*SQB_TAB(sW, kd + K);
        }
    } else {
        const short *p = (const short*)I.pts + c*(long)a.stride;
#pragma unroll
        for(int d = 0; d < D; d++){
            int kd = p[d] - (((b >> d) & 1) ? st : 0);
            kk[d] = kd;
            if(kd < -K){ in = false; kd = -K; }
            sf[d] = SQB_TAB(sX, kd + K); ww = ww*SQB_TAB(sW, kd + K);
        }
    }
    *w = ww;
    if(!in) return 0;
    if(a.cfl && (a.cfl[ig] & 1)) return 0;          /* left out by the predictor */
    if constexpr(!ORB) return 1;               /* list mode: the select pass has the orbit weight */
    return cells && a.sym.n > 1 ? sqb_orbit<D>(a.sym, kk) : 1;
}

template<int D>
__device__ __forceinline__ int sqb_skip(const sqb_eval_t &a, const sqb_inst_t &I, long c){
    if(a.skip) return a.skip[c];
    if(a.flag_at >= 0 && a.abskip){
        int fl = a.esize == 1 ? ((const signed char*)I.pts)[c*(long)a.stride + a.flag_at]
                              : ((const short*)I.pts)[c*(long)a.stride + a.flag_at];
        return fl & 1;
    }
    return 0;
}

/* the launch's tables into shared memory (X then the weight factor Wt = X H when a batch has no Wt) and
 * the integral records: one batch (ninst = 0) fills sI[0] */
__device__ __forceinline__ void sqb_tables(const sqb_eval_t &a, double *sm, sqb_inst_t *sI){
    if(a.ninst <= 0){
        const int nt = 2*a.K + 1;
        for(int j = threadIdx.x; j < nt; j += blockDim.x){ sm[j] = a.X[j]; sm[nt + j] = a.Wt ? a.Wt[j] : a.X[j]*a.H; }
        if(threadIdx.x == 0) sqb_inst_of(a, &sI[0]);
    } else {
        for(int q = 0; q < a.ninst; q++){
            const sqb_inst_t &I = a.inst[q];
            const int nt = 2*I.K + 1;
            for(int j = threadIdx.x; j < nt; j += blockDim.x){ sm[I.toff + j] = I.X[j]; sm[I.toff + nt + j] = I.Wt[j]; }
        }
        if(threadIdx.x < a.ninst) sI[threadIdx.x] = a.inst[threadIdx.x];
    }
    __syncthreads();
}

/* the per-point tests of finish() (driver/eval.c:33-53) on the FP64 value fw = f w and |.| sum abw = ab w
 * of point i: skipped points keep fw; otherwise the bound abw 16 eps / DDSLACK sets the near flag and,
 * above ABSERR, queues the point for the double-double pass (value 0 until then).  Writes v[i] and
 * stt[i]; returns the value */
__device__ __forceinline__ double sqb_point_test(const sqb_eval_t &a, const sqb_inst_t &I, long i, int sk, bool noab,
                                                 double fw, double abw, bool *fallback){
    unsigned char s = SQB_PRESENT | (sk ? SQB_SKIPPED : 0);
    double v;
    *fallback = false;
    if(noab) v = isfinite(fw) ? fw : 0.0;
    else {
        const double bnd = abw*16*DBL_EPSILON/a.ddslack;
        if(!(bnd <= I.near_thr)) s |= SQB_NEAR;
        if(!(bnd <= I.abserr)){
            s |= SQB_FALLBACK; v = 0.0; *fallback = true;
            const unsigned long long q = atomicAdd(a.nfb, 1ULL);
            if((long)q < a.fbcap) a.fb[q] = i;
        } else v = isfinite(fw) ? fw : 0.0;
    }
    a.v[i] = v; a.stt[i] = s;
    return v;
}

/* the tile's sums in level mode: thread t's running sums sit in shared memory (column t), out of the
 * registers that the integrand needs; at the tile's end warp 0 adds the columns in a fixed order */
#if SQB_FUSE
static_assert(SQB_BLOCK == SQB_TILE_THREADS, "the tile sums have one column per thread of the FP64 kernel's block");
#endif

__device__ __forceinline__ void sqb_acc_dd(double (*x)[SQB_BLOCK], int t, double y){
    const sqdd z = sqdd_add_d(sqdd(x[0][t], x[1][t]), y);
    x[0][t] = z.hi; x[1][t] = z.lo;
}

/* warp 0: the tile's sums in a fixed order (lane l adds columns l, l+32, l+64, l+96, then a shuffle
 * tree), written to part[tile]; the block's threads have synchronised before */
__device__ __forceinline__ void sqb_tile_flush(const sqb_eval_t &a, sqb_tile_acc &ta, long tile){
    if(threadIdx.x >= 32) return;
    const int l = threadIdx.x;
    sqdd S, b1, b2; double A = 0, dr = 0; unsigned ne = 0, nsk = 0, keep = 0;
    for(int q = l; q < SQB_BLOCK; q += 32){
        S = S + sqdd(ta.S[0][q], ta.S[1][q]); b1 = b1 + sqdd(ta.b1[0][q], ta.b1[1][q]); b2 = b2 + sqdd(ta.b2[0][q], ta.b2[1][q]);
        A += ta.A[q]; dr += ta.dr[q]; ne += ta.ne[q]; nsk += ta.nsk[q]; keep += ta.keep[q];
    }
    sqdd Ad(A), dd(dr);
    for(int off = 16; off; off >>= 1){
        S = S + sqdd(__shfl_down_sync(0xffffffffu, S.hi, off), __shfl_down_sync(0xffffffffu, S.lo, off));
        Ad = Ad + sqdd(__shfl_down_sync(0xffffffffu, Ad.hi, off), __shfl_down_sync(0xffffffffu, Ad.lo, off));
        dd = dd + sqdd(__shfl_down_sync(0xffffffffu, dd.hi, off), __shfl_down_sync(0xffffffffu, dd.lo, off));
        b1 = b1 + sqdd(__shfl_down_sync(0xffffffffu, b1.hi, off), __shfl_down_sync(0xffffffffu, b1.lo, off));
        b2 = b2 + sqdd(__shfl_down_sync(0xffffffffu, b2.hi, off), __shfl_down_sync(0xffffffffu, b2.lo, off));
        ne += __shfl_down_sync(0xffffffffu, ne, off); nsk += __shfl_down_sync(0xffffffffu, nsk, off);
        keep += __shfl_down_sync(0xffffffffu, keep, off);
    }
    if(l == 0){
        sqb_part_t p;
        p.S[0] = S.hi; p.S[1] = S.lo; p.A[0] = Ad.hi; p.A[1] = Ad.lo; p.drop[0] = dd.hi; p.drop[1] = dd.lo;
        p.b1[0] = b1.hi; p.b1[1] = b1.lo; p.b2[0] = b2.hi; p.b2[1] = b2.lo; p.u[0] = 0; p.u[1] = 0;
        p.ne = ne; p.nq = 0; p.unres = 0; p.skipped = nsk;
        a.part[tile] = p; a.tkeep[tile] = keep; a.tfb[tile] = 0;
    }
}

/* The point function as a real call (contracted unit): its two forms (without and with the |.| sums) are
 * compiled as functions apart from the callers' loop state, so that the level kernel and the general one
 * share them instead of each inlining both (measured on the B200: as fast as the inlined function in the
 * level kernel). */
template<int D> struct sqb_pt { double s[D]; };
struct sqb_fab { double f, ab; };
template<class F, int D, int AB>
__device__ __noinline__ sqb_fab sqb_fcall(const sqb_pt<D> p){
    double sf[D];
#pragma unroll
    for(int d = 0; d < D; d++) sf[d] = p.s[d];
    sqb_fab r; r.ab = 0; r.f = F::template f<double, AB>(sf, &r.ab);
    return r;
}

/* The FP64 pass.  The CTAs take tiles of consecutive points in turn: tile b, b + gridDim.x, ... of one
 * batch, or, in a multi-instance launch, the next tile of the device counter queue (the tile's integral
 * from its position); SQB_TILE points per tile in level mode and in multi-instance launches, SQB_BLOCK
 * otherwise.  In a tile, thread t evaluates points t, t + SQB_BLOCK, ... (consecutive threads, consecutive
 * points).
 * In level mode (a.part) each CTA also sums the tiles of its integrals that it is asked to (sqb_inst_t
 * fused): the children that need no fallback add v*pw and the rest into the thread's column of shared
 * memory; a tile with a fallback point, or of an integral the reduce kernel sums, is only flagged (a.tfb),
 * and the reduce kernel sums it after the double-double pass.
 * LV = 1 is the level kernel: the same pass compiled for level batches alone (cells of int8 coordinates,
 * tiles from the device queue, no list, no plain-form output), which leaves the other modes' code out of
 * the kernel that runs almost every point (measured 3-4 % faster on the three-loop graphs); with
 * SQB_SWEEPS = 2 it takes every tile twice, first for the children of cells that skip the |.| sums, then
 * for the others.  LV = 0 runs every other launch. */
template<class F, int D, int LV = 0>
__global__ void __launch_bounds__(SQB_BLOCK, SQB_MINB) sqb_k_f64(const __grid_constant__ sqb_eval_t a){
    extern __shared__ double sqb_sm[];
    __shared__ sqb_inst_t sI[SQB_MAXINST];
    __shared__ long s_tile;
    __shared__ int s_k;
#if SQB_FUSE
    /* the tile sums' columns follow the tables in dynamic shared memory (level launches only) */
    sqb_tile_acc &ta = *(sqb_tile_acc*)(sqb_sm + sqb_table_words(a));
    const bool lvl = LV || a.part != NULL;
#else
    const bool lvl = false;
#endif
    constexpr int NSW = LV ? SQB_SWEEPS : 1;
    sqb_tables(a, sqb_sm, sI);
    const bool multi = LV || a.ninst > 0;
    const bool list = !LV && a.sel;
    const long n1 = multi ? 0 : (a.cells ? (a.n << D) : a.n);      /* one batch: its points */
    const long tl = (lvl || multi) ? SQB_TILE : SQB_BLOCK;          /* other modes: one point per thread per step */
    const long nsel = list ? (long)*a.nsel : 0;                     /* list mode (one integral, queue): its entries */
    const long ntiles = list ? (nsel + tl - 1)/tl : multi ? a.ntile : (n1 + tl - 1)/tl;
    const int t = threadIdx.x;
    long q = blockIdx.x;                                            /* the work item: sweep*ntiles + tile */
    if(multi){ if(t == 0) s_tile = (long)atomicAdd(a.queue, 1ULL); __syncthreads(); q = s_tile; }
    while(q < NSW*ntiles){
        const int sweep = NSW > 1 ? (int)(q/ntiles) : 0;
        const long tile = NSW > 1 ? q - sweep*ntiles : q;
        int k = 0;
        if(multi){ if(t == 0) s_k = sqb_inst_at(a, tile*tl); __syncthreads(); k = s_k; }
        const sqb_inst_t &I = sI[k];
#if SQB_TABLE_GLOBAL
        const double *sX = I.X, *sW = I.Wt;
#else
        const double *sX = sqb_sm + I.toff, *sW = sX + (2*I.K + 1);
#endif
        const long base = multi ? tile*tl - I.child0 : tile*tl;     /* the tile's first point in its integral */
        const long n = multi ? ((LV || a.cells) ? (I.n << D) : I.n) : n1;
        const long off = multi ? I.child0 : 0;                       /* global index = local index + off */
#if SQB_FUSE
        const bool tsum = lvl && I.fused && !list && NSW == 1;
        if(tsum){
            ta.S[0][t] = ta.S[1][t] = ta.A[t] = ta.dr[t] = ta.b1[0][t] = ta.b1[1][t] = ta.b2[0][t] = ta.b2[1][t] = 0;
            ta.ne[t] = ta.nsk[t] = ta.keep[t] = 0;
            if(t == 0) ta.fb = 0;
            __syncthreads();
        }
#else
        const bool tsum = false;
#endif
        for(int j = 0; j < tl/SQB_BLOCK; j++){
            long il, i; int mw;
            long c; double sf[D], w;
            if(list){
                const long e_ = tile*tl + (long)j*SQB_BLOCK + t;
                if(e_ >= nsel) break;
                const unsigned long long e = a.sel[e_];
                il = i = (long)(e & ((1ULL << SQB_SEL_SHIFT) - 1));
                sqb_point<D, false, LV>(a, I, sX, sW, il, i, &c, sf, &w);
                mw = (int)(e >> SQB_SEL_SHIFT);
            } else {
                il = base + (long)j*SQB_BLOCK + t; i = il + off;
                if(il >= n) break;
                /* two sweeps: this child only in its cell's sweep (0: skips the |.| sums, 1: the others) */
                if(NSW > 1 && (sqb_skip<D>(a, I, il >> D) ? 0 : 1) != sweep) continue;
                mw = sqb_point<D, true, LV>(a, I, sX, sW, il, i, &c, sf, &w);
            }
            if(!mw){
                a.v[i] = 0;
                if(!LV && a.raw) a.ab[i] = 0; else a.stt[i] = 0;
                continue;
            }
            const int sk = sqb_skip<D>(a, I, c);
            const bool noab = sk && !a.abcheck;
            double ab = 0, f;
#if SQB_LEVEL_KERNEL
            {
                sqb_pt<D> p;
#pragma unroll
                for(int d = 0; d < D; d++) p.s[d] = sf[d];
                const sqb_fab r = noab ? sqb_fcall<F, D, 0>(p) : sqb_fcall<F, D, 1>(p);
                f = r.f; ab = r.ab;
            }
#else
            if(noab) f = F::template f<double, 0>(sf, &ab);
            else     f = F::template f<double, 1>(sf, &ab);
#endif
            const double fw = f*w;
            if(!LV && a.raw){ a.v[i] = fw; a.ab[i] = ab*w; continue; }
            bool fallback;
            const double v = sqb_point_test(a, I, i, sk, noab, fw, ab*w, &fallback);
#if SQB_FUSE
            if(tsum){
                if(fallback){ ta.fb = 1; continue; }
                /* a folded point stands for its orbit: (mw v) pw and mw |v| (driver/sum.c:734-745) */
                const double m = (double)mw, vp = (m*v)*I.pw, av = fabs(v);
                sqb_acc_dd(ta.S, t, vp); ta.A[t] += m*av; ta.ne[t]++; ta.nsk[t] += sk ? 1 : 0;
                if(I.last){
                    const int te = a.cfl ? (a.cfl[i] >> 1) & 3
                                         : (((const signed char*)I.pts)[c*(long)a.stride + a.flag_at] >> 1) & 3;
                    if(te >= 1) sqb_acc_dd(ta.b1, t, vp);
                    if(te >= 2) sqb_acc_dd(ta.b2, t, vp);
                } else if(av >= I.thr) ta.keep[t] += mw;
                else ta.dr[t] += (m*av)*I.pw;
            }
#else
            (void)fallback;
#endif
        }
#if SQB_FUSE
        if(tsum){
            __syncthreads();
            if(ta.fb){ if(t == 0) a.tfb[tile] = 1; }
            else sqb_tile_flush(a, ta, tile);
            __syncthreads();
        } else
#endif
        if(multi && a.tfb && !list && t == 0) a.tfb[tile] = 1;       /* summed by the reduce kernel */
        if(multi){
            __syncthreads();                                          /* every thread has read s_tile, s_k */
            if(t == 0) s_tile = (long)atomicAdd(a.queue, 1ULL);
            __syncthreads();
            q = s_tile;
        } else q += gridDim.x;
    }
}

template<class F, int D>
__global__ void __launch_bounds__(SQB_BLOCK) sqb_k_dd(const __grid_constant__ sqb_dd_t a){
    extern __shared__ double sqb_sm[];
    __shared__ sqb_inst_t sI[SQB_MAXINST];
    const sqb_eval_t &e = a.e;
    sqb_tables(e, sqb_sm, sI);
    const bool multi = e.ninst > 0;
    long n;
    if(a.all) n = multi ? e.ntile*SQB_TILE : (e.cells ? (e.n << D) : e.n);
    else { n = (long)*a.nlist; if(n > a.listcap) n = a.listcap; }
    for(long j = blockIdx.x*(long)blockDim.x + threadIdx.x; j < n; j += (long)gridDim.x*blockDim.x){
        const long i = a.all ? j : a.list[j];
        const int k = multi ? sqb_inst_at(e, i) : 0;
        const sqb_inst_t &I = sI[k];
        const double *sX = sqb_sm + I.toff, *sW = sX + (2*I.K + 1);
        const long il = i - I.child0;
        if(multi && il >= (e.cells ? (I.n << D) : I.n)) continue;    /* a tile's padding: no point */
        long c; double sf[D], w;
        if(!sqb_point<D>(e, I, sX, sW, il, i, &c, sf, &w)){ e.v[i] = 0; e.stt[i] = 0; a.uu[i] = 0; continue; }
        sqdd sq[D], abq;
#pragma unroll
        for(int d = 0; d < D; d++) sq[d] = sqdd(sf[d]);
        const sqdd vq = F::template f<sqdd, 1>(sq, &abq);
        if(e.raw){ e.v[i] = vq.hi; e.vlo[i] = vq.lo; e.ab[i] = abq.hi; e.ablo[i] = abq.lo; continue; }
        const double vqd = vq.value(), abqd = abq.value();
        /* qvalue(), driver/eval.c:25-30 */
        const double ee = abqd*w*SQB_QEPS;
        const double u = !(ee*16 <= I.abserr) ? (isfinite(ee) ? ee*ee : 0.0) : 0.0;
        double v = isfinite(vqd) ? vqd*w : 0.0;
        unsigned char s;
        if(a.all){
            /* the all-double-double form: the near flag from the double-double |.| sum */
            s = SQB_PRESENT | SQB_FALLBACK | (sqb_skip<D>(e, I, c) ? SQB_SKIPPED : 0);
            if(!(abqd*w*16*DBL_EPSILON/e.ddslack <= I.near_thr)) s |= SQB_NEAR;
        } else s = e.stt[i];
        if(!(ee <= fabs(v))){ s |= SQB_UNRES; if(a.dropunres) v = 0.0; }
        e.v[i] = v; e.stt[i] = s; a.uu[i] = u;
    }
}

/* A graph whose point function is a flat sum of independent forest nodes (kgen.split_plan: g3_lbl) can
 * run the FP64 pass of a level batch as NP passes and a final one.  Pass P evaluates the nodes of group P
 * at every point and adds their contributions to the point's running (tot, tota) in tt[i], ta[i]; the
 * final pass applies f_'s own arithmetic to them and the tests of finish().  The operations and their
 * order are those of the single function, so the values are the same; each pass's code is a fraction of
 * the whole, which fits the instruction caches (the single kernel of g3_lbl waits on instruction fetch). */
template<class F, int D, int P>
__global__ void __launch_bounds__(SQB_BLOCK) sqb_k_part(const sqb_eval_t a, double *tt, double *ta){
    extern __shared__ double sqb_sm[];
    __shared__ sqb_inst_t sI[1];
    sqb_tables(a, sqb_sm, sI);                       /* one batch (ninst = 0) */
    const sqb_inst_t &I = sI[0];
    const double *sX = sqb_sm, *sW = sqb_sm + (2*a.K + 1);
    const long n = a.cells ? (a.n << D) : a.n;
    for(long i = blockIdx.x*(long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x*blockDim.x){
        long c; double sf[D], w;
        if(!sqb_point<D>(a, I, sX, sW, i, i, &c, sf, &w)) continue;
        const int sk = sqb_skip<D>(a, I, c);
        double T = P ? tt[i] : 0.0, A = P ? ta[i] : 0.0;
        if(sk && !a.abcheck) F::template part<P, 0>(sf, &T, &A);
        else                 F::template part<P, 1>(sf, &T, &A);
        tt[i] = T; ta[i] = A;
    }
}

template<class F, int D>
__global__ void __launch_bounds__(SQB_BLOCK) sqb_k_fin(const sqb_eval_t a, const double *tt, const double *ta){
    extern __shared__ double sqb_sm[];
    __shared__ sqb_inst_t sI[1];
    sqb_tables(a, sqb_sm, sI);                       /* one batch (ninst = 0) */
    const sqb_inst_t &I = sI[0];
    const double *sX = sqb_sm, *sW = sqb_sm + (2*a.K + 1);
    const long n = a.cells ? (a.n << D) : a.n;
    for(long i = blockIdx.x*(long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x*blockDim.x){
        long c; double sf[D], w;
        if(!sqb_point<D>(a, I, sX, sW, i, i, &c, sf, &w)){ a.v[i] = 0; a.stt[i] = 0; continue; }
        const int sk = sqb_skip<D>(a, I, c);
        const bool noab = sk && !a.abcheck;
        double ab = 0, f;
        if(noab) f = F::template fin<0>(sf, tt[i], ta[i], &ab);
        else     f = F::template fin<1>(sf, tt[i], ta[i], &ab);
        bool fallback;
        sqb_point_test(a, I, i, sk, noab, f*w, ab*w, &fallback);
    }
}

/* launch pass P (P < NP) or the final pass (P == NP) */
template<class F, int D, int NP>
static void sqb_split_launch(int P, const sqb_eval_t *a, double *tt, double *ta, int grid, int block, size_t smem, cudaStream_t st){
    static_assert(NP >= 1 && NP <= 16, "at most sixteen passes have launchers");
#define SQB_PASS_(Q) if constexpr((Q) < NP) if(P == (Q)){ sqb_k_part<F, D, (Q) < NP ? (Q) : 0><<<grid, block, smem, st>>>(*a, tt, ta); return; }
    SQB_PASS_(0) SQB_PASS_(1) SQB_PASS_(2) SQB_PASS_(3) SQB_PASS_(4) SQB_PASS_(5) SQB_PASS_(6) SQB_PASS_(7)
    SQB_PASS_(8) SQB_PASS_(9) SQB_PASS_(10) SQB_PASS_(11) SQB_PASS_(12) SQB_PASS_(13) SQB_PASS_(14) SQB_PASS_(15)
#undef SQB_PASS_
    sqb_k_fin<F, D><<<grid, block, smem, st>>>(*a, tt, ta);
}
template<class K_>
static int sqb_attr_of(K_ kernel, int block, size_t smem, sqb_kattr_t *o){
    cudaFuncAttributes fa; int nb = 0;
    if(cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) return 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, block, smem) != cudaSuccess) return 0;
    o->regs = fa.numRegs; o->local_bytes = (int)fa.localSizeBytes; o->max_threads = fa.maxThreadsPerBlock;
    o->blocks_per_sm = nb; o->fused = 0; o->sweeps = 1; return 1;
}
/* an FP64 (or dd) kernel's attributes; lv: the level kernel, which sums level tiles itself unless it sweeps
 * twice */
template<class K_>
static int sqb_f64_attr(K_ kernel, int lv, int block, size_t smem, sqb_kattr_t *o){
    if(!sqb_attr_of(kernel, block, smem, o)) return 0;
    o->fused = SQB_FUSE && !(lv && SQB_SWEEPS > 1);
    o->sweeps = lv ? SQB_SWEEPS : 1;
    return 1;
}
template<class F, int D, int NP>
static int sqb_split_attr(int P, int block, size_t smem, sqb_kattr_t *o){
    static_assert(NP >= 1 && NP <= 16, "at most sixteen passes have launchers");
#define SQB_PASS_(Q) if constexpr((Q) < NP) if(P == (Q)) return sqb_attr_of(sqb_k_part<F, D, (Q) < NP ? (Q) : 0>, block, smem, o);
    SQB_PASS_(0) SQB_PASS_(1) SQB_PASS_(2) SQB_PASS_(3) SQB_PASS_(4) SQB_PASS_(5) SQB_PASS_(6) SQB_PASS_(7)
    SQB_PASS_(8) SQB_PASS_(9) SQB_PASS_(10) SQB_PASS_(11) SQB_PASS_(12) SQB_PASS_(13) SQB_PASS_(14) SQB_PASS_(15)
#undef SQB_PASS_
    return sqb_attr_of(sqb_k_fin<F, D>, block, smem, o);
}

/* the scaling test (sqb_scale_t): one thread per (direction, q); P::pt is the graph's raw double-double
 * point function (pt_<name> of the QREAL half, SQ_AB = 1 as the reference's default) */
template<class P>
__global__ void __launch_bounds__(SQB_BLOCK) sqb_k_scale(const sqb_scale_t a){
    for(long j = blockIdx.x*(long)blockDim.x + threadIdx.x; j < 3*a.ndir; j += (long)gridDim.x*blockDim.x)
        a.g[j] = sqb_scale_value<P>(a, j);
}

/* SQ_GRAPH(name, volkov, L, D, weight, n, fixed): the generated file ends with it, after namespace
 * SQG_NS(name) with the class template K<Real, SQ_AB> holding f_<name>.
 *
 * Every graph has two translation units.  The first (compiled with -fmad=false) holds the FP64 kernel
 * whose roundings are those of the source, the double-double kernel and the registry entry SQB_<name>.
 * The second (SQB_FMA_TU, compiled with -fmad=true, namespace sqgf_<name> so that no symbol is shared)
 * holds only the FP64 kernel with multiplies and adds contracted into fused multiply-adds, exported as
 * SQB_<name>_f64fma and SQB_<name>_attrfma; the registry entry refers to them weakly. */
/* the split form's point functions (SQ_GRAPH_SPLIT): pass P and the final pass in FP64 */
#define SQ_SPLIT_F(NAME)                                                                           \
namespace SQG_NS(NAME) {                                                                           \
struct FS {                                                                                        \
    template<int P, int AB> static __device__ __forceinline__ void part(const double *sf, double *T, double *A){ \
        K<double, AB>::template fpart_##NAME<P>(sf, T, A); }                                       \
    template<int AB> static __device__ __forceinline__ double fin(const double *sf, double T, double A, double *ab){ \
        return K<double, AB>::ffin_##NAME(sf, T, A, ab); }                                         \
};                                                                                                 \
}
#if defined(SQB_FMA_TU)
#define SQ_SCALE(NAME)
#define SQ_GRAPH(NAME, VOLKOV, L, D, W, NP, FIX)                                                    \
namespace SQG_NS(NAME) {                                                                           \
struct F {                                                                                         \
    template<class R, int AB> static __device__ __forceinline__ R f(const R *sf, R *ab){           \
        return K<R, AB>::f_##NAME(sf, ab); }                                                       \
};                                                                                                 \
}                                                                                                  \
extern "C" void SQB_##NAME##_f64fma(const sqb_eval_t *a, int grid, int block, size_t smem, void *st){ \
    if(sqb_level_launch(a)) sqb_k_f64<SQG_NS(NAME)::F, D, 1><<<grid, block, smem, (cudaStream_t)st>>>(*a); \
    else sqb_k_f64<SQG_NS(NAME)::F, D, 0><<<grid, block, smem, (cudaStream_t)st>>>(*a); }           \
extern "C" int SQB_##NAME##_attrfma(int lv, int block, size_t smem, sqb_kattr_t *o){               \
    return lv ? sqb_f64_attr(sqb_k_f64<SQG_NS(NAME)::F, D, 1>, 1, block, smem, o)                  \
              : sqb_f64_attr(sqb_k_f64<SQG_NS(NAME)::F, D, 0>, 0, block, smem, o); }
#define SQ_GRAPH_SPLIT(NAME, VOLKOV, L, D, W, NP, FIX, NPARTS)                                      \
SQ_GRAPH(NAME, VOLKOV, L, D, W, NP, FIX)                                                           \
SQ_SPLIT_F(NAME)                                                                                   \
extern "C" void SQB_##NAME##_splitfma(int P, const sqb_eval_t *a, double *tt, double *ta, int grid, int block, \
                                      size_t smem, void *st){                                      \
    sqb_split_launch<SQG_NS(NAME)::FS, D, NPARTS>(P, a, tt, ta, grid, block, smem, (cudaStream_t)st); } \
extern "C" int SQB_##NAME##_splitattrfma(int P, int block, size_t smem, sqb_kattr_t *o){          \
    return sqb_split_attr<SQG_NS(NAME)::FS, D, NPARTS>(P, block, smem, o); }
#else
/* SQ_SCALE(name) follows SQ_GRAPH for a graph with a raw point function: its scaling-test launcher */
#define SQ_SCALE(NAME)                                                                              \
namespace SQG_NS(NAME) {                                                                           \
struct PT {                                                                                        \
    static __device__ __forceinline__ sqdd pt(const sqdd *x, sqdd Vx, sqdd *ab){                   \
        return KD<sqdd, 1>::pt_##NAME(x, Vx, ab); }                                                \
};                                                                                                 \
}                                                                                                  \
extern "C" void SQB_##NAME##_scale(const sqb_scale_t *a, int grid, int block, void *st){           \
    sqb_k_scale<SQG_NS(NAME)::PT><<<grid, block, 0, (cudaStream_t)st>>>(*a); }
#define SQ_GRAPH_CORE(NAME, D)                                                                      \
extern "C" void SQB_##NAME##_f64fma(const sqb_eval_t *, int, int, size_t, void *) __attribute__((weak)); \
extern "C" void SQB_##NAME##_scale(const sqb_scale_t *, int, int, void *) __attribute__((weak));   \
extern "C" int SQB_##NAME##_attrfma(int, int, size_t, sqb_kattr_t *) __attribute__((weak));        \
namespace SQG_NS(NAME) {                                                                           \
struct F {                                                                                         \
    template<class R, int AB> static __device__ __forceinline__ R f(const R *sf, R *ab){           \
        return K<R, AB>::f_##NAME(sf, ab); }                                                       \
};                                                                                                 \
template<> __device__ __forceinline__ sqdd F::f<sqdd, 1>(const sqdd *sf, sqdd *ab){                \
    return KD<sqdd, 1>::f_##NAME(sf, ab); }                                                        \
static void f64(const sqb_eval_t *a, int grid, int block, size_t smem, void *st){                  \
    if(SQB_LEVEL_KERNEL && sqb_level_launch(a))                                                    \
        sqb_k_f64<F, D, SQB_LEVEL_KERNEL><<<grid, block, smem, (cudaStream_t)st>>>(*a);            \
    else sqb_k_f64<F, D, 0><<<grid, block, smem, (cudaStream_t)st>>>(*a); }                        \
static void dd(const sqb_dd_t *a, int grid, int block, size_t smem, void *st){                     \
    sqb_k_dd<F, D><<<grid, block, smem, (cudaStream_t)st>>>(*a); }                                 \
static int attr(int which, int block, size_t smem, sqb_kattr_t *o){                                \
    const int lv = (which & SQB_ATTR_LEVEL) != 0; which &= ~SQB_ATTR_LEVEL;                        \
    if(which == 2) return SQB_##NAME##_attrfma ? SQB_##NAME##_attrfma(lv, block, smem, o) : 0;      \
    if(which == 1) return sqb_f64_attr(sqb_k_dd<F, D>, 0, block, smem, o);                         \
    return SQB_LEVEL_KERNEL && lv ? sqb_f64_attr(sqb_k_f64<F, D, SQB_LEVEL_KERNEL>, 1, block, smem, o) \
                                  : sqb_f64_attr(sqb_k_f64<F, D, 0>, 0, block, smem, o); }         \
}
#define SQ_GRAPH(NAME, VOLKOV, L, D, W, NP, FIX)                                                    \
SQ_GRAPH_CORE(NAME, D)                                                                             \
extern "C" const sqb_graph_t SQB_##NAME = {#NAME, VOLKOV, L, D, W, NP, FIX, 0,                     \
    SQG_NS(NAME)::f64, SQG_NS(NAME)::dd, SQG_NS(NAME)::attr, SQB_##NAME##_f64fma, 0, NULL, NULL,     \
    SQB_##NAME##_scale};
#define SQ_GRAPH_SPLIT(NAME, VOLKOV, L, D, W, NP, FIX, NPARTS)                                      \
SQ_GRAPH_CORE(NAME, D)                                                                             \
SQ_SPLIT_F(NAME)                                                                                   \
extern "C" void SQB_##NAME##_splitfma(int, const sqb_eval_t *, double *, double *, int, int, size_t, void *) \
    __attribute__((weak));                                                                         \
extern "C" int SQB_##NAME##_splitattrfma(int, int, size_t, sqb_kattr_t *) __attribute__((weak));   \
namespace SQG_NS(NAME) {                                                                           \
static void split(int P, int fma, const sqb_eval_t *a, double *tt, double *ta, int grid, int block, size_t smem, \
                  void *st){                                                                       \
    if(fma && SQB_##NAME##_splitfma) SQB_##NAME##_splitfma(P, a, tt, ta, grid, block, smem, st);    \
    else sqb_split_launch<FS, D, NPARTS>(P, a, tt, ta, grid, block, smem, (cudaStream_t)st); }     \
static int split_attr(int P, int fma, int block, size_t smem, sqb_kattr_t *o){                     \
    if(fma && SQB_##NAME##_splitattrfma) return SQB_##NAME##_splitattrfma(P, block, smem, o);       \
    return sqb_split_attr<FS, D, NPARTS>(P, block, smem, o); }                                      \
}                                                                                                  \
extern "C" const sqb_graph_t SQB_##NAME = {#NAME, VOLKOV, L, D, W, NP, FIX, 0,                     \
    SQG_NS(NAME)::f64, SQG_NS(NAME)::dd, SQG_NS(NAME)::attr, SQB_##NAME##_f64fma, NPARTS,           \
    SQG_NS(NAME)::split, SQG_NS(NAME)::split_attr, SQB_##NAME##_scale};
#endif
