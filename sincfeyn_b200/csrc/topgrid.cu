/* topgrid.cu -- the top level of the hierarchical sum on the device: the support-following grow's
 * bookkeeping, the shadow-tier flood fill and the dilation (driver/sumkey.h:20-461).
 *
 * Points of the top grid (step st) are identified by the reference's mixed-radix key
 * 1 c_0 ... c_{D-1} in base W = 2(K/st)+1, c_i = k_i/st + K/st (driver/sumkey.h:7-18): numeric order is
 * lexicographic order in k, and an axis step is +-P[j].
 *
 * One device hash table holds every evaluated point of the grow with a 32-bit claim word: SEEN for a
 * point already evaluated, else the best claim of this frontier's candidates, stored as
 * 0xFFFFFFFE - id so that atomicMax keeps the lowest candidate id (the reference's parallel claims,
 * driver/sumkey.h:288-374).  The winners, compacted in id order, are the next frontier: exactly the
 * not-yet-seen neighbours of the kept points in (kept point, axis, sign) order.
 *
 * Order-preserving compactions (kept points, winners, re-threshold) use per-tile counts, one exclusive
 * scan and a per-tile ranked scatter.  The dilation inserts every cell and its in-box axis neighbours
 * into a hash table merging the flags (skip bit AND, tier max, driver/sumkey.h:41-44), collects the
 * distinct keys and sorts them with a stable LSD radix sort (8-bit digits), the reference's summation
 * order.  Every probe loop is bounded by the table size and reports overflow instead of spinning. */
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "sqb_rt.h"

#define TG_T 256                 /* threads per CTA of the compaction kernels */
#define TG_I 8                   /* items per thread */
#define TG_TILE (TG_T*TG_I)
#define SEEN 0xFFFFFFFFu
#define CLAIM(id) (0xFFFFFFFEu - (unsigned)(id))

static thread_local char terr[512];   /* the state of this file is per host thread, like the runtime's */
#define TCK(x) do { cudaError_t e_ = (x); if(e_ != cudaSuccess){                                    \
    snprintf(terr, sizeof terr, "%s at %s:%d: %s", #x, __FILE__, __LINE__, cudaGetErrorString(e_));   \
    return (int)e_; } } while(0)
extern "C" const char *sqb_top_error(void){ return terr; }

__device__ __forceinline__ unsigned long long hslot(unsigned long long y, unsigned long long mask){
    return ((y*0x9E3779B97F4A7C15ULL) >> 21) & mask;
}
/* slot of key y, inserting it if absent (*isnew = 1); -1 if the table is full */
__device__ long h_insert(unsigned long long *key, unsigned long long mask, unsigned long long y, int *isnew){
    unsigned long long i = hslot(y, mask);
    for(unsigned long long p = 0; p <= mask; p++){
        unsigned long long c = key[i];
        if(c == y){ *isnew = 0; return (long)i; }
        if(c == 0){
            unsigned long long o = atomicCAS(&key[i], 0ULL, y);
            if(o == 0){ *isnew = 1; return (long)i; }
            if(o == y){ *isnew = 0; return (long)i; }
        }
        i = (i + 1) & mask;
    }
    return -1;
}
__device__ long h_find(const unsigned long long *key, unsigned long long mask, unsigned long long y){
    unsigned long long i = hslot(y, mask);
    for(unsigned long long p = 0; p <= mask; p++){
        unsigned long long c = key[i];
        if(c == y) return (long)i;
        if(c == 0) return -1;
        i = (i + 1) & mask;
    }
    return -1;
}

struct geom_t { int D, K, st, W; unsigned long long P[SQB_MAXD]; };

__device__ __forceinline__ unsigned long long key_of(const geom_t &g, const signed char *k){
    unsigned long long y = 1;
    for(int i = 0; i < g.D; i++) y = y*g.W + (unsigned long long)(k[i]/g.st + g.K/g.st);
    return y;
}

/* --------------------------------- generic ordered compaction ----------------------------------- */
/* Op: __device__ bool pred(long i); __device__ void emit(long i, unsigned long long rank) */
template<class Op>
__global__ void __launch_bounds__(TG_T) k_count(Op op, long n, unsigned *bcnt){
    const long t0 = blockIdx.x*(long)TG_TILE + threadIdx.x*(long)TG_I;
    unsigned c = 0;
    for(int j = 0; j < TG_I; j++){ long i = t0 + j; if(i < n && op.pred(i)) c++; }
    for(int off = 16; off; off >>= 1) c += __shfl_down_sync(0xffffffffu, c, off);
    __shared__ unsigned ws[TG_T/32];
    if((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
    __syncthreads();
    if(threadIdx.x == 0){ unsigned s = 0; for(int w = 0; w < TG_T/32; w++) s += ws[w]; bcnt[blockIdx.x] = s; }
}
/* one CTA: exclusive scan of nb counts; total into *tot */
__global__ void __launch_bounds__(256) k_scan(const unsigned *bcnt, long nb, unsigned long long *boff, unsigned long long *tot){
    __shared__ unsigned long long pre[256];
    const int t = threadIdx.x; const long ch = (nb + 255)/256, j0 = t*ch, j1 = j0 + ch < nb ? j0 + ch : nb;
    unsigned long long s = 0; for(long j = j0; j < j1; j++) s += bcnt[j];
    pre[t] = s; __syncthreads();
    if(t == 0){ unsigned long long x = 0; for(int j = 0; j < 256; j++){ unsigned long long y = pre[j]; pre[j] = x; x += y; } *tot = x; }
    __syncthreads();
    unsigned long long x = pre[t]; for(long j = j0; j < j1; j++){ boff[j] = x; x += bcnt[j]; }
}
template<class Op>
__global__ void __launch_bounds__(TG_T) k_scatter(Op op, long n, const unsigned long long *boff){
    const long t0 = blockIdx.x*(long)TG_TILE + threadIdx.x*(long)TG_I;
    unsigned mask = 0; int c = 0;
    for(int j = 0; j < TG_I; j++){ long i = t0 + j; if(i < n && op.pred(i)){ mask |= 1u << j; c++; } }
    __shared__ int ws[TG_T/32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    int x = c;
    for(int off = 1; off < 32; off <<= 1){ int y = __shfl_up_sync(0xffffffffu, x, off); if(l >= off) x += y; }
    if(l == 31) ws[w] = x;
    __syncthreads();
    if(threadIdx.x == 0){ int s = 0; for(int q = 0; q < TG_T/32; q++){ int y = ws[q]; ws[q] = s; s += y; } }
    __syncthreads();
    unsigned long long r = boff[blockIdx.x] + (unsigned long long)(ws[w] + x - c);
    for(int j = 0; j < TG_I; j++) if(mask >> j & 1) op.emit(t0 + j, r++);
}

struct Scratch { unsigned *bcnt; unsigned long long *boff, *tot; long nbcap; };
static thread_local Scratch SC;
static thread_local cudaStream_t TS;
/* stream-ordered allocation from the device's memory pool: no device-wide synchronisation, and the pool
 * keeps freed memory for the next integral (the runtime sets its release threshold) */
#define DMALLOC(p, n) cudaMallocAsync((void**)(p), (n), TS)
#define DFREE(p) cudaFreeAsync((p), TS)
static thread_local unsigned long long TL;    /* kernels launched by this file */
extern "C" unsigned long long sqb_top_launches(void){ return TL; }
extern "C" void sqb_dev_count_copy(unsigned long long h2d, unsigned long long d2h);

static int scratch(long n){
    long nb = (n + TG_TILE - 1)/TG_TILE; if(nb < 1) nb = 1;
    if(nb <= SC.nbcap) return 0;
    if(SC.bcnt){ DFREE(SC.bcnt); DFREE(SC.boff); }
    long c = 1024; while(c < nb) c <<= 1;
    TCK(DMALLOC(&SC.bcnt, c*sizeof(unsigned))); TCK(DMALLOC(&SC.boff, c*sizeof(unsigned long long)));
    if(!SC.tot) TCK(DMALLOC(&SC.tot, sizeof(unsigned long long)));
    SC.nbcap = c;
    return 0;
}
/* ordered compaction; returns the count (synchronous) */
template<class Op>
static int compact(const Op &op, long n, long *count){
    *count = 0;
    if(n <= 0) return 0;
    if(scratch(n)) return -1;
    const long nb = (n + TG_TILE - 1)/TG_TILE;
    k_count<Op><<<(unsigned)nb, TG_T, 0, TS>>>(op, n, SC.bcnt);
    k_scan<<<1, 256, 0, TS>>>(SC.bcnt, nb, SC.boff, SC.tot);
    k_scatter<Op><<<(unsigned)nb, TG_T, 0, TS>>>(op, n, SC.boff);
    TL += 3;
    TCK(cudaGetLastError());
    unsigned long long t = 0;
    TCK(cudaMemcpyAsync(&t, SC.tot, sizeof t, cudaMemcpyDeviceToHost, TS));
    TCK(cudaStreamSynchronize(TS));
    sqb_dev_count_copy(0, sizeof t);
    *count = (long)t;
    return 0;
}

/* --------------------------------------------- grow --------------------------------------------- */
struct Grow {
    geom_t g;
    unsigned long long *key; unsigned *word; unsigned long long mask; long nseen;   /* seen table */
    sqb_pt_t *fr, *nx; unsigned char *frsk, *nxsk, *cls; long nfr, frcap;         /* frontier, next */
    sqb_pt_t *keep; double *kv; long nkeep, keepcap;                              /* kept so far */
    long *kj; long kjcap;                                                        /* this frontier's kept */
    long *qs; long qscap;                                                        /* slot per candidate */
    unsigned long long *err;
    int gs, abskip;
    unsigned char *hcls; long hclscap;     /* pinned: the frontier's shell classes, read after the next sync */
    unsigned long long *herr;              /* pinned: the overflow count, read after the next sync */
};
static thread_local Grow GR;

__global__ void k_rehash(const unsigned long long *ok, const unsigned *ow, long ocap, unsigned long long *key,
                         unsigned *word, unsigned long long mask, unsigned long long *err){
    for(long i = blockIdx.x*(long)blockDim.x + threadIdx.x; i < ocap; i += (long)gridDim.x*blockDim.x){
        if(!ok[i]) continue;
        int nw; long q = h_insert(key, mask, ok[i], &nw);
        if(q < 0){ atomicAdd(err, 1ULL); continue; }
        word[q] = ow[i];
    }
}
/* keep the seen table at most 60% full after extra more keys */
static int table_room(long extra){
    long cap = (long)GR.mask + 1;
    if((double)(GR.nseen + extra) <= 0.6*cap) return 0;
    long nc = cap; while((double)(GR.nseen + extra) > 0.6*nc) nc <<= 1;
    unsigned long long *k2; unsigned *w2;
    TCK(DMALLOC(&k2, nc*sizeof(unsigned long long))); TCK(DMALLOC(&w2, nc*sizeof(unsigned)));
    TCK(cudaMemsetAsync(k2, 0, nc*sizeof(unsigned long long), TS)); TCK(cudaMemsetAsync(w2, 0, nc*sizeof(unsigned), TS));
    k_rehash<<<1184, 256, 0, TS>>>(GR.key, GR.word, cap, k2, w2, (unsigned long long)(nc - 1), GR.err); TL++;
    TCK(cudaGetLastError());
    TCK(cudaStreamSynchronize(TS));
    DFREE(GR.key); DFREE(GR.word);
    GR.key = k2; GR.word = w2; GR.mask = (unsigned long long)(nc - 1);
    return 0;
}
/* device array of at least n elements, keeping the first keep elements */
template<class T> static int devbuf(T **p, long *cap, long n, long keep){
    if(n <= *cap && *p) return 0;
    long c = 1L << 16; while(c < n) c <<= 1;
    T *q; TCK(DMALLOC(&q, c*sizeof(T)));
    if(*p && keep > 0){ TCK(cudaMemcpyAsync(q, *p, keep*sizeof(T), cudaMemcpyDeviceToDevice, TS)); TCK(cudaStreamSynchronize(TS)); }
    if(*p) DFREE(*p);
    *p = q; *cap = c;
    return 0;
}
/* frontier buffers for n points, the current frontier kept */
static int frontier_room(long n){
    if(n <= GR.frcap && GR.fr) return 0;
    long c = 1L << 16; while(c < n) c <<= 1;
    sqb_pt_t *a, *b; unsigned char *s1, *s2, *s3;
    TCK(DMALLOC(&a, c*sizeof(sqb_pt_t))); TCK(DMALLOC(&b, c*sizeof(sqb_pt_t)));
    TCK(DMALLOC(&s1, c)); TCK(DMALLOC(&s2, c)); TCK(DMALLOC(&s3, c));
    if(GR.fr){
        TCK(cudaMemcpyAsync(a, GR.fr, GR.nfr*sizeof(sqb_pt_t), cudaMemcpyDeviceToDevice, TS));
        TCK(cudaMemcpyAsync(s1, GR.frsk, GR.nfr, cudaMemcpyDeviceToDevice, TS));
        TCK(cudaStreamSynchronize(TS));
        DFREE(GR.fr); DFREE(GR.nx); DFREE(GR.frsk); DFREE(GR.nxsk); DFREE(GR.cls);
    }
    GR.fr = a; GR.nx = b; GR.frsk = s1; GR.nxsk = s2; GR.cls = s3; GR.frcap = c;
    return 0;
}

__global__ void k_seed(unsigned long long *key, unsigned *word, unsigned long long mask, unsigned long long y0,
                       sqb_pt_t *fr, unsigned char *frsk, unsigned long long *err){
    int nw; long q = h_insert(key, mask, y0, &nw);
    if(q < 0){ atomicAdd(err, 1ULL); return; }
    word[q] = SEEN;
    for(int i = 0; i < SQB_MAXD; i++) fr[0].k[i] = 0;
    frsk[0] = 0;
}

/* a new grow at step st; the frontier is z = 0 */
extern "C" int sqb_grow_begin(int D, int K, int st, int W, const unsigned long long *P, int gs, int abskip, void *stream){
    TS = (cudaStream_t)stream;
    memset(&GR.g, 0, sizeof GR.g);
    GR.g.D = D; GR.g.K = K; GR.g.st = st; GR.g.W = W; for(int i = 0; i < D; i++) GR.g.P[i] = P[i];
    GR.gs = gs; GR.abskip = abskip; GR.nseen = 1; GR.nkeep = 0; GR.nfr = 0;
    const long cap = 1L << 22;
    if(GR.key){ DFREE(GR.key); DFREE(GR.word); GR.key = NULL; }
    TCK(DMALLOC(&GR.key, cap*sizeof(unsigned long long))); TCK(DMALLOC(&GR.word, cap*sizeof(unsigned)));
    TCK(cudaMemsetAsync(GR.key, 0, cap*sizeof(unsigned long long), TS)); TCK(cudaMemsetAsync(GR.word, 0, cap*sizeof(unsigned), TS));
    GR.mask = (unsigned long long)(cap - 1);
    if(!GR.err) TCK(DMALLOC(&GR.err, sizeof(unsigned long long)));
    TCK(cudaMemsetAsync(GR.err, 0, sizeof(unsigned long long), TS));
    if(frontier_room(1)) return -1;
    unsigned long long y0 = 1; for(int i = 0; i < D; i++) y0 = y0*W + (unsigned long long)(K/st);
    k_seed<<<1, 1, 0, TS>>>(GR.key, GR.word, GR.mask, y0, GR.fr, GR.frsk, GR.err); TL++;
    TCK(cudaGetLastError());
    TCK(cudaStreamSynchronize(TS));
    GR.nfr = 1;
    return 0;
}
extern "C" long sqb_grow_frontier(const sqb_pt_t **pts, const unsigned char **skip){
    *pts = GR.fr; *skip = GR.gs ? GR.frsk : NULL; return GR.nfr;
}

/* per frontier point: bit 1 mx == K, bit 2 mx == K - st (the outer shells, driver/sumkey.h:236-238) */
__global__ void k_shell(const sqb_pt_t *fr, long n, geom_t g, unsigned char *cls){
    for(long i = blockIdx.x*(long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x*blockDim.x){
        int mx = 0; for(int d = 0; d < g.D; d++){ int x = abs((int)fr[i].k[d]); if(x > mx) mx = x; }
        cls[i] = mx == g.K ? 2 : (mx == g.K - g.st ? 4 : 0);
    }
}
/* the frontier's shell classes: the kernel and the copy to pinned memory are queued on the grow's stream
 * without waiting (sqb_grow_shells_async, before the frontier's evaluation, whose results the caller waits
 * for anyway), and sqb_grow_shells_take copies them out after that wait */
extern "C" int sqb_grow_shells_async(void){
    if(!GR.nfr) return 0;
    if(GR.nfr > GR.hclscap){
        if(GR.hcls) cudaFreeHost(GR.hcls);
        long c = 1L << 16; while(c < GR.nfr) c <<= 1;
        TCK(cudaMallocHost(&GR.hcls, c)); GR.hclscap = c;
    }
    k_shell<<<1184, 256, 0, TS>>>(GR.fr, GR.nfr, GR.g, GR.cls); TL++;
    TCK(cudaGetLastError());
    TCK(cudaMemcpyAsync(GR.hcls, GR.cls, GR.nfr, cudaMemcpyDeviceToHost, TS));
    sqb_dev_count_copy(0, GR.nfr);
    return 0;
}
extern "C" void sqb_grow_shells_take(unsigned char *cls_host){
    if(GR.nfr) memcpy(cls_host, GR.hcls, GR.nfr);
}

struct KeepOp {                  /* kept frontier points appended to the keep list, their index to kj */
    const sqb_pt_t *fr; const double *v; const unsigned char *stt; double thr; int abskip, D;
    sqb_pt_t *keep; double *kv; long *kj; long base;
    __device__ bool pred(long i) const { return fabs(v[i]) >= thr; }
    __device__ void emit(long i, unsigned long long r) const {
        sqb_pt_t p; for(int q = 0; q < SQB_MAXD; q++) p.k[q] = 0;
        for(int d = 0; d < D; d++) p.k[d] = fr[i].k[d];
        if(abskip) p.k[SQB_PFLAG] = (stt[i] & SQB_NEAR) ? 0 : 1;
        keep[base + r] = p; kv[base + r] = fabs(v[i]); kj[r] = i;
    }
};

__global__ void k_claim(geom_t g, const sqb_pt_t *fr, const long *kj, long nk, unsigned long long *key, unsigned *word,
                        unsigned long long mask, long *qs, unsigned long long *err){
    const int D2 = 2*g.D;
    const long nc = nk*D2;
    for(long id = blockIdx.x*(long)blockDim.x + threadIdx.x; id < nc; id += (long)gridDim.x*blockDim.x){
        const long j = id/D2; const int c = (int)(id - j*D2), d = c >> 1, sg = (c & 1) ? 1 : -1;
        const signed char *k = fr[kj[j]].k;
        const int kk = k[d] + g.st*sg;
        if(kk > g.K || kk < -g.K){ qs[id] = -1; continue; }
        const unsigned long long y = key_of(g, k) + (sg > 0 ? g.P[d] : (unsigned long long)0 - g.P[d]);
        int nw; const long q = h_insert(key, mask, y, &nw);
        if(q < 0){ atomicAdd(err, 1ULL); qs[id] = -1; continue; }
        qs[id] = q;
        atomicMax(&word[q], CLAIM(id));
    }
}
struct WinOp {                   /* winners in id order become the next frontier */
    const sqb_pt_t *fr; const long *kj; const long *qs; unsigned *word; const unsigned char *frsk; const unsigned char *stt;
    sqb_pt_t *nx; unsigned char *nxsk; int D2, st, gs;
    __device__ bool pred(long id) const { const long q = qs[id]; return q >= 0 && word[q] == CLAIM(id); }
    __device__ void emit(long id, unsigned long long r) const {
        const long j = id/D2; const int c = (int)(id - j*D2), d = c >> 1, sg = (c & 1) ? 1 : -1;
        const long pi = kj[j];
        sqb_pt_t p = fr[pi];
        p.k[d] = (signed char)(p.k[d] + st*sg);
        if(gs){ const int pg = fr[pi].k[SQB_PFLAG];
            p.k[SQB_PFLAG] = (signed char)(!frsk[pi] ? ((stt[pi] & SQB_NEAR) ? 0 : 1) : (pg < gs ? pg + 1 : 0));
            nxsk[r] = p.k[SQB_PFLAG] > 0; }
        else p.k[SQB_PFLAG] = 0;
        nx[r] = p;
        word[qs[id]] = SEEN;
    }
};

/* after the host has the frontier's threshold: kept points appended, next frontier built */
extern "C" int sqb_grow_expand(const double *v_dev, const unsigned char *stt_dev, double thr, long *nkept, long *nnext){
    const long n = GR.nfr;
    long kc = GR.keepcap, vc = GR.keepcap;
    if(devbuf(&GR.keep, &kc, GR.nkeep + n, GR.nkeep) || devbuf(&GR.kv, &vc, GR.nkeep + n, GR.nkeep)) return -1;
    GR.keepcap = kc;
    if(devbuf(&GR.kj, &GR.kjcap, n, 0)) return -1;
    KeepOp ko; ko.fr = GR.fr; ko.v = v_dev; ko.stt = stt_dev; ko.thr = thr; ko.abskip = GR.abskip; ko.D = GR.g.D;
    ko.keep = GR.keep; ko.kv = GR.kv; ko.kj = GR.kj; ko.base = GR.nkeep;
    long nk = 0;
    if(compact(ko, n, &nk)) return -1;
    GR.nkeep += nk; *nkept = nk;
    const long nc = nk*2*GR.g.D;
    if(nc >= 0xFFFFFFF0L){ snprintf(terr, sizeof terr, "grow: %ld candidates exceed the 32-bit claim ids", nc); return -1; }
    if(table_room(nc)) return -1;
    if(devbuf(&GR.qs, &GR.qscap, nc, 0)) return -1;
    if(frontier_room(nc)) return -1;
    if(nc){ k_claim<<<1184, 256, 0, TS>>>(GR.g, GR.fr, GR.kj, nk, GR.key, GR.word, GR.mask, GR.qs, GR.err); TL++; }
    TCK(cudaGetLastError());
    /* the overflow count after the claims (the only writers), read once the next compaction has waited */
    if(!GR.herr) TCK(cudaMallocHost(&GR.herr, sizeof(unsigned long long)));
    TCK(cudaMemcpyAsync(GR.herr, GR.err, sizeof(unsigned long long), cudaMemcpyDeviceToHost, TS));
    WinOp wo; wo.fr = GR.fr; wo.kj = GR.kj; wo.qs = GR.qs; wo.word = GR.word; wo.frsk = GR.frsk; wo.stt = stt_dev;
    wo.nx = GR.nx; wo.nxsk = GR.nxsk; wo.D2 = 2*GR.g.D; wo.st = GR.g.st; wo.gs = GR.gs;
    long nn = 0;
    if(compact(wo, nc, &nn)) return -1;
    GR.nseen += nn;
    { sqb_pt_t *t = GR.fr; GR.fr = GR.nx; GR.nx = t; unsigned char *q = GR.frsk; GR.frsk = GR.nxsk; GR.nxsk = q; }
    GR.nfr = nn; *nnext = nn;
    if(nc <= 0) TCK(cudaStreamSynchronize(TS));          /* no compaction waited for the copy */
    if(*GR.herr){ snprintf(terr, sizeof terr, "grow: hash table overflow"); return -1; }
    return 0;
}

/* kept |f| values in keep order (host), for the final threshold's dropped weight */
extern "C" int sqb_grow_kv(double *kv_host, long n){
    TCK(cudaMemcpyAsync(kv_host, GR.kv, n*sizeof(double), cudaMemcpyDeviceToHost, TS));
    TCK(cudaStreamSynchronize(TS));
    sqb_dev_count_copy(0, n*sizeof(double));
    return 0;
}

struct RethOp {
    const sqb_pt_t *keep; const double *kv; double thr; sqb_pt_t *out; double *okv;
    __device__ bool pred(long i) const { return kv[i] >= thr; }
    __device__ void emit(long i, unsigned long long r) const { out[r] = keep[i]; okv[r] = kv[i]; }
};

/* shadow tiers: breadth-first from z = 0 through kept points with |f| >= lim (driver/sumkey.h:402-444) */
__global__ void k_index(geom_t g, const sqb_pt_t *keep, long m, unsigned long long *key, unsigned *word,
                        unsigned long long mask, unsigned long long *err){
    for(long i = blockIdx.x*(long)blockDim.x + threadIdx.x; i < m; i += (long)gridDim.x*blockDim.x){
        int nw; long q = h_insert(key, mask, key_of(g, keep[i].k), &nw);
        if(q < 0){ atomicAdd(err, 1ULL); continue; }
        word[q] = (unsigned)i;
    }
}
__global__ void k_tier_seed(geom_t g, const unsigned long long *key, const unsigned *word, unsigned long long mask,
                            const double *kv, double lim, int t, unsigned *tr, long *cu, unsigned long long *ncu){
    unsigned long long y = 1; for(int i = 0; i < g.D; i++) y = y*g.W + (unsigned long long)(g.K/g.st);
    long q = h_find(key, mask, y);
    *ncu = 0;
    if(q < 0) return;
    long i = word[q];
    if(kv[i] >= lim){ atomicMax(&tr[i], (unsigned)t); cu[0] = i; *ncu = 1; }
}
__global__ void k_tier_step(geom_t g, const sqb_pt_t *keep, const unsigned long long *key, const unsigned *word,
                            unsigned long long mask, const double *kv, double lim, int t, unsigned *tr,
                            const long *cu, const unsigned long long *ncu, long *nw, unsigned long long *nnw){
    const int D2 = 2*g.D;
    const long nc = (long)*ncu;          /* the frontier's size, written by the step (or seed) before */
    for(long x = blockIdx.x*(long)blockDim.x + threadIdx.x; x < nc*D2; x += (long)gridDim.x*blockDim.x){
        const long i = cu[x/D2]; const int c = (int)(x % D2), d = c >> 1, sg = (c & 1) ? 1 : -1;
        const int kk = keep[i].k[d] + g.st*sg;
        if(kk > g.K || kk < -g.K) continue;
        const unsigned long long y = key_of(g, keep[i].k) + (sg > 0 ? g.P[d] : (unsigned long long)0 - g.P[d]);
        const long q = h_find(key, mask, y);
        if(q < 0) continue;
        const long j = word[q];
        if(kv[j] >= lim && atomicMax(&tr[j], (unsigned)t) < (unsigned)t) nw[atomicAdd(nnw, 1ULL)] = j;
    }
}
__global__ void k_tier_apply(sqb_pt_t *keep, const unsigned *tr, long m){
    for(long i = blockIdx.x*(long)blockDim.x + threadIdx.x; i < m; i += (long)gridDim.x*blockDim.x)
        keep[i].k[SQB_PFLAG] = (signed char)((keep[i].k[SQB_PFLAG] & 1) | (tr[i] << 1));
}

/* the final threshold and the tiers; *m = kept points left; the keep list stays on the device */
extern "C" int sqb_grow_finish(double thr, int tiers, long *m_out){
    sqb_pt_t *out; double *okv; const long n = GR.nkeep;
    TCK(DMALLOC(&out, (n ? n : 1)*sizeof(sqb_pt_t))); TCK(DMALLOC(&okv, (n ? n : 1)*sizeof(double)));
    RethOp ro; ro.keep = GR.keep; ro.kv = GR.kv; ro.thr = thr; ro.out = out; ro.okv = okv;
    long m = 0;
    if(compact(ro, n, &m)) return -1;
    DFREE(GR.keep); DFREE(GR.kv); GR.keep = out; GR.kv = okv; GR.keepcap = n ? n : 1; GR.nkeep = m;
    *m_out = m;
    if(!tiers || !m) return 0;
    long cap = 1L << 20; while(cap < 2*m) cap <<= 1;
    unsigned long long *key; unsigned *word, *tr; long *cu, *nw; unsigned long long *cnt;
    TCK(DMALLOC(&key, cap*sizeof(unsigned long long))); TCK(DMALLOC(&word, cap*sizeof(unsigned)));
    TCK(DMALLOC(&tr, m*sizeof(unsigned))); TCK(DMALLOC(&cu, m*sizeof(long))); TCK(DMALLOC(&nw, m*sizeof(long)));
    TCK(DMALLOC(&cnt, 2*sizeof(unsigned long long)));
    TCK(cudaMemsetAsync(key, 0, cap*sizeof(unsigned long long), TS)); TCK(cudaMemsetAsync(tr, 0, m*sizeof(unsigned), TS));
    k_index<<<1184, 256, 0, TS>>>(GR.g, GR.keep, m, key, word, (unsigned long long)(cap - 1), GR.err); TL++;
    /* breadth-first steps read the frontier's size on the device, so the host checks for the end only
     * every TSTEPS steps (steps after the end find an empty frontier and do nothing) */
    const int TSTEPS = 8;
    for(int t = 1; t <= 2; t++){
        const double lim = (t == 1 ? 10 : 100)*thr;
        unsigned long long *ca = cnt, *cb = cnt + 1;
        k_tier_seed<<<1, 1, 0, TS>>>(GR.g, key, word, (unsigned long long)(cap - 1), GR.kv, lim, t, tr, cu, ca); TL++;
        for(;;){
            for(int s = 0; s < TSTEPS; s++){
                TCK(cudaMemsetAsync(cb, 0, sizeof(unsigned long long), TS));
                k_tier_step<<<1184, 256, 0, TS>>>(GR.g, GR.keep, key, word, (unsigned long long)(cap - 1), GR.kv, lim, t, tr,
                                                  cu, ca, nw, cb); TL++;
                TCK(cudaGetLastError());
                long *x = cu; cu = nw; nw = x;
                unsigned long long *y = ca; ca = cb; cb = y;
            }
            unsigned long long nc = 0;
            TCK(cudaMemcpyAsync(&nc, ca, sizeof nc, cudaMemcpyDeviceToHost, TS)); TCK(cudaStreamSynchronize(TS));
            if(!nc) break;
        }
    }
    k_tier_apply<<<1184, 256, 0, TS>>>(GR.keep, tr, m); TL++;
    TCK(cudaGetLastError());
    TCK(cudaStreamSynchronize(TS));
    DFREE(key); DFREE(word); DFREE(tr); DFREE(cu); DFREE(nw); DFREE(cnt);
    return 0;
}

/* ------------------------------------------- dilation -------------------------------------------- */
__global__ void k_dil_insert(geom_t g, const sqb_pt_t *cur, long n0, unsigned long long *key, unsigned *skb, unsigned *trm,
                             unsigned long long mask, unsigned long long *cnt, unsigned long long *err){
    const int C = 2*g.D + 1;
    for(long x = blockIdx.x*(long)blockDim.x + threadIdx.x; x < n0*C; x += (long)gridDim.x*blockDim.x){
        const long q0 = x/C; const int c = (int)(x - q0*C);
        const signed char *k = cur[q0].k; const int fl = k[SQB_PFLAG];
        unsigned long long y = key_of(g, k);
        if(c > 0){
            const int j = (c - 1) >> 1, sg = ((c - 1) & 1) ? 1 : -1, kk = k[j] + g.st*sg;
            if(kk > g.K || kk < -g.K) continue;
            y = sg > 0 ? y + g.P[j] : y - g.P[j];
        }
        int nw; const long q = h_insert(key, mask, y, &nw);
        if(q < 0){ atomicAdd(err, 1ULL); continue; }
        if(nw) atomicAdd(cnt, 1ULL);
        if(!(fl & 1)) atomicAnd(&skb[q], 0u);
        atomicMax(&trm[q], (unsigned)(fl >> 1));
    }
}
struct SlotOp {
    const unsigned long long *key; unsigned long long *out;
    __device__ bool pred(long i) const { return key[i] != 0; }
    __device__ void emit(long i, unsigned long long r) const { out[r] = key[i]; }
};
__global__ void k_dil_decode(geom_t g, const unsigned long long *U, long m, const unsigned long long *key, const unsigned *skb,
                             const unsigned *trm, unsigned long long mask, sqb_pt_t *out){
    for(long j = blockIdx.x*(long)blockDim.x + threadIdx.x; j < m; j += (long)gridDim.x*blockDim.x){
        unsigned long long y = U[j]; sqb_pt_t p;
        for(int i = 0; i < SQB_MAXD; i++) p.k[i] = 0;
        for(int i = g.D - 1; i >= 0; i--){ p.k[i] = (signed char)(((int)(y % g.W) - g.K/g.st)*g.st); y /= g.W; }
        const long q = h_find(key, mask, U[j]);
        if(q >= 0) p.k[SQB_PFLAG] = (signed char)((skb[q] & 1) | (trm[q] << 1));
        out[j] = p;
    }
}

/* stable LSD radix sort of n 64-bit keys, nbits significant, 8-bit digits; result in *a (a, b swapped) */
#define RS_T 256
#define RS_I 16
#define RS_TILE (RS_T*RS_I)
__global__ void __launch_bounds__(RS_T) k_rs_hist(const unsigned long long *a, long n, int sh, unsigned *hist, long nblk){
    __shared__ unsigned h[256];
    h[threadIdx.x] = 0; __syncthreads();
    const long t0 = blockIdx.x*(long)RS_TILE;
    for(int j = 0; j < RS_I; j++){ long i = t0 + j*RS_T + threadIdx.x; if(i < n) atomicAdd(&h[(a[i] >> sh) & 255], 1u); }
    __syncthreads();
    hist[(long)threadIdx.x*nblk + blockIdx.x] = h[threadIdx.x];
}
__global__ void __launch_bounds__(RS_T) k_rs_scatter(const unsigned long long *a, unsigned long long *b, long n, int sh,
                                                     const unsigned long long *off, long nblk){
    __shared__ unsigned long long base[256];
    __shared__ unsigned wc[RS_T/32][256];
    base[threadIdx.x] = off[(long)threadIdx.x*nblk + blockIdx.x];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const long t0 = blockIdx.x*(long)RS_TILE;
    for(int j = 0; j < RS_I; j++){
        for(int q = 0; q < RS_T/32; q++) wc[q][threadIdx.x] = 0;
        __syncthreads();
        const long i = t0 + j*RS_T + threadIdx.x;
        const bool in = i < n;
        const unsigned long long x = in ? a[i] : 0;
        const unsigned dg = in ? (unsigned)((x >> sh) & 255) : 256u + l;   /* out-of-range lanes never match */
        const unsigned peers = __match_any_sync(0xffffffffu, dg);
        const unsigned lt = peers & ((1u << l) - 1);
        if(in && lt == 0) wc[w][dg] = __popc(peers);
        __syncthreads();
        if(in){
            unsigned long long o = base[dg] + __popc(lt);
            for(int q = 0; q < w; q++) o += wc[q][dg];
            b[o] = x;
        }
        __syncthreads();
        unsigned s = 0; for(int q = 0; q < RS_T/32; q++) s += wc[q][threadIdx.x];
        base[threadIdx.x] += s;
        __syncthreads();
    }
}
static int radix_sort(unsigned long long **a, unsigned long long **b, long n, int nbits){
    if(n <= 1) return 0;
    const long nblk = (n + RS_TILE - 1)/RS_TILE;
    unsigned *hist; unsigned long long *off, *tot;
    TCK(DMALLOC(&hist, 256*nblk*sizeof(unsigned))); TCK(DMALLOC(&off, 256*nblk*sizeof(unsigned long long)));
    TCK(DMALLOC(&tot, sizeof(unsigned long long)));
    for(int sh = 0; sh < nbits; sh += 8){
        k_rs_hist<<<(unsigned)nblk, RS_T, 0, TS>>>(*a, n, sh, hist, nblk); TL++;
        k_scan<<<1, 256, 0, TS>>>(hist, 256*nblk, off, tot); TL++;
        k_rs_scatter<<<(unsigned)nblk, RS_T, 0, TS>>>(*a, *b, n, sh, off, nblk); TL++;
        TCK(cudaGetLastError());
        unsigned long long *t = *a; *a = *b; *b = t;
    }
    TCK(cudaStreamSynchronize(TS));
    DFREE(hist); DFREE(off); DFREE(tot);
    return 0;
}
extern "C" int sqb_radix_sort_u64(unsigned long long *keys_dev, long n, int nbits, void *stream){
    TS = (cudaStream_t)stream;
    unsigned long long *b, *a = keys_dev;
    TCK(DMALLOC(&b, (n ? n : 1)*sizeof(unsigned long long)));
    if(radix_sort(&a, &b, n, nbits)) return -1;
    if(a != keys_dev){ TCK(cudaMemcpy(keys_dev, a, n*sizeof(unsigned long long), cudaMemcpyDeviceToDevice)); DFREE(a); }
    else DFREE(b);
    return 0;
}

/* the kept list (from sqb_grow_finish) and its axis neighbours at the top step, sorted, flags merged;
 * *out is a device list of *n cells owned by the caller (sqb_dev_free) */
extern "C" int sqb_grow_dilate(int nbits, sqb_pt_t **out, long *n){
    const long n0 = GR.nkeep;
    *out = NULL; *n = 0;
    if(!n0) return 0;
    long cap = 1L << 20; while(cap < 4*n0) cap <<= 1;
    for(;;){
        unsigned long long *key, *cnt; unsigned *skb, *trm;
        TCK(DMALLOC(&key, cap*sizeof(unsigned long long))); TCK(DMALLOC(&skb, cap*sizeof(unsigned)));
        TCK(DMALLOC(&trm, cap*sizeof(unsigned))); TCK(DMALLOC(&cnt, sizeof(unsigned long long)));
        TCK(cudaMemsetAsync(key, 0, cap*sizeof(unsigned long long), TS)); TCK(cudaMemsetAsync(skb, 0xff, cap*sizeof(unsigned), TS));
        TCK(cudaMemsetAsync(trm, 0, cap*sizeof(unsigned), TS)); TCK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), TS));
        TCK(cudaMemsetAsync(GR.err, 0, sizeof(unsigned long long), TS));
        k_dil_insert<<<1184, 256, 0, TS>>>(GR.g, GR.keep, n0, key, skb, trm, (unsigned long long)(cap - 1), cnt, GR.err); TL++;
        TCK(cudaGetLastError());
        unsigned long long m = 0, e = 0;
        TCK(cudaMemcpyAsync(&m, cnt, sizeof m, cudaMemcpyDeviceToHost, TS));
        TCK(cudaMemcpyAsync(&e, GR.err, sizeof e, cudaMemcpyDeviceToHost, TS));
        TCK(cudaStreamSynchronize(TS));
        if(e || (double)m > 0.75*cap){ DFREE(key); DFREE(skb); DFREE(trm); DFREE(cnt); cap *= 2; continue; }
        unsigned long long *U, *T;
        TCK(DMALLOC(&U, m*sizeof(unsigned long long))); TCK(DMALLOC(&T, m*sizeof(unsigned long long)));
        SlotOp so; so.key = key; so.out = U; long mm = 0;
        if(compact(so, cap, &mm)) return -1;
        if(radix_sort(&U, &T, mm, nbits)) return -1;
        sqb_pt_t *o; TCK(DMALLOC(&o, mm*sizeof(sqb_pt_t)));
        k_dil_decode<<<1184, 256, 0, TS>>>(GR.g, U, mm, key, skb, trm, (unsigned long long)(cap - 1), o); TL++;
        TCK(cudaGetLastError());
        TCK(cudaStreamSynchronize(TS));
        DFREE(U); DFREE(T); DFREE(key); DFREE(skb); DFREE(trm); DFREE(cnt);
        *out = o; *n = mm;
        return 0;
    }
}

/* the kept list after sqb_grow_finish (tiers in the flag byte), on the device */
extern "C" void sqb_grow_kept(const sqb_pt_t **keep, long *m){ *keep = GR.keep; *m = GR.nkeep; }

/* top = 0 keeps no list; the kept list is released with the table */
extern "C" void sqb_grow_end(void){
    if(GR.key){ DFREE(GR.key); DFREE(GR.word); GR.key = NULL; }
    if(GR.keep){ DFREE(GR.keep); GR.keep = NULL; GR.keepcap = 0; }
    if(GR.kv){ DFREE(GR.kv); GR.kv = NULL; }
    GR.nkeep = 0;
}
