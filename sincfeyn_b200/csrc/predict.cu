/* predict.cu -- the last-level predictor (SINCQED_PREDICT = alpha, driver/sum.c:64-140, 379-422) on the
 * device.
 *
 * The table of step-2h values.  Every point the grow evaluates (|f w|, tier 0), then -- after the grow's
 * shadow-tier flood fill -- the origin (tier 2) and the axis neighbours of every kept point of tier t
 * (raised to t), then every child evaluated at the level before the last (tier = its parent's; under a
 * symmetry fold the whole orbit): a key of the point's coordinates (vhash, driver/sum.c:88-92) with the
 * float log of the value and the tier, in open addressing on 16-byte slots at (key >> 17) mod capacity.
 * A later insert of the same point overwrites the earlier one, as the reference's vput does.  The slots
 * have the bytes of the reference's vslot_t, so a table goes into and out of SQCK4 checkpoints as it is.
 *
 * The prediction (driver/sum.c:379-422).  Child k - st b of a cell k at the last level is the centre of
 * the 2 st cube whose corners are k - 2 st c for the subsets c of b; the mean over those corners of the
 * stored |f| (a corner never stored counts as thr) is formed for all b at once by a subset-sum transform
 * over the 2^D corners, in the reference's order (bit 0 first, then bit 1, ...; each pass adds
 * st[c ^ bit] into st[c] for the c that have the bit), and divided by 2^|b|.  A child whose mean is below
 * alpha thr is not evaluated (counted as predicted); with the shadow runs on, the same means with the
 * eps*10 and eps*100 thresholds cap the child's tier.  One warp per cell; the corner sums sit in shared
 * memory.  The result is one byte per child of the batch: bit 0 = not evaluated, bits 1-2 = its tier. */
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>
#include "sqb_rt.h"
#include "sqorbit.cuh"

struct VSlot { unsigned long long k; float v; unsigned t; };   /* the reference's vslot_t bytes (t < 256) */
static_assert(sizeof(VSlot) == 16, "one slot is 16 bytes, as the checkpoint stores it");

static thread_local char perr[256];
extern "C" const char *sqb_vtab_error(void){ return perr; }
#define PCK(x) do { cudaError_t e_ = (x); if(e_ != cudaSuccess){ snprintf(perr, sizeof perr, "%s: %s", #x, cudaGetErrorString(e_)); return -1; } } while(0)

__device__ __forceinline__ unsigned long long v_hash(const int *k, int D){
    unsigned long long y = 0x9E3779B97F4A7C15ULL;
    for(int i = 0; i < D; i++){
        y ^= (unsigned long long)(unsigned)k[i] + 0x9E3779B97F4A7C15ULL + (y << 6) + (y >> 2);
        y *= 0xBF58476D1CE4E5B9ULL;
    }
    return y | 1;
}
__device__ __forceinline__ long v_pos(unsigned long long y, long cap){ return (long)(y >> 17) & (cap - 1); }

/* insert or overwrite; the probe is bounded by the capacity (a full table counts a failure) */
__device__ void v_put(VSlot *T, long cap, unsigned long long y, float v, unsigned t, unsigned long long *vn,
                      unsigned long long *full){
    long i = v_pos(y, cap);
    for(long n = 0; n < cap; n++){
        const unsigned long long c = atomicCAS(&T[i].k, 0ULL, y);
        if(c == 0ULL || c == y){
            if(c == 0ULL) atomicAdd(vn, 1ULL);
            T[i].v = v; T[i].t = t;
            return;
        }
        i = (i + 1) & (cap - 1);
    }
    atomicAdd(full, 1ULL);
}
/* 0 if absent, else 1 + tier, and the stored log value */
__device__ __forceinline__ int v_get(const VSlot *T, long cap, unsigned long long y, float *lv){
    long i = v_pos(y, cap);
    for(long n = 0; n < cap; n++){
        const unsigned long long c = T[i].k;
        if(!c) return 0;
        if(c == y){ *lv = T[i].v; return 1 + (int)T[i].t; }
        i = (i + 1) & (cap - 1);
    }
    return 0;
}
__device__ void v_raise(VSlot *T, long cap, unsigned long long y, unsigned t){
    long i = v_pos(y, cap);
    for(long n = 0; n < cap; n++){
        const unsigned long long c = T[i].k;
        if(!c) return;
        if(c == y){ atomicMax(&T[i].t, t); return; }
        i = (i + 1) & (cap - 1);
    }
}
__device__ __forceinline__ float v_log(double a){ return (float)log(a > 1e-300 ? a : 1e-300); }

__global__ void k_vput_nodes(const sqb_pt_t *pts, const double *v, long n, int D, VSlot *T, long cap,
                             unsigned long long *vn, unsigned long long *full){
    for(long i = blockIdx.x*(long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x*blockDim.x){
        int k[SQB_MAXD];
        for(int d = 0; d < D; d++) k[d] = pts[i].k[d];
        v_put(T, cap, v_hash(k, D), v_log(fabs(v[i])), 0, vn, full);
    }
}

/* after the grow's tiers: the origin to tier 2, the in-box axis neighbours of each kept point of tier t
 * to t (driver/sumkey.h:445-451) */
__global__ void k_vraise_kept(const sqb_pt_t *keep, long m, int D, int st, int K, VSlot *T, long cap){
    const long i0 = blockIdx.x*(long)blockDim.x + threadIdx.x;
    if(i0 == 0){ int z[SQB_MAXD] = {0}; v_raise(T, cap, v_hash(z, D), 2); }
    for(long i = i0; i < m; i += (long)gridDim.x*blockDim.x){
        const unsigned t = (unsigned)((keep[i].k[SQB_PFLAG] >> 1) & 3);
        if(!t) continue;
        int k[SQB_MAXD];
        for(int d = 0; d < D; d++) k[d] = keep[i].k[d];
        for(int d = 0; d < D; d++) for(int sg = -1; sg <= 1; sg += 2){
            const int o = k[d]; k[d] = o + st*sg;
            if(k[d] <= K && k[d] >= -K) v_raise(T, cap, v_hash(k, D), t);
            k[d] = o;
        }
    }
}

/* the children evaluated at the level before the last (driver/sum.c:738-740): |v| with the parent's
 * tier, and under a fold the other members of the child's orbit with the same value */
__global__ void k_vput_children(const signed char *cells, long nch, int D, int st, const double *v,
                                const unsigned char *stt, sqb_sym_t sym, VSlot *T, long cap,
                                unsigned long long *vn, unsigned long long *full){
    for(long i = blockIdx.x*(long)blockDim.x + threadIdx.x; i < nch; i += (long)gridDim.x*blockDim.x){
        if(!(stt[i] & SQB_PRESENT)) continue;
        const long c = i >> D; const int b = (int)(i & ((1L << D) - 1));
        const signed char *p = cells + c*SQB_MAXD;
        int k[SQB_MAXD], im[SQB_MAXD];
        for(int d = 0; d < D; d++) k[d] = p[d] - (((b >> d) & 1) ? st : 0);
        const unsigned t = (unsigned)((p[SQB_PFLAG] >> 1) & 3);
        const float lv = v_log(fabs(v[i]));
        const int ng = sym.n > 1 ? sym.n : 1;
        for(int e = 0; e < ng; e++){
            if(!sqb_image_new(sym, k, D, e)) continue;
            sqb_image(sym, k, D, e, im);
            v_put(T, cap, v_hash(im, D), lv, t, vn, full);
        }
    }
}

__global__ void k_vrehash(const VSlot *O, long ocap, VSlot *T, long cap, unsigned long long *vn, unsigned long long *full){
    for(long i = blockIdx.x*(long)blockDim.x + threadIdx.x; i < ocap; i += (long)gridDim.x*blockDim.x)
        if(O[i].k) v_put(T, cap, O[i].k, O[i].v, O[i].t, vn, full);
}

/* the prediction for the cells of one last-level batch: cfl[(c - c0) << D | b] for the batch's cells */
__global__ void __launch_bounds__(32) k_predict(const signed char *cells, long ncell, int D, int st, int K,
                                                double thr, double alpha, int esok, sqb_sym_t sym,
                                                const VSlot *T, long cap, unsigned char *cfl,
                                                unsigned long long *pskip){
    extern __shared__ double pm[];
    const int nc = 1 << D, l = threadIdx.x;
    double *s0 = pm, *s1 = pm + nc, *s2 = pm + 2*nc;
    for(long c = blockIdx.x; c < ncell; c += gridDim.x){
        const signed char *p = cells + c*SQB_MAXD;
        int kp[SQB_MAXD];
        for(int d = 0; d < D; d++) kp[d] = p[d];
        const int tp = (p[SQB_PFLAG] >> 1) & 3;
        for(int cc = l; cc < nc; cc += 32){
            int kn[SQB_MAXD];
            for(int d = 0; d < D; d++) kn[d] = kp[d] - (((cc >> d) & 1) ? 2*st : 0);
            float lv = 0;
            const int f = v_get(T, cap, v_hash(kn, D), &lv);
            s0[cc] = f ? exp((double)lv) : thr;
            if(esok){ s1[cc] = f >= 2 ? s0[cc] : 10*thr; s2[cc] = f >= 3 ? s0[cc] : 100*thr; }
        }
        __syncwarp();
        for(int d = 0; d < D; d++){
            for(int cc = l; cc < nc; cc += 32) if((cc >> d) & 1){
                s0[cc] += s0[cc ^ (1 << d)];
                if(esok){ s1[cc] += s1[cc ^ (1 << d)]; s2[cc] += s2[cc ^ (1 << d)]; }
            }
            __syncwarp();
        }
        for(int cc = l; cc < nc; cc += 32){
            const double dv = (double)(1 << __popc(cc));
            s0[cc] /= dv;
            if(esok){ s1[cc] /= dv; s2[cc] /= dv; }
        }
        __syncwarp();
        unsigned nsk = 0;
        for(int b = l; b < nc; b += 32){
            int k[SQB_MAXD]; bool in = true;
            for(int d = 0; d < D; d++){ k[d] = kp[d] - (((b >> d) & 1) ? st : 0); if(k[d] < -K) in = false; }
            unsigned char out = (unsigned char)(tp << 1);
            if(in){
                const bool canon = sym.n <= 1 || sqb_orbit_n(sym, k, D) > 0;
                if(canon && s0[b] < alpha*thr){ out = 1; nsk++; }
                else if(canon && esok){
                    const int tq = (s1[b] >= alpha*10*thr) + (s1[b] >= alpha*10*thr && s2[b] >= alpha*100*thr);
                    out = (unsigned char)((tq < tp ? tq : tp) << 1);
                }
            }
            cfl[(c << D) + b] = out;
        }
        for(int off = 16; off; off >>= 1) nsk += __shfl_down_sync(0xffffffffu, nsk, off);
        if(l == 0 && nsk) atomicAdd(pskip, (unsigned long long)nsk);
        __syncwarp();
    }
}

/* ------------------------------------------- host side ------------------------------------------ */
static int vt_alloc(sqb_vtab_t *t, long cap, cudaStream_t s){
    void *p = NULL;
    PCK(cudaMallocAsync(&p, (size_t)cap*sizeof(VSlot), s));
    PCK(cudaMemsetAsync(p, 0, (size_t)cap*sizeof(VSlot), s));
    t->tab = p; t->cap = cap;
    return 0;
}
extern "C" int sqb_vtab_reserve(sqb_vtab_t *t, long more, void *stream){
    cudaStream_t s = (cudaStream_t)stream;
    if(!t->vn){
        PCK(cudaMallocAsync((void**)&t->vn, 2*sizeof(unsigned long long), s));
        PCK(cudaMemsetAsync(t->vn, 0, 2*sizeof(unsigned long long), s));
        t->full = t->vn + 1;
    }
    unsigned long long n = 0;
    PCK(cudaMemcpyAsync(&n, t->vn, sizeof n, cudaMemcpyDeviceToHost, s));
    PCK(cudaStreamSynchronize(s));
    const double need = 4.0/3.0*((double)n + (double)more);          /* at most 3/4 full */
    if(t->tab && (double)t->cap >= need) return 0;
    long cap = t->cap ? t->cap : (1L << 20);
    while((double)cap < need) cap <<= 1;
    sqb_vtab_t o = *t;
    if(vt_alloc(t, cap, s)) return -1;
    PCK(cudaMemsetAsync(t->vn, 0, sizeof(unsigned long long), s));
    if(o.tab){
        k_vrehash<<<1184, 256, 0, s>>>((const VSlot*)o.tab, o.cap, (VSlot*)t->tab, cap, t->vn, t->full);
        PCK(cudaGetLastError());
        cudaFreeAsync(o.tab, s);
    }
    return 0;
}
extern "C" int sqb_vtab_put_nodes(sqb_vtab_t *t, const sqb_pt_t *pts, const double *v, long n, int D, void *stream){
    if(n <= 0) return 0;
    k_vput_nodes<<<1184, 256, 0, (cudaStream_t)stream>>>(pts, v, n, D, (VSlot*)t->tab, t->cap, t->vn, t->full);
    PCK(cudaGetLastError());
    return 0;
}
extern "C" int sqb_vtab_raise_kept(sqb_vtab_t *t, const sqb_pt_t *keep, long m, int D, int st, int K, void *stream){
    if(!t->tab) return 0;
    k_vraise_kept<<<1184, 256, 0, (cudaStream_t)stream>>>(keep, m, D, st, K, (VSlot*)t->tab, t->cap);
    PCK(cudaGetLastError());
    return 0;
}
extern "C" int sqb_vtab_put_children(sqb_vtab_t *t, const void *cells, long nch, int D, int st, const double *v,
                                     const unsigned char *stt, const sqb_sym_t *sym, void *stream){
    if(nch <= 0) return 0;
    sqb_sym_t s; memset(&s, 0, sizeof s); if(sym && sym->n > 1) s = *sym;
    k_vput_children<<<1184, 256, 0, (cudaStream_t)stream>>>((const signed char*)cells, nch, D, st, v, stt, s,
                                                             (VSlot*)t->tab, t->cap, t->vn, t->full);
    PCK(cudaGetLastError());
    return 0;
}
extern "C" int sqb_vtab_predict(const sqb_vtab_t *t, const void *cells, long ncell, int D, int st, int K, double thr,
                                double alpha, int esok, const sqb_sym_t *sym, unsigned char *cfl,
                                unsigned long long *pskip, int nsm, void *stream){
    if(ncell <= 0) return 0;
    sqb_sym_t s; memset(&s, 0, sizeof s); if(sym && sym->n > 1) s = *sym;
    const size_t smem = 3*sizeof(double) << D;
    if(smem > 48*1024){ snprintf(perr, sizeof perr, "predictor: D = %d needs %zu bytes of shared memory per cell", D, smem); return -1; }
    const long want = ncell, full = (long)nsm*32;
    k_predict<<<(unsigned)(want < full ? want : full), 32, smem, (cudaStream_t)stream>>>((const signed char*)cells, ncell, D, st, K,
                                                                                       thr, alpha, esok, s, (const VSlot*)t->tab,
                                                                                       t->cap, cfl, pskip);
    PCK(cudaGetLastError());
    return 0;
}
/* keys stored, and inserts that found the table full (both synchronise the stream) */
extern "C" int sqb_vtab_counts(const sqb_vtab_t *t, long *vn, long *full, void *stream){
    *vn = 0; *full = 0;
    if(!t->vn) return 0;
    unsigned long long h[2];
    PCK(cudaMemcpyAsync(h, t->vn, sizeof h, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    PCK(cudaStreamSynchronize((cudaStream_t)stream));
    *vn = (long)h[0]; *full = (long)h[1];
    return 0;
}
/* the slots to or from host memory (cap slots of 16 bytes: the checkpoint's predictor table) */
extern "C" int sqb_vtab_download(const sqb_vtab_t *t, void *host, void *stream){
    if(!t->tab) return 0;
    PCK(cudaMemcpyAsync(host, t->tab, (size_t)t->cap*sizeof(VSlot), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    PCK(cudaStreamSynchronize((cudaStream_t)stream));
    return 0;
}
extern "C" int sqb_vtab_upload(sqb_vtab_t *t, const void *host, long cap, long vn, void *stream){
    cudaStream_t s = (cudaStream_t)stream;
    if(cap <= 0 || (cap & (cap - 1))) return 0;
    if(sqb_vtab_reserve(t, 0, stream)) return -1;
    if(t->tab) cudaFreeAsync(t->tab, s);
    t->tab = NULL; t->cap = 0;
    if(vt_alloc(t, cap, s)) return -1;
    PCK(cudaMemcpyAsync(t->tab, host, (size_t)cap*sizeof(VSlot), cudaMemcpyHostToDevice, s));
    const unsigned long long h[2] = {(unsigned long long)vn, 0ULL};
    PCK(cudaMemcpyAsync(t->vn, h, sizeof h, cudaMemcpyHostToDevice, s));
    PCK(cudaStreamSynchronize(s));
    return 0;
}
extern "C" void sqb_vtab_free(sqb_vtab_t *t, void *stream){
    if(t->tab) cudaFreeAsync(t->tab, (cudaStream_t)stream);
    if(t->vn) cudaFreeAsync(t->vn, (cudaStream_t)stream);
    memset(t, 0, sizeof *t);
}
