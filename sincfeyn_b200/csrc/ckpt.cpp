/* ckpt.cpp -- the reference's checkpoint file, format SQCK4 (driver/checkpoint.c:59-120).
 *
 * The file is the fields of ckpt_t (driver/sq.h:84-93) written one after another in native byte order
 * (x86-64: little-endian, int 4 bytes, long 8 bytes): the 72-byte header ckhead_t {char magic[8] =
 * "SQCK4", char name[32]; double h, eps; int N, top, dim, k}, then lev, next, s, a, drop, u, ne, q,
 * Slev[16], nl, res_t (96 bytes), the cell lists cur and nxt (a long count, then 12-byte pt_t cells),
 * es[5], cnt[3], esok, vsz, vcap, vn and vcap slots of vsz bytes.  Reader and writer here are this
 * project's own; the layout is the reference's because the files are exchanged with it. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "sincfeyn_b200.h"

namespace {

struct Head { char magic[8], name[32]; double h, eps; int N, top, dim, k; };
static_assert(sizeof(Head) == 72, "ckhead_t is 72 bytes");
struct Res { double S[3], Ah, ref, prune, trunc, unres, t; long nev, nq, kept_top; };
static_assert(sizeof(Res) == 96, "res_t is 96 bytes");
static_assert(sizeof(long) == 8 && sizeof(int) == 4, "LP64 layout");
const int PT = 12;                      /* sizeof(pt_t) at MAXD = 12 */

struct W {
    FILE *f; bool ok = true;
    template<class T> void put(const T &x){ if(ok) ok = fwrite(&x, sizeof x, 1, f) == 1; }
    void raw(const void *p, size_t sz, size_t n){ if(ok && n) ok = fwrite(p, sz, n, f) == n; }
};
struct R {
    FILE *f; bool ok = true;
    template<class T> void get(T &x){ if(ok) ok = fread(&x, sizeof x, 1, f) == 1; }
    void raw(void *p, size_t sz, size_t n){ if(ok && n) ok = fread(p, sz, n, f) == n; }
};

Head head_of(const sqb_ckpt_t *c){
    Head h; memset(&h, 0, sizeof h);
    memcpy(h.magic, "SQCK4", 6);
    snprintf(h.name, sizeof h.name, "%s", c->name);
    h.h = c->h; h.eps = c->eps; h.N = c->N; h.top = c->top; h.dim = c->dim; h.k = c->k;
    return h;
}

bool read_cells(R &r, long *n, signed char **p){
    long m = -1; r.get(m);
    if(!r.ok || m < 0) return false;
    *p = (signed char*)malloc((size_t)(m ? m : 1)*PT);
    if(!*p) return false;
    *n = m;
    r.raw(*p, PT, (size_t)m);
    return r.ok;
}

}  // namespace

extern "C" void sqb_ckpt_name(char *buf, size_t n, const char *dir, const char *graph){
    snprintf(buf, n, "%s/sincqed_%s.ckpt", dir && *dir ? dir : ".", graph);
}

extern "C" int sqb_ckpt_save(const char *path, const sqb_ckpt_t *c){
    char tmp[4200]; snprintf(tmp, sizeof tmp, "%s.tmp", path);
    FILE *f = fopen(tmp, "wb");
    if(!f) return -1;
    W w; w.f = f;
    Head h = head_of(c); w.put(h);
    w.put(c->lev); w.put(c->next);
    w.put(c->s); w.put(c->a); w.put(c->drop); w.put(c->u); w.put(c->ne); w.put(c->q);
    w.raw(c->Slev, sizeof(double), 16); w.put(c->nl);
    Res rs; memcpy(rs.S, c->S, sizeof rs.S); rs.Ah = c->Ah; rs.ref = c->ref; rs.prune = c->prune;
    rs.trunc = c->trunc; rs.unres = c->unres; rs.t = c->t; rs.nev = c->nev; rs.nq = c->nq; rs.kept_top = c->kept_top;
    w.put(rs);
    w.put(c->ncur); w.raw(c->cur, PT, (size_t)c->ncur);
    w.put(c->nnxt); w.raw(c->nxt, PT, (size_t)c->nnxt);
    w.raw(c->es, sizeof(double), 5); w.raw(c->cnt, sizeof(long), 3); w.put(c->esok);
    w.put(c->vsz); w.put(c->vcap); w.put(c->vn);
    if(c->vcap > 0) w.raw(c->vs, (size_t)c->vsz, (size_t)c->vcap);
    bool ok = (fclose(f) == 0) && w.ok;
    if(!ok || rename(tmp, path)){ remove(tmp); return -1; }
    return 0;
}

extern "C" void sqb_ckpt_free(sqb_ckpt_t *c){
    free(c->cur); free(c->nxt); free(c->vs);
    c->cur = c->nxt = NULL; c->vs = NULL; c->ncur = c->nnxt = 0;
}

extern "C" int sqb_ckpt_load(const char *path, sqb_ckpt_t *c){
    memset(c, 0, sizeof *c);
    FILE *f = fopen(path, "rb");
    if(!f) return 0;
    R r; r.f = f;
    Head h; r.get(h);
    if(!r.ok || memcmp(h.magic, "SQCK4\0\0", 8)){ fclose(f); return -1; }
    memcpy(c->name, h.name, sizeof c->name); c->name[31] = 0;
    c->h = h.h; c->eps = h.eps; c->N = h.N; c->top = h.top; c->dim = h.dim; c->k = h.k;
    r.get(c->lev); r.get(c->next);
    r.get(c->s); r.get(c->a); r.get(c->drop); r.get(c->u); r.get(c->ne); r.get(c->q);
    r.raw(c->Slev, sizeof(double), 16); r.get(c->nl);
    Res rs; r.get(rs);
    if(r.ok){
        memcpy(c->S, rs.S, sizeof rs.S); c->Ah = rs.Ah; c->ref = rs.ref; c->prune = rs.prune; c->trunc = rs.trunc;
        c->unres = rs.unres; c->t = rs.t; c->nev = rs.nev; c->nq = rs.nq; c->kept_top = rs.kept_top;
    }
    bool ok = r.ok && read_cells(r, &c->ncur, &c->cur) && read_cells(r, &c->nnxt, &c->nxt);
    if(ok){
        r.raw(c->es, sizeof(double), 5); r.raw(c->cnt, sizeof(long), 3); r.get(c->esok);
        r.get(c->vsz); r.get(c->vcap); r.get(c->vn);
        ok = r.ok && c->vsz == SQB_CKPT_VSLOT && c->vcap >= 0 && (c->vcap & (c->vcap - 1)) == 0 && c->nl >= 0 && c->nl <= 16;
        if(ok && c->vcap){
            c->vs = malloc((size_t)c->vcap*c->vsz);
            ok = c->vs != NULL;
            if(ok){ r.raw(c->vs, (size_t)c->vsz, (size_t)c->vcap); ok = r.ok; }
        }
    }
    fclose(f);
    if(!ok){ sqb_ckpt_free(c); return -1; }
    return 1;
}
