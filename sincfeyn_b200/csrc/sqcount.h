/* sqcount.h -- host-side counting number type: the generated kernels compiled over it count the
 * algorithmic FP64 operations of their double path (+ - * / each 1; negation, |.| and comparisons 0),
 * the convention of scripts/plot5_cost.py:11 ("count of the kernel's double path"). */
#pragma once
#include <math.h>
extern long sq_flops;
extern long sq_trans;      /* exp and log calls, counted apart from the flops */
struct sq_count {
    double v;
    sq_count() : v(0) {}
    sq_count(double x) : v(x) {}
    sq_count(int x) : v(x) {}
};
#define SQC_BIN(OP)                                                                                 \
static inline sq_count operator OP(const sq_count &a, const sq_count &b){ sq_flops++; return sq_count(a.v OP b.v); } \
static inline sq_count operator OP(const sq_count &a, double b){ sq_flops++; return sq_count(a.v OP b); }            \
static inline sq_count operator OP(double a, const sq_count &b){ sq_flops++; return sq_count(a OP b.v); }            \
static inline sq_count operator OP(const sq_count &a, int b){ sq_flops++; return sq_count(a.v OP b); }               \
static inline sq_count operator OP(int a, const sq_count &b){ sq_flops++; return sq_count(a OP b.v); }               \
static inline sq_count &operator OP##=(sq_count &a, const sq_count &b){ sq_flops++; a.v = a.v OP b.v; return a; }
SQC_BIN(+) SQC_BIN(-) SQC_BIN(*) SQC_BIN(/)
static inline sq_count operator-(const sq_count &a){ return sq_count(-a.v); }
#define SQC_CMP(OP)                                                                                 \
static inline bool operator OP(const sq_count &a, const sq_count &b){ return a.v OP b.v; }         \
static inline bool operator OP(const sq_count &a, int b){ return a.v OP b; }                       \
static inline bool operator OP(const sq_count &a, double b){ return a.v OP b; }
SQC_CMP(<) SQC_CMP(>) SQC_CMP(<=) SQC_CMP(>=) SQC_CMP(==) SQC_CMP(!=)
static inline sq_count sq_rabs(const sq_count &x){ return sq_count(fabs(x.v)); }
/* exp and log (the synthetic integrands) are counted in sq_trans, one each, not in the flops */
static inline sq_count sq_exp(const sq_count &x){ sq_trans++; return sq_count(exp(x.v)); }
static inline sq_count sq_log(const sq_count &x){ sq_trans++; return sq_count(log(x.v)); }
