/* sqdd.cuh -- double-double numbers for the precision fallback, usable in device and host code.
 *
 * A value is hi + lo with |lo| <= ulp(hi)/2, about 32 significant digits.  The operations are the
 * error-free transformations of Dekker and Knuth (two-sum, quick-two-sum) and the fma two-product, as
 * published for the QD library by Hida, Li and Bailey ("Algorithms for quad-double precision floating
 * point arithmetic", 2001).  The reference evaluator fixes which variant of each operation its
 * fallback uses (driver/dd.h:18-75), and the fallback test assumes that error model, so the same
 * variants are used here:
 *   - addition is the "sloppy" form (absolute error ~2^-104 (|a|+|b|), driver/dd.h:30-32);
 *   - dd op double does not promote the double (driver/dd.h:35-36);
 *   - multiplication adds both cross terms to the low part (driver/dd.h:39-41);
 *   - division takes three quotient digits (driver/dd.h:42-47).
 * Every rounding step is an explicit round-to-nearest intrinsic on the device (and plain IEEE
 * operations on the host, compiled without contraction), so no compiler contraction can change a
 * result: the values agree bit for bit with the reference's double-double built with
 * -ffp-contract=off. */
#pragma once
#include <math.h>

#if defined(__CUDACC__)
#define SQDD_HD __host__ __device__ __forceinline__
#define SQDD_M __host__ __device__ __forceinline__
#else
#define SQDD_HD static inline
#define SQDD_M inline
#endif

#if defined(__CUDA_ARCH__)
#define SQ_ADD(a, b) __dadd_rn((a), (b))
#define SQ_SUB(a, b) __dsub_rn((a), (b))
#define SQ_MUL(a, b) __dmul_rn((a), (b))
#define SQ_DIV(a, b) __ddiv_rn((a), (b))
#define SQ_FMA(a, b, c) __fma_rn((a), (b), (c))
#else
#define SQ_ADD(a, b) ((a) + (b))
#define SQ_SUB(a, b) ((a) - (b))
#define SQ_MUL(a, b) ((a) * (b))
#define SQ_DIV(a, b) ((a) / (b))
#define SQ_FMA(a, b, c) fma((a), (b), (c))
#endif

struct sqdd {
    double hi, lo;
    SQDD_M sqdd() : hi(0), lo(0) {}
    SQDD_M sqdd(double x) : hi(x), lo(0) {}
    SQDD_M sqdd(int x) : hi((double)x), lo(0) {}
    SQDD_M sqdd(double h, double l) : hi(h), lo(l) {}
    SQDD_M double value() const { return SQ_ADD(hi, lo); }
};

/* s + e = a + b exactly (Knuth) */
SQDD_HD sqdd sqdd_two_sum(double a, double b){
    double s = SQ_ADD(a, b), bb = SQ_SUB(s, a);
    double e = SQ_ADD(SQ_SUB(a, SQ_SUB(s, bb)), SQ_SUB(b, bb));
    return sqdd(s, e);
}
/* s + e = a + b exactly, given |a| >= |b| (Dekker) */
SQDD_HD sqdd sqdd_quick_two_sum(double a, double b){
    double s = SQ_ADD(a, b);
    return sqdd(s, SQ_SUB(b, SQ_SUB(s, a)));
}
/* p + e = a * b exactly (fma) */
SQDD_HD sqdd sqdd_two_prod(double a, double b){
    double p = SQ_MUL(a, b);
    return sqdd(p, SQ_FMA(a, b, -p));
}

SQDD_HD sqdd operator+(const sqdd &a, const sqdd &b){
    sqdd s = sqdd_two_sum(a.hi, b.hi);
    s.lo = SQ_ADD(s.lo, SQ_ADD(a.lo, b.lo));
    return sqdd_quick_two_sum(s.hi, s.lo);
}
SQDD_HD sqdd sqdd_add_d(const sqdd &a, double b){
    sqdd s = sqdd_two_sum(a.hi, b);
    s.lo = SQ_ADD(s.lo, a.lo);
    return sqdd_quick_two_sum(s.hi, s.lo);
}
SQDD_HD sqdd sqdd_mul_d(const sqdd &a, double b){
    sqdd p = sqdd_two_prod(a.hi, b);
    p.lo = SQ_ADD(p.lo, SQ_MUL(a.lo, b));
    return sqdd_quick_two_sum(p.hi, p.lo);
}
SQDD_HD sqdd operator-(const sqdd &a){ return sqdd(-a.hi, -a.lo); }
SQDD_HD sqdd operator-(const sqdd &a, const sqdd &b){ return a + (-b); }
SQDD_HD sqdd operator*(const sqdd &a, const sqdd &b){
    sqdd p = sqdd_two_prod(a.hi, b.hi);
    p.lo = SQ_ADD(p.lo, SQ_ADD(SQ_MUL(a.hi, b.lo), SQ_MUL(a.lo, b.hi)));
    return sqdd_quick_two_sum(p.hi, p.lo);
}
SQDD_HD sqdd operator/(const sqdd &a, const sqdd &b){
    double q1 = SQ_DIV(a.hi, b.hi);
    sqdd r = a - b*sqdd(q1);
    double q2 = SQ_DIV(r.hi, b.hi);
    r = r - b*sqdd(q2);
    double q3 = SQ_DIV(r.hi, b.hi);
    sqdd q = sqdd_quick_two_sum(q1, q2);
    return q + sqdd(q3);
}
SQDD_HD sqdd &operator+=(sqdd &a, const sqdd &b){ a = a + b; return a; }
SQDD_HD sqdd &operator-=(sqdd &a, const sqdd &b){ a = a - b; return a; }
SQDD_HD sqdd &operator*=(sqdd &a, const sqdd &b){ a = a * b; return a; }
SQDD_HD sqdd &operator/=(sqdd &a, const sqdd &b){ a = a / b; return a; }
SQDD_HD bool operator<(const sqdd &a, const sqdd &b){ return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
SQDD_HD bool operator>(const sqdd &a, const sqdd &b){ return b < a; }
SQDD_HD bool operator<=(const sqdd &a, const sqdd &b){ return !(b < a); }
SQDD_HD bool operator>=(const sqdd &a, const sqdd &b){ return !(a < b); }
SQDD_HD bool operator==(const sqdd &a, const sqdd &b){ return a.hi == b.hi && a.lo == b.lo; }
SQDD_HD bool operator!=(const sqdd &a, const sqdd &b){ return !(a == b); }
/* mixed forms with int and double operands: the scalar is not promoted to a double-double */
SQDD_HD sqdd operator+(int a, const sqdd &b){ return sqdd_add_d(b, (double)a); }
SQDD_HD sqdd operator+(const sqdd &a, int b){ return sqdd_add_d(a, (double)b); }
SQDD_HD sqdd operator-(int a, const sqdd &b){ return sqdd_add_d(-b, (double)a); }
SQDD_HD sqdd operator-(const sqdd &a, int b){ return sqdd_add_d(a, -(double)b); }
SQDD_HD sqdd operator*(int a, const sqdd &b){ return sqdd_mul_d(b, (double)a); }
SQDD_HD sqdd operator*(const sqdd &a, int b){ return sqdd_mul_d(a, (double)b); }
SQDD_HD sqdd operator/(int a, const sqdd &b){ return sqdd((double)a) / b; }
SQDD_HD sqdd operator/(const sqdd &a, int b){ return a / sqdd((double)b); }
SQDD_HD sqdd operator+(double a, const sqdd &b){ return sqdd_add_d(b, a); }
SQDD_HD sqdd operator+(const sqdd &a, double b){ return sqdd_add_d(a, b); }
SQDD_HD sqdd operator-(double a, const sqdd &b){ return sqdd_add_d(-b, a); }
SQDD_HD sqdd operator-(const sqdd &a, double b){ return sqdd_add_d(a, -b); }
SQDD_HD sqdd operator*(double a, const sqdd &b){ return sqdd_mul_d(b, a); }
SQDD_HD sqdd operator*(const sqdd &a, double b){ return sqdd_mul_d(a, b); }
SQDD_HD bool operator<(const sqdd &a, int b){ return a < sqdd((double)b); }
SQDD_HD bool operator>(const sqdd &a, int b){ return a > sqdd((double)b); }
SQDD_HD bool operator!=(const sqdd &a, int b){ return a != sqdd((double)b); }
SQDD_HD bool operator==(const sqdd &a, int b){ return a == sqdd((double)b); }

/* |x| with the reference's RABS semantics (x < 0 ? -x : x, driver/common.h:23) */
SQDD_HD sqdd sq_rabs(const sqdd &x){ return x < sqdd(0.0) ? -x : x; }
/* in double the sign of a zero never reaches a result (every |.| value is only added and multiplied
 * into non-negative sums), so the single sign-clearing instruction is used */
SQDD_HD double sq_rabs(double x){ return fabs(x); }

/* e^a in double-double, by the method of argument reduction and repeated squaring published for
 * double-double arithmetic by Hida, Li and Bailey (2001): a = m ln2 + r with m = rint(a/ln2), r scaled
 * by 2^-10 (|r| <= 3.4e-4), e^r - 1 by its Taylor series to degree 9 in Horner form (truncation below
 * 1e-33 relative), ten doublings e^{2x} - 1 = (e^x - 1)(e^x + 1), then (1 + s) 2^m.  ln 2 is a
 * triple-double and 1/n! double-double roundings of 300-bit values.  Relative error about 1e-32 for
 * |a| <= 700 while the result's low part stays normal (|a| <= ~670).  Every step is a double-double operation of this file,
 * so host and device results agree bit for bit. */
SQDD_HD sqdd sqdd_exp(const sqdd &a){
    if(a.hi > 709.0) return sqdd(exp(a.hi));          /* overflow: +inf */
    if(a.hi < -745.0) return sqdd(0.0);
    const sqdd LN2(6.9314718055994529e-01, 2.3190468138462996e-17);
    const double LN2C = 5.7077084384162121e-34;        /* third term of ln 2: r stays accurate for |m| ~ 1000 */
    const double m = rint(SQ_DIV(a.hi, LN2.hi));
    sqdd r = a - LN2*m;
    r = sqdd_add_d(r, -SQ_MUL(LN2C, m));
    r = sqdd(SQ_MUL(r.hi, 0x1p-10), SQ_MUL(r.lo, 0x1p-10));
    const sqdd C[7] = {
    /* 1/9! */ sqdd(2.7557319223985893e-06, -1.8583932740464721e-22),
    /* 1/8! */ sqdd(2.4801587301587302e-05, 2.1511947866775882e-23),
    /* 1/7! */ sqdd(0.00019841269841269841, 1.7209558293420705e-22),
    /* 1/6! */ sqdd(0.0013888888888888889, -5.3005439543735771e-20),
    /* 1/5! */ sqdd(0.0083333333333333332, 1.1564823173178714e-19),
    /* 1/4! */ sqdd(0.041666666666666664, 2.3129646346357427e-18),
    /* 1/3! */ sqdd(0.16666666666666666, 9.2518585385429707e-18),
    };
    sqdd s = C[0];
    for(int i = 1; i < 7; i++) s = s*r + C[i];
    s = s*r + 0.5;
    s = s*r + 1.0;
    s = s*r;
    for(int i = 0; i < 10; i++) s = s*(s + 2.0);
    s = s + 1.0;
    return sqdd(ldexp(s.hi, (int)m), ldexp(s.lo, (int)m));
}
/* log a in double-double: one Newton step x + a e^{-x} - 1 from the double logarithm of the high part */
SQDD_HD sqdd sqdd_log(const sqdd &a){
    if(!(a.hi > 0)) return sqdd(log(a.hi));
    const sqdd x(log(a.hi));
    return x + a*sqdd_exp(-x) - 1;
}
/* exp and log for the integrands that need them (SQ_EXP, SQ_LOG): the double versions are the math
 * library's, the double-double versions the ones above */
SQDD_HD double sq_exp(double x){ return exp(x); }
SQDD_HD double sq_log(double x){ return log(x); }
SQDD_HD sqdd sq_exp(const sqdd &x){ return sqdd_exp(x); }
SQDD_HD sqdd sq_log(const sqdd &x){ return sqdd_log(x); }
