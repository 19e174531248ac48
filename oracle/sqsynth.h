/* Test infrastructure: exp and log for the synthetic integrands (sincfeyn_b200/synth/*.c) in the oracle
 * build, where QREAL is the reference's double-double type (driver/dd.h, whose exp is only accurate to
 * double, driver/dd.h:75).  The double versions are libm's.  The double-double versions are this
 * oracle's own, written for clarity rather than speed and checked against 300-bit mpmath values
 * (tests/test_synth.py):
 *   exp: a = m ln2 + r with |r| <= ln2/2, e^r by its Taylor series to 30 terms, times 2^m;
 *   log: one Newton step x + a e^{-x} - 1 from the double logarithm of the high part. */
#pragma once
#include <math.h>
static inline double sq_exp(double x){ return exp(x); }
static inline double sq_log(double x){ return log(x); }
#if defined(QREAL_DD)
static inline dd sq_exp(const dd &a){
    if(a.hi > 709.0) return dd(INFINITY);
    if(a.hi < -745.0) return dd(0.0);
    const dd ln2(6.9314718055994529e-01, 2.3190468138462996e-17);
    const double m = nearbyint(a.hi/ln2.hi);
    const dd r = a - ln2*m;
    dd s = dd(1.0), t = dd(1.0);
    for(int n = 1; n <= 30; n++){ t = t*r/dd((double)n); s = s + t; }
    return dd(ldexp(s.hi, (int)m), ldexp(s.lo, (int)m));
}
static inline dd sq_log(const dd &a){
    if(!(a.hi > 0)) return dd(NAN);
    dd x(log(a.hi));
    return x + a*sq_exp(-x) - 1;
}
#endif
#define SQ_EXP(x) sq_exp(x)
#define SQ_LOG(x) sq_log(x)
