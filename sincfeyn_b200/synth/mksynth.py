#!/usr/bin/env python3
"""Writes the synthetic Sinc-sum integrands in the generated-kernel format (one file per dimension).

    f(z) = prod_i sech(a_i z_i + b_i) * (exp(eps * sum_i exp(-|z_i|)) - 1) / eps,   eps = 1e-9

with the expm1 term computed naively (exp, then subtract 1) so that it cancels catastrophically, and
the sum of |terms| for the precision test (exp(x) + 1)/eps * prod_i sech.  The parameters are drawn
from splitmix64 (seed 1, 2, 3 for d = 5, 8, 11): a_i = 0.5 + 1.5 u, b_i = -1 + 2 u with
u = (next() >> 11) * 2^-53, all a_i first, then all b_i.

The files follow the layout of the reference's generated kernels (a double half and a QREAL half over
the REAL/FN macros, and a `const graph_t G_<name>` descriptor), so that the evaluator's code generator
compiles them like every other graph and the reference's own hsum() can run them as extra registry
entries (the CPU baseline).  The lattice gives s = e^z; the integrand takes z = log s and divides by
prod s, so that the driver's weight prod(s h) leaves f(z) h^d.  exp and log come from SQ_EXP/SQ_LOG,
which each build defines for double and for its double-double type.

    python3 sincfeyn_b200/synth/mksynth.py        # rewrites syn_d5.c, syn_d8.c, syn_d11.c here
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))
DIMS = {5: 1, 8: 2, 11: 3}
M64 = (1 << 64) - 1


def splitmix64(seed):
    s = seed & M64
    while True:
        s = (s + 0x9E3779B97F4A7C15) & M64
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        yield z ^ (z >> 31)


def params(d):
    g = splitmix64(DIMS[d])
    u = [(next(g) >> 11) * 2.0**-53 for _ in range(2*d)]
    return [0.5 + 1.5*x for x in u[:d]], [-1.0 + 2.0*x for x in u[d:]]


def half(name, d, real):
    return '''#define REAL %(real)s
#define FN(x) x##_%(sfx)s
static REAL FN(f_%(n)s)(const REAL *sf, REAL *ab){
  REAL x=0, p=1, js=1;
  for(int i=0;i<%(d)d;i++){
    const REAL z=SQ_LOG(sf[i]);
    const REAL e=SQ_EXP(SYA_%(n)s[i]*z+SYB_%(n)s[i]);
    p=p*2/(e+1/e);
    x=x+SQ_EXP(-RABS(z));
    js=js*sf[i];
  }
  const REAL ex=SQ_EXP(x*1e-9);
  *ab=(ex+1)*1e9*p/js;
  return (ex-1)*1e9*p/js;
}
#undef REAL
#undef FN
''' % dict(real=real, sfx='d' if real == 'double' else 'q', n=name, d=d)


def source(d):
    name = 'syn_d%d' % d
    a, b = params(d)
    fmt = lambda v: ','.join('%.17g' % x for x in v)
    return '\n'.join([
        '/* Synthetic Sinc-sum integrand, d = %d, splitmix64 seed %d: written by sincfeyn_b200/synth/mksynth.py */' % (d, DIMS[d]),
        '#include "common.h"', '#include "sqsynth.h"',
        'static const double SYA_%s[%d]={%s};' % (name, d, fmt(a)),
        'static const double SYB_%s[%d]={%s};' % (name, d, fmt(b)),
        half(name, d, 'double') + half(name, d, 'QREAL') +
        'const graph_t G_%s={"%s","synthetic sech expm1 d=%d",0,%d,1,%d,0,f_%s_d,f_%s_q,0,0};' % (name, name, d, d, d, name, name),
        ''])


if __name__ == '__main__':
    for d in DIMS:
        with open(os.path.join(HERE, 'syn_d%d.c' % d), 'w') as f:
            f.write(source(d))
