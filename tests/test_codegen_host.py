"""The kernel code generator (sincfeyn_b200/codegen/kgen.py) checked on the CPU: its output for every
graph, compiled for the host over double and over the double-double type of the device code
(sincfeyn_b200/csrc/sqdd.cuh), without FP contraction, reproduces the reference kernels' values bit for
bit at the seeded nodes of the golden fixtures (the double half f_d with SQ_AB = 1 and 0, and the
double-double fq).  This is the same arithmetic the sm_100a build runs with -fmad=false."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GEN = os.path.join(ROOT, 'sincfeyn_b200', '_build', 'gen')
CSRC = os.path.join(ROOT, 'sincfeyn_b200', 'csrc')
GOLD = os.path.join(ROOT, 'tests', 'golden')
OUT = os.path.join(ROOT, 'tests', '_hostgen')
# graphs whose double half is a differently compacted copy of the integrand: kgen compiles the QREAL
# half, so their FP64 values agree with the reference's double half only to rounding, checked against
# 4 ulp of the |.| sum (and the |.| sum itself to 1e-12 relative; the double-double half is the same text
# and stays bit for bit)
NOT_BITWISE = {'g3_lbl': 'pt4_g3_lbl (double half) and pt_g3_lbl (QREAL half) are compacted differently'}

SRC = r'''
#include <math.h>
#include "sqdd.cuh"
#define SQ_TABLE static const
#define SQ_FUNC
#define SQ_FUNC_K
#define SQ_CHUNK
#define SQ_CHUNK_DD
#define RABS(x) sq_rabs(x)
#define SQ_EXP(x) sq_exp(x)
#define SQ_LOG(x) sq_log(x)
#define SQG_NS(n) sqg_##n
#define SQ_GRAPH_SPLIT(NAME, VOLKOV, L, D, W, NP, FIX, NPARTS) SQ_GRAPH(NAME, VOLKOV, L, D, W, NP, FIX)
#define SQ_SCALE(NAME)
#define SQ_GRAPH(NAME, VOLKOV, L, D, W, NP, FIX)                                                    \
extern "C" int hg_##NAME(long n, const double *sf, int prec, int ab, double *f, double *a){       \
    for(long i = 0; i < n; i++){                                                                   \
        if(prec == 0){ double s[D], x = 0; for(int d = 0; d < D; d++) s[d] = sf[i*D + d];           \
            f[i] = ab ? sqg_##NAME::K<double, 1>::f_##NAME(s, &x) : sqg_##NAME::K<double, 0>::f_##NAME(s, &x); a[i] = x; } \
        else { sqdd s[D], x; for(int d = 0; d < D; d++) s[d] = sqdd(sf[i*D + d]);                   \
            sqdd v = sqg_##NAME::K<sqdd, 1>::f_##NAME(s, &x);                                      \
            f[2*i] = v.hi; f[2*i + 1] = v.lo; a[2*i] = x.hi; a[2*i + 1] = x.lo; } }              \
    return D; }
'''


def hostlib(names):
    os.makedirs(OUT, exist_ok=True)
    tag = '%d_%s' % (len(names), names[0])
    so = os.path.join(OUT, 'hostgen_%s.so' % tag)
    cuhs = [os.path.join(GEN, n + '.cuh') for n in names]
    if not os.path.exists(so) or any(os.path.getmtime(c) > os.path.getmtime(so) for c in cuhs + [os.path.join(CSRC, 'sqdd.cuh')]):
        cc = os.path.join(OUT, 'hostgen_%s.cc' % tag)
        with open(cc, 'w') as f:
            f.write(SRC + ''.join('#include "%s"\n' % c for c in cuhs))
        subprocess.run(['g++', '-O0', '-ffp-contract=off', '-std=c++17', '-shared', '-fPIC', '-I' + CSRC,
                        '-o', so, cc], check=True)
    return C.CDLL(so)


@pytest.mark.parametrize('cls', ['g2', 'v3', 'g3', 'v4', 'w4'])
def test_generated_kernels_match_the_reference_bitwise(cls):
    z = np.load(os.path.join(GOLD, 'pointwise_%s.npz' % cls))
    names = sorted({k.split('.')[0] for k in z.files})
    have = [n for n in names if os.path.exists(os.path.join(GEN, n + '.cuh'))]
    if not have:
        pytest.skip('no generated kernels for %s (python -m sincfeyn_b200.build)' % cls)
    L = hostlib(have)
    for n in have:
        sf = np.ascontiguousarray(z[n + '.sf'])
        m = sf.shape[0]
        fn = getattr(L, 'hg_' + n)
        fn.argtypes = [C.c_long, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        for ab, key in ((1, '.fd1'), (0, '.fd0')):
            f = np.empty(m); a = np.empty(m)
            fn(m, sf.ctypes.data, 0, ab, f.ctypes.data, a.ctypes.data)
            want = z[n + key]
            if n in NOT_BITWISE:
                tol = 4*np.finfo(float).eps*z[n + '.fd1'][:, 1]
                assert np.all(np.abs(f - want[:, 0]) <= tol), (n, ab)
                if ab:
                    assert np.all(np.abs(a - want[:, 1]) <= 1e-12*want[:, 1]), (n, 'ab')
                continue
            assert np.array_equal(f, want[:, 0], equal_nan=True), (n, ab, np.nanmax(np.abs(f - want[:, 0])))
            if ab:
                assert np.array_equal(a, want[:, 1], equal_nan=True), (n, 'ab')
        f = np.empty((m, 2)); a = np.empty((m, 2))
        fn(m, sf.ctypes.data, 1, 1, f.ctypes.data, a.ctypes.data)
        want = z[n + '.fq']
        assert np.array_equal(np.concatenate([f, a], 1), want, equal_nan=True), (n, 'dd')
