"""The kernel code generator (sincfeyn_b200/codegen/kgen.py) checked on the CPU: its output for every
graph, compiled for the host over double and over the double-double type of the device code
(sincfeyn_b200/csrc/sqdd.cuh), without FP contraction, reproduces the reference kernels' values bit for
bit at the seeded nodes of the golden fixtures (the double half f_d with SQ_AB = 1 and 0, and the
double-double fq).  This is the same arithmetic the sm_100a build runs with -fmad=false.  The pi6 class,
which the device library is not built with by default, is generated (build.generate_only) and checked
here too."""
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
#include "sqscale.cuh"
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
#define SQ_SCALE(NAME)                                                                              \
namespace sqg_##NAME { struct PT { static sqdd pt(const sqdd *x, sqdd Vx, sqdd *ab){                 \
    return KD<sqdd, 1>::pt_##NAME(x, Vx, ab); } }; }                                                \
extern "C" void hs_##NAME(const sqb_scale_t *a){                                                   \
    for(long j = 0; j < 3*a->ndir; j++) a->g[j] = sqb_scale_value<sqg_##NAME::PT>(*a, j); }
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
    cc = os.path.join(OUT, 'hostgen_%s.cc' % tag)
    text = SRC + ''.join('#include "%s"\n' % c for c in cuhs)
    deps = cuhs + [os.path.join(CSRC, f) for f in ('sqdd.cuh', 'sqscale.cuh', 'sqb_internal.h')]
    if not os.path.exists(so) or not os.path.exists(cc) or open(cc).read() != text or \
            any(os.path.getmtime(c) > os.path.getmtime(so) for c in deps):
        with open(cc, 'w') as f:
            f.write(text)
        subprocess.run(['g++', '-O0', '-ffp-contract=off', '-std=c++17', '-shared', '-fPIC', '-I' + CSRC,
                        '-o', so, cc], check=True)
    return C.CDLL(so)


def class_lib(cls):
    """the host build of a class's generated kernels (those of the class's pointwise fixture)"""
    z = np.load(os.path.join(GOLD, 'pointwise_%s.npz' % cls))
    names = sorted({k.split('.')[0] for k in z.files})
    have = [n for n in names if os.path.exists(os.path.join(GEN, n + '.cuh'))]
    if not have:
        pytest.skip('no generated kernels for %s (python -m sincfeyn_b200.build)' % cls)
    return z, have, hostlib(have)


@pytest.mark.parametrize('cls', ['g2', 'v3', 'g3', 'v4', 'w4', 'pi6'])
def test_generated_kernels_match_the_reference_bitwise(cls):
    z, have, L = class_lib(cls)
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


class ScaleArgs(C.Structure):
    """sqb_scale_t"""
    _fields_ = [('n', C.c_int), ('fixed', C.c_int), ('E', C.c_int), ('ndir', C.c_long), ('x0', C.c_double * 16),
                ('xs', C.c_void_p), ('g', C.c_void_p)]


def test_scaling_test_values_match_the_reference():
    """`sincqed scale` on the host build: the values of sqscale.cuh (the function the device kernel runs per
    value) over the generated raw double-double point functions, with the library's host halves
    (sqb_scale_setup, sqb_scale_summary), print every line of the reference's output
    (tests/golden/scale.json); graphs without a raw point function (VP) have no scale entry"""
    import json
    from sincfeyn_b200 import sq
    from scalefmt import scale_lines
    with open(os.path.join(GOLD, 'scale.json')) as f:
        gold = json.load(f)
    libs = {cls: class_lib(cls)[2] for cls in ('g2', 'g3', 'v3')}
    info = {g['name']: g for g in sq.graphs()}
    E = gold['E']
    checked = 0
    for run in gold['runs']:
        for name, want in run['lines'].items():
            L = libs['g3' if name.startswith('g3_') else 'v3' if name.startswith('v3_') else 'g2']
            if '(no scale test' in want[-1]:
                assert not hasattr(L, 'hs_' + name), name
                assert scale_lines(name, info[name]['volkov'], None, run['kappa']) == want
                continue
            n, fixed = info[name]['n'], info[name]['fixed']
            ndir = (2 * E + 1) ** (n - 1)
            x0, xs = sq.scale_setup(n, fixed, run['kappa'], run['seed'], E)
            g = np.zeros(3 * ndir)
            a = ScaleArgs(n, fixed, E, ndir)
            a.x0[:n] = list(x0)
            a.xs, a.g = xs.ctypes.data, g.ctypes.data
            getattr(L, 'hs_' + name)(C.byref(a))
            r = sq.scale_summary(n, fixed, E, g)
            assert scale_lines(name, info[name]['volkov'], r, run['kappa']) == want, name
            checked += 1
    assert checked >= 8
