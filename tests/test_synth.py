"""The synthetic Sinc-sum integrands (sincfeyn_b200/synth) on the CPU.

  - The device code's double-double exp and log (sincfeyn_b200/csrc/sqdd.cuh), compiled for the host
    without FP contraction, against 250-bit mpmath values.
  - The generator's sources against their own definition f(z) = prod sech(a z + b) (exp(eps X) - 1)/eps,
    X = sum exp(-|z_i|), evaluated in mpmath at the golden nodes: the oracle's double-double values
    (pointwise_synth.npz, the oracle build with oracle/sqsynth.h) to the double-double error model,
    its double values to the cancellation the naive expm1 leaves.
  - The evaluator's generated kernels for them (host build of the code generator's output): the double
    half bit for bit equal to the oracle's (both use the C library's exp and log here), the
    double-double half to 2 QEPS of the |.| sum (the two builds' exp and log differ in the last bits).
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, 'sincfeyn_b200', 'csrc')
GOLD = os.path.join(ROOT, 'tests', 'golden')
OUT = os.path.join(ROOT, 'tests', '_hostgen')
sys.path.insert(0, ROOT)
from sincfeyn_b200.synth import mksynth  # noqa: E402

mp = pytest.importorskip('mpmath')
QEPS = 4.93e-32

DDX = r'''
#include "sqdd.cuh"
extern "C" void ddexp(long n, const double *x, double *o){
    for(long i = 0; i < n; i++){ sqdd r = sqdd_exp(sqdd(x[2*i], x[2*i+1])); o[2*i] = r.hi; o[2*i+1] = r.lo; } }
extern "C" void ddlog(long n, const double *x, double *o){
    for(long i = 0; i < n; i++){ sqdd r = sqdd_log(sqdd(x[2*i], x[2*i+1])); o[2*i] = r.hi; o[2*i+1] = r.lo; } }
'''


def _ddlib():
    os.makedirs(OUT, exist_ok=True)
    so = os.path.join(OUT, 'ddx.so')
    hdr = os.path.join(CSRC, 'sqdd.cuh')
    if not os.path.exists(so) or os.path.getmtime(hdr) > os.path.getmtime(so):
        cc = os.path.join(OUT, 'ddx.cc')
        with open(cc, 'w') as f:
            f.write(DDX)
        subprocess.run(['g++', '-O1', '-ffp-contract=off', '-shared', '-fPIC', '-I' + CSRC, '-o', so, cc], check=True)
    L = C.CDLL(so)
    for fn in (L.ddexp, L.ddlog):
        fn.argtypes = [C.c_long, C.c_void_p, C.c_void_p]
    return L


def _dd(v):
    hi = float(v)
    return hi, float(v - mp.mpf(hi))


def _mp(hi, lo):
    return mp.mpf(hi) + mp.mpf(lo)


def test_dd_exp_and_log_against_mpmath():
    mp.mp.prec = 250
    L = _ddlib()
    rng = np.random.default_rng(7)
    scale = rng.choice([1.0, 1e-3, 1e-6, 1e-12], size=1500)
    xs = [mp.mpf(u) * s for u, s in zip(rng.uniform(-600, 600, size=1500), scale)]
    x = np.array([_dd(v) for v in xs]).ravel()
    o = np.empty_like(x)
    L.ddexp(len(xs), x.ctypes.data, o.ctypes.data)
    for i in range(len(xs)):
        a = _mp(x[2*i], x[2*i + 1])
        t = mp.exp(a)
        # backward error about one double-double rounding of the argument: 4e-32 |a| relative
        assert abs(_mp(o[2*i], o[2*i + 1]) - t) <= 4e-32 * max(1, abs(a)) * t, float(a)
    ys = [mp.exp(mp.mpf(u)) for u in rng.uniform(-600, 600, size=1500)]
    y = np.array([_dd(v) for v in ys]).ravel()
    L.ddlog(len(ys), y.ctypes.data, o.ctypes.data)
    for i in range(len(ys)):
        t = mp.log(_mp(y[2*i], y[2*i + 1]))
        assert abs(_mp(o[2*i], o[2*i + 1]) - t) <= 4e-32 * max(1, abs(t)), float(t)


def _f_exact(name, s):
    d = int(name.split('_d')[1])
    a, b = mksynth.params(d)
    p, X, js = mp.mpf(1), mp.mpf(0), mp.mpf(1)
    for i in range(d):
        z = mp.log(mp.mpf(s[i]))
        p *= mp.sech(mp.mpf(a[i]) * z + mp.mpf(b[i]))
        X += mp.exp(-abs(z))
        js *= mp.mpf(s[i])
    ex = mp.exp(X * mp.mpf(1e-9))
    return (ex - 1) * mp.mpf(1e9) * p / js, (ex + 1) * mp.mpf(1e9) * p / js


def test_oracle_values_against_the_definition():
    mp.mp.prec = 200
    z = np.load(os.path.join(GOLD, 'pointwise_synth.npz'))
    names = sorted({k.split('.')[0] for k in z.files})
    assert names == ['syn_d11', 'syn_d5', 'syn_d8']
    eps = np.finfo(float).eps
    for n in names:
        sf, fq, fd = z[n + '.sf'], z[n + '.fq'], z[n + '.fd1']
        for i in range(sf.shape[0]):
            f, ab = _f_exact(n, sf[i])
            # double-double: within the fallback's error model QEPS * |.| sum (measured: 0.2 QEPS)
            assert abs(_mp(fq[i, 0], fq[i, 1]) - f) <= QEPS * ab, (n, i)
            assert abs(_mp(fq[i, 2], fq[i, 3]) - ab) <= 1e-29 * ab, (n, i)
            # double: exp(eps X) - 1 cancels, leaving about an ulp of the |.| sum (measured: 0.25)
            assert abs(fd[i, 0] - f) <= 2 * eps * ab, (n, i)


@pytest.fixture(scope='module')
def hostgen():
    gen = os.path.join(ROOT, 'sincfeyn_b200', '_build', 'gen')
    names = ['syn_d5', 'syn_d8', 'syn_d11']
    if not all(os.path.exists(os.path.join(gen, n + '.cuh')) for n in names):
        pytest.skip('no generated kernels (python -m sincfeyn_b200.build)')
    sys.path.insert(0, os.path.join(ROOT, 'tests'))
    import test_codegen_host as T
    return T.hostlib(names), names


def test_generated_synth_kernels_match_the_oracle(hostgen):
    L, names = hostgen
    z = np.load(os.path.join(GOLD, 'pointwise_synth.npz'))
    for n in names:
        sf = np.ascontiguousarray(z[n + '.sf'])
        m = sf.shape[0]
        fn = getattr(L, 'hg_' + n)
        fn.argtypes = [C.c_long, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        for ab, key in ((1, '.fd1'), (0, '.fd0')):
            f = np.empty(m)
            a = np.empty(m)
            fn(m, sf.ctypes.data, 0, ab, f.ctypes.data, a.ctypes.data)
            np.testing.assert_array_equal(f, z[n + key][:, 0])
            np.testing.assert_array_equal(a, z[n + key][:, 1])
        f = np.empty((m, 2))
        a = np.empty((m, 2))
        fn(m, sf.ctypes.data, 1, 1, f.ctypes.data, a.ctypes.data)
        q = z[n + '.fq']
        abq = q[:, 2] + q[:, 3]
        assert np.all(np.abs((f[:, 0] - q[:, 0]) + (f[:, 1] - q[:, 1])) <= 2 * QEPS * abq), n
        assert np.all(np.abs((a[:, 0] - q[:, 2]) + (a[:, 1] - q[:, 3])) <= 2e-29 * abq), n


def test_generator_is_deterministic():
    for d in mksynth.DIMS:
        with open(os.path.join(ROOT, 'sincfeyn_b200', 'synth', 'syn_d%d.c' % d)) as f:
            assert f.read() == mksynth.source(d)
    a, b = mksynth.params(5)
    assert all(0.5 <= x <= 2.0 for x in a) and all(-1.0 <= x <= 1.0 for x in b)
