"""The two-loop kernels against a quad-double oracle.

The reference's kernels/g2 sources compiled over its own quad-double type (pslq/quad/qd.h, ~64 digits;
oracle/_ref/libsqqd.so) give each point's value to far beyond double-double.  Against it, at the 400
seeded nodes per graph of the golden fixtures:

  - the double-double values (the fixtures, which the device's double-double kernels reproduce bit for
    bit) err by at most 2 QEPS x the |.| sum, the error model of the reference's fallback test
    (e = ab w QEPS, driver/eval.c:25-30);
  - the FP64 values err by at most 16 eps x the |.| sum, the bound of the fallback test itself
    (ab w 16 eps / DDSLACK, driver/eval.c:33-53), for the as-written kernels (CPU) and for both device
    kernels, as written and contracted (GPU)."""
import ctypes as C
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBQD = os.path.join(ROOT, 'oracle', '_ref', 'libsqqd.so')
GOLD = os.path.join(ROOT, 'tests', 'golden')
QEPS = 4.93e-32
EPS = np.finfo(float).eps
NAMES = ['g2_00', 'g2_01', 'g2_02', 'g2_03', 'v2_00']
mp = pytest.importorskip('mpmath')


@pytest.fixture(scope='module')
def qd():
    if not os.path.exists(LIBQD):
        pytest.skip('oracle/_ref/libsqqd.so not built (make -C oracle)')
    L = C.CDLL(LIBQD)
    L.sqqd_fq.argtypes = [C.c_char_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]
    z = np.load(os.path.join(GOLD, 'pointwise_g2.npz'))
    out = {}
    mp.mp.prec = 300
    for n in NAMES:
        sf = np.ascontiguousarray(z[n + '.sf'])
        m = sf.shape[0]
        f = np.zeros(4*m)
        a = np.zeros(4*m)
        assert L.sqqd_fq(n.encode(), m, sf.ctypes.data, f.ctypes.data, a.ctypes.data) > 0
        f = f.reshape(m, 4)
        a = a.reshape(m, 4)
        out[n] = (sf, [sum(mp.mpf(x) for x in r) for r in f], [sum(mp.mpf(x) for x in r) for r in a], z)
    return out


def worst(vals, exact, ab):
    return max(float(abs(mp.mpf(v) - e)/b) for v, e, b in zip(vals, exact, ab) if b > 0)


def test_double_double_and_fp64_against_quad_double(qd):
    for n, (sf, fq, abq, z) in qd.items():
        q = z[n + '.fq']
        dd = [mp.mpf(h) + mp.mpf(l) for h, l in q[:, :2]]
        assert worst(dd, fq, abq) <= 2*QEPS, n
        assert worst(list(z[n + '.fd1'][:, 0]), fq, abq) <= 16*EPS, n


@pytest.mark.gpu
def test_device_fp64_forms_against_quad_double(qd):
    from sincfeyn_b200 import sq
    for n, (sf, fq, abq, z) in qd.items():
        for prec in (0, 2):
            f, _ = sq.eval_points(n, sf, prec, 1)
            assert worst(list(f), fq, abq) <= 16*EPS, (n, prec)
        f, _ = sq.eval_points(n, sf, 1, 1)
        assert worst([mp.mpf(h) + mp.mpf(l) for h, l in f], fq, abq) <= 2*QEPS, n
