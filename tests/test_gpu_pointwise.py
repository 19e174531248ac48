"""Pointwise parity of the sm_100a kernels with the reference kernels (GPU).

At the seeded nodes of the golden fixtures (the tests/check_onept.sh protocol: sigma = e^z, z ~ U[-3,3])
the device FP64 kernels (nvcc -fmad=false) must give the reference double half's f and |.| sum bit for
bit, for SQ_AB = 1 and 0, and the device double-double kernels the reference's double-double fq bit for
bit.  The fixtures were written by the reference compiled with -ffp-contract=off
(tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from sincfeyn_b200 import sq

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
pytestmark = pytest.mark.gpu
# see tests/test_codegen_host.py: FP64 agrees to 4 ulp of the |.| sum, double-double bit for bit
NOT_BITWISE = {'g3_lbl'}


@pytest.mark.parametrize('cls', ['g2', 'v3', 'g3', 'v4', 'w4', 'pi6'])
def test_fp64_and_dd_bitwise(cls):
    z = np.load(os.path.join(GOLD, 'pointwise_%s.npz' % cls))
    have = {g['name'] for g in sq.graphs()}
    names = sorted({k.split('.')[0] for k in z.files} & have)
    if not names:
        pytest.skip('class %s not in this build' % cls)
    bad = []
    for n in names:
        sf = z[n + '.sf']
        for ab, key in ((1, '.fd1'), (0, '.fd0')):
            f, a = sq.eval_points(n, sf, 0, ab)
            w = z[n + key]
            if n in NOT_BITWISE:
                tol = 4*np.finfo(float).eps*z[n + '.fd1'][:, 1]
                if not (np.all(np.abs(f - w[:, 0]) <= tol) and (not ab or np.all(np.abs(a - w[:, 1]) <= 1e-12*w[:, 1]))):
                    bad.append((n, 'fp64 tolerance', ab))
                continue
            if not np.array_equal(f, w[:, 0], equal_nan=True) or (ab and not np.array_equal(a, w[:, 1], equal_nan=True)):
                bad.append((n, 'fp64', ab, float(np.nanmax(np.abs(f - w[:, 0]) / np.maximum(w[:, 1], 1e-300)))))
        f, a = sq.eval_points(n, sf, 1, 1)
        if not np.array_equal(np.concatenate([f, a], 1), z[n + '.fq'], equal_nan=True):
            bad.append((n, 'dd'))
    assert not bad, bad


@pytest.mark.parametrize('cls', ['g2', 'v3', 'g3', 'v4', 'w4', 'pi6'])
def test_contracted_fp64_within_rounding(cls):
    """The contracted FP64 kernels (fused multiply-adds, the default fast form) round differently from
    the source; at the same nodes they agree with the reference double half to a few ulp of the |.| sum,
    the scale of the fallback's own error bound (ab * 16 eps)."""
    z = np.load(os.path.join(GOLD, 'pointwise_%s.npz' % cls))
    have = {g['name'] for g in sq.graphs()}
    names = sorted({k.split('.')[0] for k in z.files} & have)
    if not names:
        pytest.skip('class %s not in this build' % cls)
    eps = np.finfo(float).eps
    worst = 0.0
    for n in names:
        sf = z[n + '.sf']
        w = z[n + '.fd1']
        f, a = sq.eval_points(n, sf, 2, 1)
        ok = np.isfinite(w[:, 0])
        r = np.abs(f[ok] - w[ok, 0])/np.maximum(w[ok, 1], 1e-300)
        worst = max(worst, float(r.max()) if r.size else 0.0)
        assert np.all(r <= 16*eps), (n, float(r.max())/eps)
        assert np.all(np.abs(a[ok] - w[ok, 1]) <= 1e-12*w[ok, 1]), n
    print('%s: worst |f_fma - f| / ab = %.2f ulp' % (cls, worst/eps))
