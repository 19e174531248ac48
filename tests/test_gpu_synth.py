"""The synthetic Sinc-sum integrands on the device (GPU).

Pointwise: the FP64 kernels against the oracle's double half (the device's exp and log round
differently from the C library's in the last bit, so within 4 ulp of the |.| sum) and the double-double
kernels against the oracle's double-double values (2 QEPS of the |.| sum).

Hierarchical sum: sqb_hsum against the reference's hsum() on the same integrands (golden runs: the
-ffp-contract=off build, symmetry fold off, one grow boundary table), h = 1.0 (N = 61) and h = 0.7
(N = 87) at d = 5 and h = 1.0 at d = 8, eps = 1e-12.  Points whose FP64 value moves by an ulp can cross
the keep threshold or the fallback bound, so the evaluation and fallback counts agree to 1e-4 and 1e-2
relative, and the value to 1e-11 relative."""
import json
import os

import numpy as np
import pytest

from sincfeyn_b200 import sq

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
pytestmark = pytest.mark.gpu
QEPS = 4.93e-32


def test_synth_pointwise_on_the_device():
    z = np.load(os.path.join(GOLD, 'pointwise_synth.npz'))
    eps = np.finfo(float).eps
    for n in ('syn_d5', 'syn_d8', 'syn_d11'):
        sf = z[n + '.sf']
        f, a = sq.eval_points(n, sf, 0, 1)
        want = z[n + '.fd1']
        assert np.all(np.abs(f - want[:, 0]) <= 4*eps*want[:, 1]), n
        assert np.all(np.abs(a - want[:, 1]) <= 8*eps*want[:, 1]), n
        fq, aq = sq.eval_points(n, sf, 1, 1)
        q = z[n + '.fq']
        abq = q[:, 2] + q[:, 3]
        assert np.all(np.abs((fq[:, 0] - q[:, 0]) + (fq[:, 1] - q[:, 1])) <= 2*QEPS*abq), n
        assert np.all(np.abs((aq[:, 0] - q[:, 2]) + (aq[:, 1] - q[:, 3])) <= 2e-29*abq), n


with open(os.path.join(GOLD, 'synth_runs.json')) as _f:
    RUNS = json.load(_f)['runs']


@pytest.mark.parametrize('case', RUNS, ids=['%s-h%g' % (r['name'], r['h']) for r in RUNS])
def test_synth_hsum_matches_the_reference(case):
    r = sq.run(case['h'], case['N'], 1e-12, [case['name']])[0]
    assert abs(r['evals'] - case['evals']) <= 1e-4*case['evals'], (r['evals'], case['evals'])
    assert abs(r['quad'] - case['quad']) <= 1e-2*case['quad'] + 10, (r['quad'], case['quad'])
    assert abs(r['value'] - case['value']) <= 1e-11*abs(case['value']), (r['value'], case['value'])
    assert abs(r['S_2h'] - case['S_2h']) <= 1e-8*abs(case['S_2h'])
