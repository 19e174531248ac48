"""The pi6 class (kernels/pi6: the 27 four-loop vertex kernels with a Pi6 insertion, w4_p6*) in the device
library (GPU), against the reference CPU run on this host (the -ffp-contract=off build, fold off, one
boundary table) at h = 1.0, N = 97, eps = 1e-12: the same evaluation count as written (fma 0), values
within the four-loop tolerance 1e-11 relative in both FP64 forms.  The pointwise checks of every pi6 kernel
are in tests/test_gpu_pointwise.py (fixture tests/golden/pointwise_pi6.npz)."""
import pytest

import refpy
from sincfeyn_b200 import sq

pytestmark = pytest.mark.gpu
GRAPHS = ['w4_p60c', 'w4_p62c']


@pytest.mark.parametrize('fma', [0, 1], ids=['as-written', 'contracted'])
@pytest.mark.parametrize('name', GRAPHS)
def test_pi6_graph_matches_the_reference_run(name, fma):
    have = {g['name'] for g in sq.graphs()}
    assert name in have, 'pi6 is in the default device library'
    rows, _ = refpy.run(refpy.SINCQED_EXACT, 1.0, 97, 1e-12, [name], env={'SINCQED_SYM': '0', 'SINCQED_KEEPBT': '1'})
    e = rows[0]
    r = sq.run(1.0, 97, 1e-12, [name], fma=fma)[0]
    if fma:
        assert abs(r['evals'] - e['evals']) <= 1e-4*e['evals'], (name, r['evals'], e['evals'])
    else:
        assert r['evals'] == e['evals'], (name, r['evals'], e['evals'])
    assert abs(r['value'] - e['value']) <= 1e-11*abs(e['value']), (name, r['value'], e['value'])
