"""The plain form as a drop-in (GPU): the reference driver, built as its GPU build (-DSQ_GPU) from its
own sources, linked against libsqb200.so instead of driver/gpu.cu (oracle/_ref/sincqed-dropin), runs
`sincqed run 1.0 97 1e-12 all2` with every batch evaluated by this library's sm_100a kernels.  Its
results must equal the reference CPU run (-ffp-contract=off, fold off as in the GPU build): same
evaluation counts, values within 1e-13 relative."""
import json
import os

import pytest

import refpy

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refpy.available(refpy.SINCQED_DROPIN), reason='make -C oracle dropin')]


def test_reference_driver_on_the_plain_form():
    with open(os.path.join(GOLD, 'all2_h1.0_N97_eps1e-12.json')) as f:
        ref = {r['name']: r for r in json.load(f)['reference_exact_unfolded']}
    rows, out = refpy.run(refpy.SINCQED_DROPIN, 1.0, 97, 1e-12, ['all2'], env={'SINCQED_GPU': '1'})
    assert 'on the GPU' in out
    for r in rows:
        e = ref[r['name']]
        assert r['evals'] == e['evals'], r['name']
        assert abs(r['value'] - e['value']) <= 1e-13*abs(e['value']), (r['name'], r['value'], e['value'])
