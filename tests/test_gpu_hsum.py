"""The chosen form (sqb_hsum, every refinement level on the device) against the reference CPU run
(GPU).

Configuration: `sincqed run 1.0 97 1e-12 all2`, the five two-loop integrals.  The reference is the
-ffp-contract=off build with the symmetry fold off (the reference's GPU build turns the fold off too,
driver/sum.c:571), whose point values round exactly like the device kernels; so the evaluated point set
must be the same (evaluation counts equal) and each graph's value must agree within 1e-13 relative
(the two-loop tolerance), the difference being only the summation (double-double on the device,
Neumaier in blocks on the CPU).  Also against the reference as shipped (fold on, FP contraction on) and
the exact values."""
import json
import math
import os

import pytest

from sincfeyn_b200 import sq

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
pytestmark = pytest.mark.gpu

EXACT = {'g2_00': -0.064020941344682816, 'g2_01': -0.58997802228274215, 'g2_02': -0.46764544609361365,
         'g2_03': 0.77747802228274215, 'v2_00': 0.015687421859103}


@pytest.fixture(scope='module')
def golden():
    with open(os.path.join(GOLD, 'all2_h1.0_N97_eps1e-12.json')) as f:
        return json.load(f)


@pytest.fixture(scope='module')
def rows():
    """every FP64 operation rounded as written (fma 0): the reference's point set exactly"""
    return sq.run(1.0, 97, 1e-12, ['all2'], fma=0)


@pytest.fixture(scope='module')
def rows_fast():
    """the default form: contracted FP64 kernels"""
    return sq.run(1.0, 97, 1e-12, ['all2'])


def test_all2_matches_the_reference_unfolded_exact(rows, golden):
    ref = {r['name']: r for r in golden['reference_exact_unfolded']}
    for r in rows:
        e = ref[r['name']]
        assert r['evals'] == e['evals'], (r['name'], r['evals'], e['evals'])
        assert abs(r['value'] - e['value']) <= 1e-13*abs(e['value']), (r['name'], r['value'], e['value'])
        assert abs(r['S_2h'] - e['S_2h']) <= 1e-8*abs(e['S_2h'])
        for k in ('prune', 'trunc'):
            assert abs(r[k] - e[k]) <= 0.01*abs(e[k]) + 1e-16, (r['name'], k, r[k], e[k])


def test_all2_matches_the_shipped_reference_and_exact_values(rows, golden):
    ref = {r['name']: r for r in golden['reference']}
    tot = 0
    for r in rows:
        assert abs(r['value'] - ref[r['name']]['value']) <= 1e-13*abs(ref[r['name']]['value'])
        assert abs(r['value'] - EXACT[r['name']]) < 2e-6
        tot += r['value']
    assert abs(tot - (-0.328478965579)) < 3e-5


def test_all2_contracted_form_agrees(rows_fast, golden):
    ref = {r['name']: r for r in golden['reference_exact_unfolded']}
    for r in rows_fast:
        e = ref[r['name']]
        assert abs(r['evals'] - e['evals']) <= 1e-4*e['evals'], (r['name'], r['evals'], e['evals'])
        assert abs(r['value'] - e['value']) <= 1e-13*abs(e['value']), (r['name'], r['value'], e['value'])
        assert abs(r['value'] - EXACT[r['name']]) < 2e-6


def test_all_dd_form_agrees(rows):
    dd = sq.run(1.0, 97, 1e-12, ['all2'], alldd=1)
    for a, b in zip(rows, dd):
        assert a['evals'] == b['evals'] or abs(a['evals'] - b['evals']) < 1e-3*a['evals']
        assert abs(a['value'] - b['value']) <= 1e-12*abs(b['value']), (a['name'], a['value'], b['value'])


THREE_LOOP = ['g3_07', 'g3_17', 'v3_01', 'v3_p4Sm', 'w3_p40c']


@pytest.mark.parametrize('fma', [0, 1], ids=['as-written', 'contracted'])
@pytest.mark.parametrize('name', THREE_LOOP)
def test_three_loop_graphs_match_the_reference_run(name, fma):
    """three-loop kernels (D = 4..5) at h = 1.0, N = 97, eps = 1e-12: the reference CPU run (exact build,
    fold off) on this host, same evaluation count, value within 1e-11 relative"""
    import refpy
    if name not in {g['name'] for g in sq.graphs()}:
        pytest.skip('%s not in this build' % name)
    rows, _ = refpy.run(refpy.SINCQED_EXACT, 1.0, 97, 1e-12, [name], top=1, env={'SINCQED_SYM': '0', 'SINCQED_KEEPBT': '1'})
    e = rows[0]
    r = sq.run(1.0, 97, 1e-12, [name], top=1, fma=fma)[0]
    if fma:
        assert abs(r["evals"] - e["evals"]) <= 1e-4*e["evals"], (name, r["evals"], e["evals"])
    else:
        assert r['evals'] == e['evals'], (name, r['evals'], e['evals'])
    assert abs(r['value'] - e['value']) <= 1e-11*abs(e['value']) + 1e-15, (name, r['value'], e['value'])
