"""The four-loop lepton-loop kernels (kernels/v4, kernels/w4) at h = 1.0 (N = 97) and h = 0.9 (N = 107),
eps = 1e-12, against the reference CPU run of a dimension-stratified sample (D = 6, 7, 8 and 9;
tests/golden/vp4_sample.json: -ffp-contract=off build, SINCQED_SYM=0, SINCQED_KEEPBT=1; with v4_65 and
w4_04Sm, whose contracted level kernel takes each batch in two sweeps over many cells near the fallback),
and the lepton-loop sets with exactly known values (docs/LEPTON_LOOPS.md:5-17) (GPU).

  * every graph of the sample, as written (fma = 0): the same evaluation count, the value within 1e-11
    relative (the four-loop tolerance); contracted (the default form, the sample as one batch): the
    value within 1e-11, the count within 1e-4;
  * the sets I(a) = v4_00, I(b) = w4_00{Sc,Sm,Vm} and I(c) = w4_0i{Sc,Sm,Vm}: the weighted sum against its
    exact value within the Sinc sum's discretisation error at that h (at most 5e-6 at h = 1.0 and 1e-6 at
    h = 0.9; measured 3.7e-7 .. 3.0e-6 and 6.2e-8 .. 4.9e-7), each set closer at h = 0.9 than at 1.0."""
import json
import os

import pytest

from sincfeyn_b200 import sq

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'vp4_sample.json')
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(GOLD), reason='tests/golden/make_golden.py vp4 not run')]
HN = {1.0: 97, 0.9: 107}
SETS = {'I(a)': (['v4_00'], 0.000876865858890),
        'I(b)': (['w4_00Sc', 'w4_00Sm', 'w4_00Vm'], 0.015325282902013),
        'I(c)': (['w4_0iSc', 'w4_0iSm', 'w4_0iVm'], 0.011130913987517)}
TOL = {1.0: 5e-6, 0.9: 1e-6}


@pytest.fixture(scope='module')
def gold():
    with open(GOLD) as f:
        return {(r['name'], r['h']): r for r in json.load(f)['runs']}


@pytest.fixture(scope='module')
def info():
    return {g['name']: g for g in sq.graphs()}


def test_vp4_sample_is_stratified(gold, info):
    dims = {info[g]['D'] for g, h in gold}
    assert dims >= {6, 7, 8, 9}, dims
    assert {h for _, h in gold} == {1.0, 0.9}


@pytest.mark.parametrize('h', [1.0, 0.9])
def test_vp4_sample_matches_the_reference(gold, info, h):
    names = sorted(g for g, hh in gold if hh == h)
    for g in names:
        e = gold[(g, h)]
        r = sq.hsum(g, h, HN[h], 1e-12, fma=0)
        v = r['S'][0]*info[g]['weight']
        assert r['nev'] == e['evals'], (g, h, r['nev'], e['evals'])
        assert abs(v - e['value']) <= 1e-11*abs(e['value']), (g, h, v, e['value'])
    jobs = [(g, h, HN[h], 1e-12, -1, float(2**info[g]['D'])) for g in names]
    res, _ = sq.hsum_batch(jobs, workers=4)
    for g, r in zip(names, res):
        e = gold[(g, h)]
        v = r['S'][0]*info[g]['weight']
        assert abs(r['nev'] - e['evals']) <= 1e-4*e['evals'], (g, h, r['nev'], e['evals'])
        assert abs(v - e['value']) <= 1e-11*abs(e['value']), (g, h, v, e['value'])


def test_lepton_loop_sets_against_their_exact_values(info):
    names = sorted({g for gs, _ in SETS.values() for g in gs})
    diff = {}
    for h in (1.0, 0.9):
        jobs = [(g, h, HN[h], 1e-12, -1, float(2**info[g]['D'])) for g in names]
        res, _ = sq.hsum_batch(jobs, workers=4)
        val = {g: r['S'][0]*info[g]['weight'] for g, r in zip(names, res)}
        for label, (gs, exact) in SETS.items():
            d = sum(val[g] for g in gs) - exact
            diff[(label, h)] = d
            print('%s h=%.1f: sum %.15f exact %.15f diff %+.2e' % (label, h, d + exact, exact, d))
            assert abs(d) <= TOL[h], (label, h, d)
    for label in SETS:
        assert abs(diff[(label, 0.9)]) < abs(diff[(label, 1.0)]), (label, diff[(label, 0.9)], diff[(label, 1.0)])
