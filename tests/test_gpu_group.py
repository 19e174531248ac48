"""Integrals of one graph at several h as one group (GPU): sqb_hsum_group runs their refinement levels as
shared launches (the FP64 and double-double kernels take tiles of every integral from a device queue; one
reduce, one finish with one block per integral, one scatter), and the batch does so for every graph with
opts.group.  The batches, tiles and summation order of each integral are those it has alone, so:

  * every result of a group is bit for bit sqb_hsum's for the same integral (values S_h, S_2h, S_4h, every
    error column, evaluation and fallback counts, kept cells), for the two-loop set, three-loop graphs of
    D = 5 and 6 (one with h = 0.7, whose step-2h level runs alone and whose last level shares the launch),
    with the symmetry fold, and in the contracted and as-written forms;
  * the two-loop part of the mixed batch (all2 at h = 1.0, 0.9, 0.8, 0.7, N = 2 ceil(48/h) + 1) as a grouped
    batch matches the reference CPU run at every h: the same evaluation counts (as written), values within
    1e-13 relative (tests/golden/all2_mixed_h.json);
  * a grouped batch of the mixed workload's sample returns what the ungrouped batch returns."""
import json
import math
import os

import pytest

from sincfeyn_b200 import sq

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'all2_mixed_h.json')
pytestmark = pytest.mark.gpu
MIX_H = (1.0, 0.9, 0.8, 0.7)
FIELDS = ('S', 'Ah', 'ref', 'prune', 'trunc', 'unres', 'nev', 'nq', 'kept_top', 'abskipped', 'unresdrop', 'es1', 'es2')


def same(a, b):
    if isinstance(a, list):
        return len(a) == len(b) and all(same(x, y) for x, y in zip(a, b))
    return a == b or (a != a and b != b)


def jobs_of(g, hs=MIX_H, eps=1e-12):
    return [(g, h, 2*math.ceil(48/h - 1e-9) + 1, eps) for h in hs]


@pytest.mark.parametrize('graph,kw', [('g2_00', {}), ('g2_02', {'fma': 0}), ('v2_00', {}), ('g3_07', {}),
                                      ('g3_07', {'sym': 'auto'}), ('g3_01', {})])
def test_group_is_bitwise_each_integral_alone(graph, kw):
    hs = MIX_H if graph != 'g3_01' else (1.0, 0.9)
    jobs = jobs_of(graph, hs)
    grp = sq.hsum_group(jobs, **kw)
    for j, r in zip(jobs, grp):
        one = sq.hsum(*j, **kw)
        for f in FIELDS:
            assert same(r[f], one[f]), (j, f, r[f], one[f])


def test_grouped_batch_of_all2_matches_the_reference_at_four_h():
    with open(GOLD) as f:
        ref = {(r['name'], r['h']): r for r in json.load(f)['runs']}
    info = {g['name']: g for g in sq.graphs()}
    jobs = [j for g in sq.select(['all2']) for j in jobs_of(g)]
    res, _ = sq.hsum_batch(jobs, workers=2, group=1, fma=0)
    assert len(res) == 20
    for j, r in zip(jobs, res):
        e = ref[(j[0], j[1])]
        v = r['S'][0]*info[j[0]]['weight']
        assert r['nev'] == e['evals'], (j, r['nev'], e['evals'])
        assert abs(v - e['value']) <= 1e-13*abs(e['value']), (j, v, e['value'])


def test_grouped_batch_equals_the_batch():
    info = {g['name']: g for g in sq.graphs()}
    names = ['g2_01', 'g3_07', 'v3_03', 'g3_09', 'v3_p4Sm']
    jobs = [(g, h, N, eps, -1, (2.0/h)**info[g]['D']) for g in names for (g_, h, N, eps) in jobs_of(g)]
    a, _ = sq.hsum_batch(jobs, workers=3)
    b, _ = sq.hsum_batch(jobs, workers=3, group=1)
    for j, x, y in zip(jobs, a, b):
        for f in FIELDS:
            assert same(x[f], y[f]), (j, f, x[f], y[f])
