"""The headline workload against the reference CPU run (GPU): the 41 integrals of all3 at h = 0.7, N = 139,
eps = 1e-12 (K = 72, default top = 2), every D = 7 graph and g3_lbl among them.

Fixture: tests/golden/all3_h0.7_N139_eps1e-12.json, `sincqed run 0.7 139 1e-12 GRAPH` of the reference's
-ffp-contract=off build with SINCQED_SYM=0 (the unfolded point set; the reference's GPU build turns the
fold off too, driver/sum.c:571) and SINCQED_KEEPBT=1 (one boundary table: its grow evaluates each point
once, as the device grow does), one graph per process (tests/golden/make_golden.py all3).

  * as written (fma = 0, every FP64 operation rounded as the reference's double half): for every graph the
    same evaluation count and fallback count, and the value within 1e-11 relative (the three-loop
    tolerance); the set sum within 1e-11 of the reference's set sum;
  * contracted (the default form, as the one concurrent batch the benchmark times): every value within
    1e-11 relative, evaluation counts within 1e-4 relative; the graphs whose counts differ are listed;
  * for each such graph the cells kept after the first refinement level by one form only are listed, and
    each lies within the kernels' rounding of the keep threshold (the contracted kernels differ from the
    as-written ones by a few ulp of the |.| sum)."""
import json
import os

import numpy as np
import pytest

from sincfeyn_b200 import sq

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'all3_h0.7_N139_eps1e-12.json')
H, N, EPS = 0.7, 139, 1e-12
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(GOLD), reason='tests/golden/make_golden.py all3 not run')]


@pytest.fixture(scope='module')
def gold():
    """the fixture's rows and the graphs of all3 that it has (all 41 once make_golden.py all3 has finished)"""
    with open(GOLD) as f:
        d = json.load(f)
    rows = {r['name']: r for r in d['rows']}
    names = sq.select(['all3'])
    assert len(names) == 41
    return rows, [g for g in names if g in rows]


def test_all3_fixture_has_every_integral(gold):
    rows, names = gold
    assert len(names) == 41, 'the reference run has %d of the 41 integrals' % len(names)


@pytest.fixture(scope='module')
def info():
    return {g['name']: g for g in sq.graphs()}


@pytest.fixture(scope='module')
def as_written(gold):
    _, names = gold
    return {g: sq.hsum(g, H, N, EPS, fma=0) for g in names}


@pytest.fixture(scope='module')
def contracted(gold, info):
    _, names = gold
    jobs = [(g, H, N, EPS, -1, float(2**info[g]['D'])*sq.flops(g, 1)) for g in names]
    res, _ = sq.hsum_batch(jobs, workers=4)
    return dict(zip(names, res))


def test_all3_as_written_matches_the_reference(gold, as_written, info):
    rows, names = gold
    for g in names:
        r, e = as_written[g], rows[g]
        v = r['S'][0]*info[g]['weight']
        assert r['nev'] == e['evals'], (g, r['nev'], e['evals'])
        assert r['nq'] == e['quad'], (g, r['nq'], e['quad'])
        assert abs(v - e['value']) <= 1e-11*abs(e['value']), (g, v, e['value'])
    ours = sum(as_written[g]['S'][0]*info[g]['weight'] for g in names)
    ref = sum(rows[g]['value'] for g in names)
    assert abs(ours - ref) <= 1e-11*sum(abs(rows[g]['value']) for g in names), (ours, ref)
    if len(names) == 41:
        d7 = [g for g in names if info[g]['D'] == 7]
        assert len(d7) == 12 and 'g3_lbl' in d7
        print('all3 h=0.7 set sum %.13f (reference CPU %.13f; A1^(6) = 1.181241456587)' % (ours, ref))


def test_all3_contracted_batch_matches_the_reference(gold, contracted, info):
    rows, names = gold
    differ = []
    for g in names:
        r, e = contracted[g], rows[g]
        v = r['S'][0]*info[g]['weight']
        assert abs(v - e['value']) <= 1e-11*abs(e['value']), (g, v, e['value'])
        assert abs(r['nev'] - e['evals']) <= 1e-4*e['evals'], (g, r['nev'], e['evals'])
        if r['nev'] != e['evals']:
            differ.append((g, r['nev'] - e['evals']))
    for g, dn in differ:
        print('%s: the contracted form evaluates %+d points against the reference run (ties at the keep threshold)' % (g, dn))


def test_all3_contracted_ties_are_at_the_threshold(tmp_path, gold, contracted, info):
    """the cells kept after the first refinement level by one form only, for every graph whose contracted
    evaluation count differs: each is kept by exactly the form whose value reaches that form's threshold,
    and lies within the two kernels' rounding of it"""
    rows, names = gold
    listing = []
    for g in names:
        if contracted[g]['nev'] == rows[g]['evals']:
            continue
        D = info[g]['D']
        ck = []
        for fma in (0, 1):
            assert sq.hsum(g, H, N, EPS, ckpt_every=600, ckpt_dir=str(tmp_path), ckpt_stop=1, fma=fma) is None
            path = os.path.join(str(tmp_path), 'sincqed_%s.ckpt' % g)
            ck.append(sq.ckpt_load(path))
            os.remove(path)
        a, b = ck
        ka = {bytes(r[:D].tobytes()) for r in a['cur']}
        kb = {bytes(r[:D].tobytes()) for r in b['cur']}
        diff = sorted(ka ^ kb)
        assert len(diff) <= 1e-4*len(ka) + 4, (g, len(diff))
        thr0, thr2 = EPS*a['ref']*1e-2, EPS*b['ref']*1e-2
        if not diff:
            listing.append('%s: the same cells after the first level (the counts differ at the top level or the last level)' % g)
            continue
        k = np.array([np.frombuffer(x, dtype=np.int8) for x in diff], dtype=np.float64)
        sf = np.exp(k*H)
        w = np.prod(sf*H, axis=1)
        f0, ab0 = sq.eval_points(g, sf, 0, 1)
        f2, _ = sq.eval_points(g, sf, 2, 1)
        for i, key in enumerate(diff):
            v0, v2 = abs(f0[i]*w[i]), abs(f2[i]*w[i])
            line = '%s k=%s kept only by the %s form: |v|/thr = %.15f (as written), %.15f (contracted)' % (
                g, tuple(int(x) for x in k[i]), 'as-written' if key in ka else 'contracted', v0/thr0, v2/thr2)
            listing.append(line)
            assert (v0 >= thr0) == (key in ka) and (v2 >= thr2) == (key in kb), line
            tol = 16*np.finfo(float).eps*ab0[i]*w[i] + abs(thr0 - thr2)
            assert abs(v0 - thr0) <= tol and abs(v2 - thr2) <= tol, line
    for line in listing:
        print(line)
