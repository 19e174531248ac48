"""The last-level predictor on the device (GPU): sqb_hsum with predict = 1 (SINCQED_PREDICT=1,
driver/sum.c:64-69, 379-422, driver/sumkey.h:219-222, 445-451) against the reference CPU run with the
same setting (-ffp-contract=off build, SINCQED_KEEPBT=1, top = 2: tests/golden/predict.json).

The table stores float logarithms and the corner means pass through exp; the device's log and exp may
round differently from the C library's in the last bit, so a child whose mean lies within that rounding of
alpha*thr can be left out by one program and evaluated by the other.  With the kernels that round as
written (fma 0): the evaluation counts and the counts of left-out points agree within 1e-3 relative (+ 10),
and each value within 1e-11 relative (a flipped child weighs about thr = eps Ref 1e-2).  Checkpoints carry
the table: a predicted run stopped after the step-2h level and resumed is bit for bit the unbroken one, and
the reference resumes the evaluator's checkpoint to its own predicted result."""
import json
import os
import sys

import pytest

from sincfeyn_b200 import sq

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
with open(os.path.join(ROOT, 'tests', 'golden', 'predict.json')) as _f:
    PRED = json.load(_f)
RUNS = PRED['runs']
EXACT = ('S', 'Ah', 'ref', 'prune', 'trunc', 'unres', 'nev', 'nq', 'kept_top', 'es1', 'es2', 'abskipped', 'pskip')


def near(a, b, rel):
    return abs(a - b) <= rel*b + 10


@pytest.mark.parametrize('case', RUNS, ids=['%s-h%g%s' % (r['name'], r['h'], '-fold' if r['fold'] else '') for r in RUNS])
def test_predicted_sum_matches_the_reference(case):
    name, h, N, top = case['name'], case['h'], case['N'], case['top']
    kw = dict(top=top, fma=0, predict=PRED['alpha'], sym='auto' if case['fold'] else None)
    r = sq.run(h, N, PRED['eps'], [name], **kw)[0]
    assert r['raw']['pskip'] > 0
    assert near(r['raw']['pskip'], case['pskip'], 1e-3), (r['raw']['pskip'], case['pskip'])
    assert near(r['evals'], case['evals'], 1e-3), (r['evals'], case['evals'])
    assert r['kept'] == case['kept_top']
    assert abs(r['value'] - case['value']) <= 1e-11*abs(case['value']), (r['value'], case['value'])
    # the predictor only leaves points out: the unpredicted run evaluates them all
    u = sq.run(h, N, PRED['eps'], [name], top=top, fma=0, sym='auto' if case['fold'] else None)[0]
    assert u['evals'] == r['evals'] + r['raw']['pskip'] and u['raw']['pskip'] == 0


def test_predicted_stop_and_resume_is_bitwise(tmp_path):
    case = RUNS[3]
    name, h, N, top = case['name'], case['h'], case['N'], case['top']
    full = sq.hsum(name, h, N, PRED['eps'], top, predict=PRED['alpha'])
    d = str(tmp_path)
    assert sq.hsum(name, h, N, PRED['eps'], top, predict=PRED['alpha'], ckpt_every=600, ckpt_dir=d, ckpt_stop=1) is None
    ck = sq.ckpt_load(os.path.join(d, 'sincqed_%s.ckpt' % name))
    assert ck['vcap'] > 0 and ck['vn'] > 0
    res = sq.hsum(name, h, N, PRED['eps'], top, predict=PRED['alpha'], ckpt_every=600, ckpt_dir=d)
    for f in EXACT:
        assert res[f] == full[f], (f, res[f], full[f])


def test_reference_resumes_our_predicted_checkpoint(tmp_path):
    """the table's slots are the reference's: it resumes with them and predicts as its own run does"""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import refpy
    if not refpy.available(refpy.SINCQED_EXACT):
        pytest.skip('oracle/_ref not built')
    case = RUNS[3]
    name, h, N, top = case['name'], case['h'], case['N'], case['top']
    d = str(tmp_path)
    assert sq.hsum(name, h, N, PRED['eps'], top, fma=0, predict=PRED['alpha'], ckpt_every=600, ckpt_dir=d,
                   ckpt_stop=1) is None
    rows, out = refpy.run(refpy.SINCQED_EXACT, h, N, PRED['eps'], [name], top=top,
                          env={'SINCQED_PREDICT': '1', 'SINCQED_KEEPBT': '1', 'SINCQED_SYM': '0', 'SINCQED_CKPT': '600',
                               'SINCQED_CKPT_DIR': d})
    assert 'resuming %s from checkpoint' % name in out
    assert near(rows[0]['evals'], case['evals'], 1e-3), (rows[0]['evals'], case['evals'])
    assert abs(rows[0]['value'] - case['value']) <= 1e-11*abs(case['value'])
