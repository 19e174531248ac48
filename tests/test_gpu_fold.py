"""The symmetry fold on the device (GPU): sqb_hsum with sym = 'auto' against the reference CPU run with
its fold on (driver/sum.c:21-46, 405-409, 734-745; the -ffp-contract=off build, SINCQED_KEEPBT=1:
tests/golden/fold.json), with top = 2 so that kept orbits go on to a second refinement level.

  - the group found on the device is the reference's (order and generators);
  - with the kernels that round as written (fma 0) the device evaluates the reference's folded point
    set: the evaluation counts are equal and the values agree within 1e-13 (two loops) or 1e-11 (three
    loops) relative;
  - the fold leaves the kept tree alone: folded and unfolded device runs keep the same top level, agree
    within the same tolerance, and the folded one evaluates fewer points;
  - the contracted kernels (the default) agree too, their evaluation counts within 1e-4;
  - checkpoints: a folded run stopped after its first level and resumed is bit for bit the unbroken one,
    and the reference (fold on) resumes the evaluator's folded checkpoint to its own folded result."""
import json
import os

import pytest

from sincfeyn_b200 import sq

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'fold.json')
pytestmark = pytest.mark.gpu

with open(GOLD) as _f:
    FOLD = json.load(_f)


@pytest.mark.parametrize('case', FOLD['runs'], ids=['%s-h%g' % (r['name'], r['h']) for r in FOLD['runs']])
def test_folded_sum_matches_the_reference(case):
    name, h, N, top = case['name'], case['h'], case['N'], case['top']
    tol = 1e-13 if case['L'] == 2 else 1e-11
    g = FOLD['groups'][name]
    f = sq.run(h, N, 1e-12, [name], top=top, fma=0, sym='auto')[0]
    assert (f['raw']['sym_order'], f['raw']['sym_desc']) == (g['order'], g['desc'])
    assert f['evals'] == case['evals'], (f['evals'], case['evals'])
    assert abs(f['quad'] - case['quad']) <= 1e-2*case['quad'] + 10, (f['quad'], case['quad'])
    assert f['kept'] == case['kept_top']
    assert abs(f['value'] - case['value']) <= tol*abs(case['value']), (f['value'], case['value'])
    assert abs(f['S_2h'] - case['S_2h']) <= 1e-8*abs(case['S_2h'])
    u = sq.run(h, N, 1e-12, [name], top=top, fma=0)[0]
    assert u['raw']['sym_order'] == 1
    assert u['kept'] == f['kept'] and f['evals'] < u['evals']
    assert abs(f['value'] - u['value']) <= tol*abs(u['value']), (f['value'], u['value'])
    c = sq.run(h, N, 1e-12, [name], top=top, sym='auto')[0]
    assert abs(c['evals'] - case['evals']) <= 1e-4*case['evals']
    assert abs(c['value'] - case['value']) <= tol*abs(case['value']), (c['value'], case['value'])


def test_manual_group_and_refusals_on_the_device():
    """SINCQED_SYM given by hand: the accepted involution folds as the search's group does, a refused
    entry is reported and leaves the sum unfolded"""
    case = next(r for r in FOLD['runs'] if r['name'] == 'g3_07')
    h, N, top = case['h'], case['N'], case['top']
    a = sq.run(h, N, 1e-12, ['g3_07'], top=top, fma=0, sym='0,2,1,4,3')[0]
    assert a['raw']['sym_order'] == 2 and a['evals'] == case['evals']
    b = sq.run(h, N, 1e-12, ['g3_07'], top=top, fma=0, sym='1,0,2,3,4')[0]
    assert b['raw']['sym_order'] == 1 and 'NOT SYMMETRIC' in b['raw']['sym_msg']
    assert b['evals'] > a['evals']


EXACT = ('S', 'Ah', 'ref', 'prune', 'trunc', 'unres', 'nev', 'nq', 'kept_top', 'es1', 'es2', 'abskipped')


def test_folded_stop_and_resume_is_bitwise(tmp_path):
    """a folded run stopped after its first checkpoint (the kept orbits of the step-2h level, in list
    order) and resumed gives every result field of the unbroken folded run"""
    case = next(r for r in FOLD['runs'] if r['name'] == 'g3_07')
    name, h, N, top = case['name'], case['h'], case['N'], case['top']
    full = sq.hsum(name, h, N, 1e-12, top, sym='auto')
    d = str(tmp_path)
    assert sq.hsum(name, h, N, 1e-12, top, sym='auto', ckpt_every=600, ckpt_dir=d, ckpt_stop=1) is None
    res = sq.hsum(name, h, N, 1e-12, top, sym='auto', ckpt_every=600, ckpt_dir=d)
    for f in EXACT:
        assert res[f] == full[f], (f, res[f], full[f])


def test_reference_resumes_our_folded_checkpoint(tmp_path):
    """the reference CPU build (fold on) resumes the evaluator's folded checkpoint and finishes with its
    own folded run's evaluation count and value"""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'oracle'))
    import refpy
    if not refpy.available(refpy.SINCQED_EXACT):
        pytest.skip('oracle/_ref not built')
    case = next(r for r in FOLD['runs'] if r['name'] == 'g3_25')
    name, h, N, top = case['name'], case['h'], case['N'], case['top']
    d = str(tmp_path)
    assert sq.hsum(name, h, N, 1e-12, top, fma=0, sym='auto', ckpt_every=600, ckpt_dir=d, ckpt_stop=1) is None
    rows, out = refpy.run(refpy.SINCQED_EXACT, h, N, 1e-12, [name], top=top,
                          env=dict(FOLD['env'], SINCQED_CKPT='600', SINCQED_CKPT_DIR=d))
    assert 'resuming %s from checkpoint' % name in out
    assert rows[0]['evals'] == case['evals'], (rows[0]['evals'], case['evals'])
    assert abs(rows[0]['value'] - case['value']) <= 1e-11*abs(case['value'])
