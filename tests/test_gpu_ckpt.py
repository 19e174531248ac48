"""Checkpoints of sqb_hsum on the device (GPU): written at the end of every level but the last, in the
reference's SQCK4 format, and resumed.

  - stopped after the first checkpoint and resumed, a run gives every result field bit for bit as an
    unbroken run (the cell list is streamed from the device in cell order, the sums are kept exactly);
  - the reference CPU build (-ffp-contract=off, fold off) resumes the evaluator's checkpoint and finishes
    with the same evaluation count and a value within 1e-13;
  - a checkpoint in mid-level (the reference writes them every SINCQED_CKPT seconds) resumes with the
    partial sums carried on: made here from the evaluator's own level-end checkpoints by splitting a
    level's cells in two, it gives the unbroken run's counts and its value within 1e-15."""
import os
import shutil
import sys

import pytest

from sincfeyn_b200 import sq

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EPS = 1e-12
EXACT = ('S', 'Ah', 'ref', 'prune', 'trunc', 'unres', 'nev', 'nq', 'kept_top', 'es1', 'es2', 'abskipped')
CASES = [('g2_01', 0.7, 139, -1), ('v3_01', 0.7, 139, -1), ('g2_03', 0.7, 139, 3)]


def ckfile(d, name):
    return os.path.join(d, 'sincqed_%s.ckpt' % name)


@pytest.mark.parametrize('name,h,N,top', CASES)
def test_stop_and_resume_is_bitwise(tmp_path, name, h, N, top):
    full = sq.hsum(name, h, N, EPS, top)
    d = str(tmp_path)
    assert sq.hsum(name, h, N, EPS, top, ckpt_every=600, ckpt_dir=d, ckpt_stop=1) is None
    ck = sq.ckpt_load(ckfile(d, name))
    assert ck['lev'] == (top if top > 0 else sq.default_top(h)) - 2 and ck['next'] == 0 and ck['ncur'] > 0
    res = sq.hsum(name, h, N, EPS, top, ckpt_every=600, ckpt_dir=d)
    assert not os.path.exists(ckfile(d, name))
    for f in EXACT:
        assert res[f] == full[f], (f, res[f], full[f])


@pytest.mark.parametrize('name', ['g2_01', 'v3_01'])
def test_reference_resumes_our_checkpoint(tmp_path, name):
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import refpy
    if not refpy.available(refpy.SINCQED_EXACT):
        pytest.skip('oracle/_ref not built')
    h, N = 0.7, 139
    full = sq.run(h, N, EPS, [name])[0]
    d = str(tmp_path)
    assert sq.hsum(name, h, N, EPS, ckpt_every=600, ckpt_dir=d, ckpt_stop=1) is None
    rows, out = refpy.run(refpy.SINCQED_EXACT, h, N, EPS, [name],
                          env={'SINCQED_CKPT': '600', 'SINCQED_CKPT_DIR': d, 'SINCQED_SYM': '0', 'SINCQED_KEEPBT': '1'})
    assert 'resuming %s from checkpoint' % name in out
    r = rows[0]
    assert r['evals'] == full['evals'], (r['evals'], full['evals'])
    assert abs(r['value'] - full['value']) <= 1e-13*abs(full['value']), (r['value'], full['value'])
    assert not os.path.exists(ckfile(d, name))


def test_mid_level_checkpoint(tmp_path):
    """g2_03 at h = 0.7 with top = 3: levels at step 4h, 2h, h.  The step-2h level is split after m of its
    n cells: its first m cells run alone (their kept children and partial sums come from the resulting
    checkpoint), then a mid-level checkpoint (next = m) resumes the rest."""
    name, h, N, top = 'g2_03', 0.7, 139, 3
    full = sq.hsum(name, h, N, EPS, top)
    d0, d1, d2 = (str(tmp_path / x) for x in ('a', 'b', 'c'))
    for x in (d0, d1, d2):
        os.makedirs(x)
    assert sq.hsum(name, h, N, EPS, top, ckpt_every=600, ckpt_dir=d0, ckpt_stop=1) is None
    base = sq.ckpt_load(ckfile(d0, name))                  # before the step-2h level
    assert base['lev'] == 1
    n = base['ncur']
    m = n//2
    half = dict(base)
    half['cur'] = base['cur'][:m]
    half['ncur'] = m
    sq.ckpt_save(ckfile(d1, name), half)
    assert sq.hsum(name, h, N, EPS, top, ckpt_every=600, ckpt_dir=d1, ckpt_stop=1) is None
    part = sq.ckpt_load(ckfile(d1, name))                  # after the first m cells of that level
    mid = dict(base)
    mid.update(next=m, s=part['s'], a=part['a'], drop=part['drop'], u=part['u'], ne=part['ne'], q=part['q'],
               nxt=part['cur'], nnxt=part['ncur'], cnt=part['cnt'])
    sq.ckpt_save(ckfile(d2, name), mid)
    res = sq.hsum(name, h, N, EPS, top, ckpt_every=600, ckpt_dir=d2)
    for f in ('nev', 'nq', 'kept_top', 'abskipped'):
        assert res[f] == full[f], (f, res[f], full[f])
    for f in ('Ah', 'prune', 'es1', 'es2'):
        assert abs(res[f] - full[f]) <= 1e-15*abs(full[f]) + 1e-300, (f, res[f], full[f])
    for i in range(3):
        assert abs(res['S'][i] - full['S'][i]) <= 1e-15*abs(full['S'][i]), (i, res['S'][i], full['S'][i])
    shutil.rmtree(str(tmp_path), ignore_errors=True)
