"""The symmetry fold's group search on the CPU (sqb_sym_find, driver/sum.c:464-592), with the reference's
own kernels as the evaluator (oracle/_ref/libsqref.so, -ffp-contract=off: the double half of the
reference build that printed the golden lines).

  - for every graph of g2 g3 v3 v4 w4, the group found (order, generators in the reference's order and
    format, and the largest deviation over the 200 check nodes, as the reference prints it) is the one in
    the reference's log line (tests/golden/fold.json);
  - SINCQED_SYM given by hand: accepted involutions, and the entries the reference refuses (wrong length,
    out of range, not an involution, the identity, not a symmetry) with its messages;
  - the closure: generated groups of a made-up integrand have the expected order and are closed under
    composition, with the identity first."""
import itertools
import json
import math
import os
import sys

import numpy as np
import pytest

from sincfeyn_b200 import sq

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
import refpy  # noqa: E402

GOLD = os.path.join(ROOT, 'tests', 'golden', 'fold.json')


@pytest.fixture(scope='module')
def gold():
    if not os.path.exists(refpy.LIBSQREF):
        pytest.skip('oracle/_ref/libsqref.so not built (make -C oracle)')
    with open(GOLD) as f:
        return json.load(f)


def reference_nodes(name, h):
    """fnode() of the reference (driver/sum.c:509): fd at sf = EX[k + K] = exp(k h)"""
    def ev(k):
        sf = np.array([[math.exp(int(x) * h) for x in row] for row in k], dtype=np.float64)
        return refpy.fd(name, sf, 1)
    return ev


def test_groups_match_the_reference(gold):
    h = gold['group_run']['h']
    have = set(refpy.names())
    checked = 0
    for name in gold['searched']:
        if name not in have:
            continue
        D = refpy.info(name)['D']
        r = sq.sym_find(D, reference_nodes(name, h), 'auto')
        want = gold['groups'].get(name)
        if want is None:
            assert r['order'] == 1, (name, r)
        else:
            assert (r['order'], r['desc'], '%.1e' % r['worst']) == (want['order'], want['desc'], want['worst']), (name, r)
        checked += 1
    assert checked >= 100


def closed(elems):
    s = {tuple(e) for e in elems}
    return all(tuple(a[b[i]] for i in range(len(a))) in s for a in elems for b in elems)


def test_manual_entries(gold):
    name, h = 'g3_07', gold['group_run']['h']
    ev = reference_nodes(name, h)
    r = sq.sym_find(5, ev, '0,2,1,4,3')
    assert r['order'] == 2 and r['desc'] == '0,2,1,4,3' and r['msg'] == ''
    assert [list(e) for e in r['elems']] == [[0, 1, 2, 3, 4], [0, 2, 1, 4, 3]]
    for spec, why in [('0,1,2', 'is not a non-trivial involution of the 5 axes'),
                      ('0,2,1,4,3,5', 'is not a non-trivial involution of the 5 axes'),
                      ('0,2,1,4,9', 'is not a non-trivial involution of the 5 axes'),
                      ('1,2,0,3,4', 'is not a non-trivial involution of the 5 axes'),
                      ('0,1,2,3,4', 'is not a non-trivial involution of the 5 axes'),
                      ('1,0,2,3,4', 'NOT SYMMETRIC: ignored')]:
        r = sq.sym_find(5, ev, spec)
        # the message quotes the entry as far as it was read (driver/sum.c:580)
        assert r['order'] == 1 and why in r['msg'] and ('SINCQED_SYM entry "%s' % spec[:5]) in r['msg'], (spec, r)
    # a refused entry does not stop the next one
    r = sq.sym_find(5, ev, '1,0,2,3,4; 0,2,1,4,3')
    assert r['order'] == 2 and r['desc'] == '0,2,1,4,3' and 'NOT SYMMETRIC' in r['msg']
    for off in (None, '', '0', 'off'):
        assert sq.sym_find(5, ev, off)['order'] == 1


def test_closure_of_a_made_up_group():
    """f symmetric under any permutation of axes {0,1,2} and the swap of 3 and 4: the search finds
    transpositions and closes them into S3 x S2 (order 12)"""
    D = 6
    a = np.array([0.7, 0.7, 0.7, 1.3, 1.3, 0.2])

    def ev(k):
        z = k.astype(np.float64) * 0.5
        g = np.exp(-np.abs(z) * a)
        f = g[:, 0] * g[:, 1] * g[:, 2] * (1 + z[:, 0] * z[:, 1] * z[:, 2]) * (g[:, 3] + g[:, 4]) * (1 + g[:, 5])
        return f, np.abs(f) + 1.0
    r = sq.sym_find(D, ev, 'auto')
    assert r['order'] == 12, r
    e = [list(x) for x in r['elems']]
    assert e[0] == list(range(D)) and closed(e)
    assert {tuple(x) for x in e} == {p + (3, 4, 5) for p in itertools.permutations(range(3))} | \
                                    {p + (4, 3, 5) for p in itertools.permutations(range(3))}
