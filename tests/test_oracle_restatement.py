"""The oracle's own serial C restatement of the hierarchical sum (oracle/sq_oracle.cc) against the
reference run (CPU): on `run 1.0 97 1e-12 all2` (fold off, exact kernels) it must evaluate the same
points (evaluation, fallback and kept-cell counts equal) and give every value to 1e-15 relative (the
level sums are restated in the reference's block order).  This pins the restatement of grow, dilate
and the level loop that the device implementation follows."""
import json
import os
import subprocess

import pytest

import refpy

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
SQO = os.path.join(refpy.REF_DIR, 'sq_oracle')
pytestmark = pytest.mark.skipif(not os.path.exists(SQO), reason='make -C oracle')


def run_oracle(h, N, eps, top, graphs):
    out = subprocess.run([SQO, repr(h), str(N), repr(eps), str(top)] + graphs, stdout=subprocess.PIPE, text=True,
                         check=True).stdout
    rows = {}
    for line in out.splitlines():
        t = line.split()
        rows[t[0]] = dict(value=float(t[1]), S_2h=float(t[2]), evals=int(t[3]), quad=int(t[4]), kept_top=int(t[5]),
                          prune=float(t[6]))
    return rows


def test_restatement_reproduces_the_reference_all2():
    with open(os.path.join(GOLD, 'all2_h1.0_N97_eps1e-12.json')) as f:
        ref = json.load(f)['reference_exact_unfolded']
    got = run_oracle(1.0, 97, 1e-12, 1, [r['name'] for r in ref])
    for r in ref:
        g = got[r['name']]
        assert (g['evals'], g['quad'], g['kept_top']) == (r['evals'], r['quad'], r['kept_top']), r['name']
        assert abs(g['value'] - r['value']) <= 1e-15*abs(r['value']), (r['name'], g['value'], r['value'])
        assert abs(g['prune'] - r['prune']) <= 0.01*r['prune'] + 1e-20


@pytest.mark.parametrize('name', ['v3_00', 'v3_p4Sc'])
def test_restatement_reproduces_the_reference_three_loop(name):
    rows, out = refpy.run(refpy.SINCQED_EXACT, 1.2, 69, 1e-10, [name], top=1, env={'SINCQED_SYM': '0', 'SINCQED_KEEPBT': '1'})
    got = run_oracle(1.2, 69, 1e-10, 1, [name])[name]
    assert got['evals'] == rows[0]['evals']
    assert abs(got['value'] - rows[0]['value']) <= 1e-15*abs(rows[0]['value']) + 1e-18
