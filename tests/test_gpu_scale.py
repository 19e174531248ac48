"""The scaling test on the device (GPU): `sincqed scale SEL kappa seed` (driver/main.c:76-115) with the graph's
raw double-double point function evaluated by sqb_k_scale, against the reference's own output (the
-ffp-contract=off build, one thread so that directions come in order: tests/golden/scale.json).

The double-double arithmetic is the reference's operation for operation, so every printed figure agrees:
the directions, the slow count, the worst ratio and its direction, |g| at kappa/3, 2 kappa/3, kappa, and
the first twelve slow directions (kappa = 3 makes directions slow, ratio ~ e^-1); VP graphs (no raw point
function) report that they have no test.  The same lines come from the command line
`sincfeyn_b200/bin/sincqed scale`."""
import json
import os
import subprocess

import pytest

from sincfeyn_b200 import sq

from scalefmt import scale_lines as lines

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, 'tests', 'golden', 'scale.json')
CLI = os.path.join(ROOT, 'sincfeyn_b200', 'bin', 'sincqed')
pytestmark = pytest.mark.gpu

with open(GOLD) as _f:
    SCALE = json.load(_f)


CASES = [(r, name) for r in SCALE['runs'] for name in sorted(r['lines'])]


@pytest.mark.parametrize('run,name', CASES, ids=['%s-k%g-s%d' % (n, r['kappa'], r['seed']) for r, n in CASES])
def test_scale_matches_the_reference(run, name):
    volkov = {g['name']: g['volkov'] for g in sq.graphs()}[name]
    r = sq.scale_test(name, run['kappa'], run['seed'], SCALE['E'])
    assert lines(name, volkov, r, run['kappa']) == run['lines'][name]


def test_scale_command_line():
    env = dict(os.environ)
    env.pop('SCALE_E', None)
    for run in (SCALE['runs'][0], SCALE['runs'][-1]):
        out = subprocess.run([CLI, 'scale', run['sel'], str(run['kappa']), str(run['seed'])], stdout=subprocess.PIPE,
                             text=True, env=env, check=True, timeout=600).stdout.splitlines()
        names = [g['name'] for g in sq.graphs() if g['name'] in run['lines']]
        assert out == [ln for n in names for ln in run['lines'][n]]
