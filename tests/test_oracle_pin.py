"""The oracle (the reference built from its own sources by oracle/Makefile) against the golden fixtures
and the reference's own known answers.  CPU only."""
import json
import math
import os
import subprocess

import numpy as np
import pytest

import refpy

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
pytestmark = pytest.mark.skipif(not refpy.available(), reason='oracle/_ref not built (make -C oracle)')


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def test_all2_reproduces_the_golden_run():
    g = load('all2_h1.0_N97_eps1e-12.json')
    rows, _ = refpy.run(refpy.SINCQED, 1.0, 97, 1e-12, ['all2'])
    assert [r['name'] for r in rows] == [r['name'] for r in g['reference']]
    for r, e in zip(rows, g['reference']):
        assert r['value'] == e['value'] and r['evals'] == e['evals'], r['name']
    rows, _ = refpy.run(refpy.SINCQED_EXACT, 1.0, 97, 1e-12, ['all2'], env={'SINCQED_SYM': '0'})
    for r, e in zip(rows, g['reference_exact_unfolded']):
        assert r['value'] == e['value'] and r['evals'] == e['evals'], r['name']


def test_all2_against_the_exact_values():
    """driver/graphs.c:36-46: the two-loop values the reference lists, to the accuracy h = 1.0 gives"""
    g = load('all2_h1.0_N97_eps1e-12.json')
    exact = {'g2_00': -0.064020941344682816, 'g2_01': -0.58997802228274215, 'g2_02': -0.46764544609361365,
             'g2_03': 0.77747802228274215, 'v2_00': 0.015687421859103}
    tot = 0
    for r in g['reference']:
        assert abs(r['value'] - exact[r['name']]) < 2e-6
        tot += r['value']
    a4 = -0.328478965579                      # A1^(4), tests/run_tests.sh:20-21
    assert abs(tot - a4) < 3e-5


def test_boxsum_known_answers():
    g = load('boxsum_gl.json')
    out = subprocess.run([refpy.BOXSUM, '1.0', '6'], stdout=subprocess.PIPE, text=True, check=True).stdout
    for line in out.splitlines():
        tok = line.split()
        if tok[1] == 'term0':
            assert float(tok[2]) == g[tok[0]]['term0'] and float(tok[4]) == g[tok[0]]['term1']
        else:
            assert float(tok[4]) == g[tok[0]]['box_h1_K6']


@pytest.mark.parametrize('cls', ['g2', 'v3', 'g3'])
def test_pointwise_kernels_reproduce_the_fixture(cls):
    z = np.load(os.path.join(GOLD, 'pointwise_%s.npz' % cls))
    names = sorted({k.split('.')[0] for k in z.files})
    assert names
    for n in names:
        sf = z[n + '.sf']
        f1, a1 = refpy.fd(n, sf, 1)
        assert np.array_equal(np.stack([f1, a1], 1), z[n + '.fd1'], equal_nan=True), n
        q, qa = refpy.fq(n, sf[:16])
        assert np.array_equal(np.concatenate([q, qa], 1), z[n + '.fq'][:16], equal_nan=True), n


def test_regression_checks_of_the_reference():
    """tests/run_tests.sh:20-27, the reference's own regression runs (two-loop sum, Pi2 insertion)"""
    rows, _ = refpy.run(refpy.SINCQED, 1.0, 81, 1e-11, ['all2'])
    assert abs(sum(r['value'] for r in rows) - (-0.328478965579)) <= 3e-5
    rows, _ = refpy.run(refpy.SINCQED, 1.0, 81, 1e-11, ['VP: 1-loop vertex + Pi2'])
    assert abs(rows[0]['value'] - 0.015687421859) <= 3e-6
