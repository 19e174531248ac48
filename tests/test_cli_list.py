"""The command line's host-only commands against the reference build (oracle/_ref/sincqed), CPU, no device:
`sincqed list` (driver/main.c:186-190) prints the same graphs in the same order with the same Volkov
strings, loop counts, dimensions and mirror weights (the registry of driver/graphs.c:8-12, first name
wins)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, 'sincfeyn_b200', 'bin', 'sincqed')
REF = os.path.join(ROOT, 'oracle', '_ref', 'sincqed')


def graph_lines(binary):
    out = subprocess.run([binary, 'list'], stdout=subprocess.PIPE, text=True, check=True, timeout=120).stdout
    return [ln for ln in out.splitlines() if ln.startswith('  ')]


def test_list_matches_the_reference():
    if not (os.path.exists(OURS) and os.path.exists(REF)):
        pytest.skip('build first (python -m sincfeyn_b200.build; make -C oracle)')
    ours, ref = graph_lines(OURS), graph_lines(REF)
    assert len(ours) >= 170
    assert ours == ref


@pytest.mark.parametrize('sel', ['vp3', 'vp4', 'VP: 1-loop vertex + Pi2 Pi2', 'v4_00'])
def test_selection_matches_the_reference(sel):
    """graph selection by group, Volkov string and name (driver/graphs.c:15-29): `sincqed scale SEL` over
    graphs without a raw point function reports each selected graph without a device, in the same order"""
    if not (os.path.exists(OURS) and os.path.exists(REF)):
        pytest.skip('build first (python -m sincfeyn_b200.build; make -C oracle)')
    want = subprocess.run([REF, 'scale', sel], stdout=subprocess.PIPE, text=True, check=True, timeout=120).stdout
    got = subprocess.run([OURS, 'scale', sel], stdout=subprocess.PIPE, text=True, check=True, timeout=120).stdout
    assert got == want and want.count('(no scale test') >= 1
