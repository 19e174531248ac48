"""The build's per-graph compile policy (CPU): which spill report decides a graph's occupancy, and which
graphs get the two-sweep level kernel.

* `_spill` reads ptxas's report of a contracted unit: the point function's calls (`sqb_fcall`, one copy per
  kernel that calls it) decide, not the kernels around them, whose stack holds only the registers saved
  across the call; an exact unit (no calls) is judged by its FP64 kernel;
* the library's occupancy record agrees with that policy: every graph with two sweeps has at least
  SWEEPS_FLOPS flops per point and D >= 5, and every graph capped at three resident CTAs reported at most
  SPILL_MAX bytes of spill stores there."""
import json
import os

import pytest

from sincfeyn_b200 import build

CONTRACTED = """ptxas info    : Compiling entry function '_Z9sqb_k_f64IN10sqgf_g3_001FELi7ELi0EEv10sqb_eval_t' for 'sm_100a'
ptxas info    : Function properties for _Z9sqb_k_f64IN10sqgf_g3_001FELi7ELi0EEv10sqb_eval_t
    112 bytes stack frame, 124 bytes spill stores, 144 bytes spill loads
ptxas info    : Used 168 registers, used 1 barriers, 112 bytes cumulative stack size, 784 bytes smem
ptxas info    : Function properties for _Z9sqb_fcallIN10sqgf_g3_001FELi7ELi0EE7sqb_fab6sqb_ptIXT0_EE
    0 bytes stack frame, 0 bytes spill stores, 0 bytes spill loads
ptxas info    : Function properties for _Z9sqb_fcallIN10sqgf_g3_001FELi7ELi1EE7sqb_fab6sqb_ptIXT0_EE
    0 bytes stack frame, 32 bytes spill stores, 32 bytes spill loads
ptxas info    : Compiling entry function '_Z9sqb_k_f64IN10sqgf_g3_001FELi7ELi1EEv10sqb_eval_t' for 'sm_100a'
ptxas info    : Function properties for _Z9sqb_k_f64IN10sqgf_g3_001FELi7ELi1EEv10sqb_eval_t
    48 bytes stack frame, 52 bytes spill stores, 76 bytes spill loads
ptxas info    : Function properties for _Z9sqb_fcallIN10sqgf_g3_001FELi7ELi1EE7sqb_fab6sqb_ptIXT0_EE
    0 bytes stack frame, 8 bytes spill stores, 8 bytes spill loads
"""

EXACT = """ptxas info    : Function properties for _Z9sqb_k_f64IN9sqg_g3_001FELi7ELi0EEv10sqb_eval_t
    64 bytes stack frame, 80 bytes spill stores, 64 bytes spill loads
ptxas info    : Used 168 registers, used 1 barriers, 64 bytes cumulative stack size, 784 bytes smem
"""


def test_spill_reads_the_point_function_calls():
    assert build._spill(CONTRACTED) == 32          # the worst sqb_fcall copy, not the kernels' 124 / 52


def test_spill_falls_back_to_the_kernel_without_calls():
    assert build._spill(EXACT) == 80
    assert build._spill('ptxas info    : Used 32 registers') == -1


def test_occupancy_record_follows_the_policy():
    if not (os.path.exists(build.OCC) and os.path.exists(build.FLOPS)):
        pytest.skip('library not built')
    with open(build.OCC) as f:
        occ = json.load(f)
    with open(build.FLOPS) as f:
        flops = json.load(f)
    from sincfeyn_b200 import sq
    dims = {g['name']: g['D'] for g in sq.graphs()}
    two = [g for g, v in occ.items() if v.get('sweeps', 1) > 1]
    assert two, 'no graph with two sweeps'
    for g in two:
        assert flops[g]['ab1'] >= build.SWEEPS_FLOPS and dims[g] >= 5, g
    for g, v in occ.items():
        if g in flops and dims.get(g, 0) >= 5 and flops[g]['ab1'] >= build.SWEEPS_FLOPS:
            assert v.get('sweeps') == 2, g
        if v.get('min_blocks') == 3:
            assert 0 <= v['spill_stores_at_3'] <= build.SPILL_MAX, (g, v)
    assert occ['g3_lbl']['sweeps'] == 2 and occ['g3_00']['sweeps'] == 1
