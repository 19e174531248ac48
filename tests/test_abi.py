"""The C-ABI library loads on the CPU host and exports every entry point include/sincfeyn_b200.h declares,
plus the reference's per-graph plug-in descriptors (GG_<name>, GPU_ALL).  No device calls."""
import ctypes as C
import os
import re

import pytest

from sincfeyn_b200 import sq

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'include', 'sincfeyn_b200.h')


def declared_functions():
    text = re.sub(r'/\*.*?\*/', '', open(HEADER).read(), flags=re.S)
    names = set(re.findall(r'^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(', text, re.M))
    names -= {'typedef', 'void', 'int', 'double'}
    return sorted(n for n in names if not n.startswith('sq_gpu_launch'))


def test_library_exports_every_declared_symbol():
    L = sq.lib()
    fns = declared_functions()
    assert {'gpu_setup', 'gpu_submit', 'gpu_wait', 'gpu_submit_cells', 'gpu_info', 'sqb_hsum'} <= set(fns)
    for fn in fns:
        assert hasattr(L, fn), fn
    C.c_void_p.in_dll(L, 'GPU_ALL')


def test_registry_and_plugin_descriptors():
    L = sq.lib()
    gs = sq.graphs()
    assert len(gs) >= 5
    names = [g['name'] for g in gs]
    assert names[:5] == ['g2_00', 'g2_01', 'g2_02', 'g2_03', 'v2_00']
    for g in gs:
        C.c_void_p.in_dll(L, 'GG_' + g['name'])
        assert 3 <= g['D'] <= 11
        assert sq.flops(g['name'], 1) >= sq.flops(g['name'], 0) > 0


def test_selectors_match_the_reference_groups():
    assert sq.select(['all2']) == ['g2_00', 'g2_01', 'g2_02', 'g2_03', 'v2_00']
    assert sq.select(['2; 1-4, 3-5', 'g2_00']) == ['g2_00']
    if any(g['name'] == 'g3_lbl' for g in sq.graphs()):
        a3 = sq.select(['all3'])
        assert len(a3) == 41 and 'g3_lbl' in a3 and not any(n.startswith('w3_') for n in a3)


def test_default_top_follows_the_reference():
    assert sq.default_top(1.0) == 1 and sq.default_top(0.9) == 1 and sq.default_top(0.8) == 1
    assert sq.default_top(0.7) == 2 and sq.default_top(0.75) == 2


def test_struct_mirrors_have_the_library_sizes():
    """the ctypes copies of the interface's structures (sincfeyn_b200/sq.py, and the level interface the
    no-alloc test drives) have the sizes the library was compiled with"""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import test_zz_no_alloc as na
    from test_codegen_host import ScaleArgs
    L = sq.lib()
    L.sqb_struct_size.argtypes = [C.c_char_p]
    L.sqb_struct_size.restype = C.c_long
    for name, cls in (('sqb_opts_t', sq.Opts), ('sqb_result_t', sq.Result), ('sqb_job_t', sq.Job),
                      ('sqb_ckpt_t', sq.Checkpoint), ('sqb_scale_result_t', sq.ScaleResult),
                      ('sqb_level_t', na.Level), ('sqb_acc_t', na.Acc), ('sqb_test_t', na.PointTestParams),
                      ('sqb_scale_t', ScaleArgs)):
        assert L.sqb_struct_size(name.encode()) == C.sizeof(cls), name
    assert L.sqb_struct_size(b'no_such_struct') == -1
