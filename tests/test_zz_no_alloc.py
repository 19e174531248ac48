"""The allocation-free level entry point, sqb_level_noalloc (GPU).

It serves callers that cannot let the library call cudaMalloc (a program whose device memory belongs to
its own pool allocator, or a service with a memory budget fixed at start-up): it runs one refinement
level's batch on a scratch array built into the library.  This test calls it through the C ABI on the
same cells as the library's allocating level pass (sqb_dev_level, the path sqb_hsum uses) and checks,
on two calls in a row, that the sums agree within the two-loop tolerance of the parity tests (1e-13
relative) and that the counters and the kept-children list are identical.  The file is named to be
collected last, so that a run stopping at the first failure has run every other test first.
"""
import ctypes as C
import math

import numpy as np
import pytest

from sincfeyn_b200 import sq

pytestmark = pytest.mark.gpu

GRAPH, H, K, ST = 'g3_07', 1.0, 48, 1       # a three-loop kernel (D = 5) with double-double fallbacks
ABSERR, NEARF, DDSLACK = 1e-15, 1e-3, 1.0


class PointTestParams(C.Structure):
    _fields_ = [('abserr', C.c_double), ('nearf', C.c_double), ('ddslack', C.c_double),
                ('abskip', C.c_int), ('abcheck', C.c_int), ('dropunres', C.c_int), ('alldd', C.c_int),
                ('fma', C.c_int), ('split', C.c_int)]


class Level(C.Structure):
    """sqb_level_t (sqb_rt.h), every field: no fold, no predictor"""
    _fields_ = [('g', C.c_void_p), ('cells', C.c_void_p), ('ncell', C.c_long), ('next', C.c_void_p),
                ('next_cap', C.c_long), ('st', C.c_int), ('last', C.c_int), ('pw', C.c_double), ('thr', C.c_double),
                ('t', PointTestParams), ('max_children', C.c_long), ('sym', C.c_void_p), ('vt', C.c_void_p),
                ('vput', C.c_int), ('predict', C.c_double), ('esok', C.c_int), ('X', C.c_void_p), ('Wt', C.c_void_p),
                ('K', C.c_int)]


class Acc(C.Structure):
    """sqb_acc_t (sqb_rt.h), every field"""
    _fields_ = [('S', C.c_double * 2), ('A', C.c_double * 2), ('drop', C.c_double * 2), ('b1', C.c_double * 2),
                ('b2', C.c_double * 2), ('u', C.c_double * 2), ('ne', C.c_ulonglong), ('keep', C.c_ulonglong),
                ('nq', C.c_ulonglong), ('unres', C.c_ulonglong), ('skipped', C.c_ulonglong), ('overflow', C.c_ulonglong),
                ('pskip', C.c_ulonglong)]


def cells_box():
    """cells of the step-2 grid with |k_i| <= 4 (3125 cells, 100,000 children); varied flags: the skip bit
    on cells with k_0 > 0, shadow tiers 0..2"""
    r = np.arange(-4, 5, 2)
    g = np.stack(np.meshgrid(*[r]*5, indexing='ij'), -1).reshape(-1, 5)
    pts = np.zeros((g.shape[0], 12), dtype=np.int8)
    pts[:, :5] = g
    tier = (np.abs(g).sum(1) // 4) % 3
    pts[:, 11] = ((g[:, 0] > 0).astype(np.int8) | (tier << 1)).astype(np.int8)
    return pts


def existing_level(L, cells_dev, n, next_dev, cap, last, thr):
    """the allocating level pass (sqb_dev_level) with the same tables and parameters"""
    L.sqb_dev_init(0)
    X = (C.c_double * (2*K + 1))(*[math.exp(k*H) for k in range(-K, K + 1)])
    W = (C.c_double * (2*K + 1))(*[X[i]*H for i in range(2*K + 1)])
    assert L.sqb_dev_tables(X, W, K) == 0
    L.sqb_find_graph.restype = C.c_void_p
    lv = Level(g=L.sqb_find_graph(GRAPH.encode()), cells=cells_dev, ncell=n, next=next_dev, next_cap=cap, st=ST,
               last=last, pw=float(ST**5), thr=thr, t=PointTestParams(ABSERR, NEARF, DDSLACK, 1, 0, 1, 0, 0, 0), max_children=0)
    acc, nn, ms = Acc(), C.c_long(), C.c_double()
    assert L.sqb_dev_level(C.byref(lv), C.byref(acc), C.byref(nn), C.byref(ms)) == 0
    sums = [x for f in ('S', 'A', 'drop', 'b1', 'b2', 'u') for x in getattr(acc, f)]
    return np.array(sums), [acc.ne, acc.keep, acc.nq, acc.unres, acc.skipped, acc.overflow]


def noalloc_lib():
    """the library with the entry point's argument and result types declared (each test sets them, so that
    any test runs alone)"""
    L = sq.lib()
    L.sqb_error.restype = C.c_char_p
    L.sqb_level_noalloc.restype = C.c_int
    L.sqb_level_noalloc.argtypes = [C.c_char_p, C.c_double, C.c_int, C.c_void_p, C.c_long, C.c_int, C.c_int,
                                    C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                    C.c_int, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]
    return L


def noalloc_level(L, cells_dev, n, next_dev, cap, last, thr):
    sums = (C.c_double * 12)()
    counts = (C.c_longlong * 6)()
    rc = L.sqb_level_noalloc(GRAPH.encode(), H, K, cells_dev, n, ST, last, float(ST**5), thr, ABSERR, NEARF,
                             DDSLACK, 1, 0, 1, next_dev, cap, sums, counts, None)
    assert rc == 0, L.sqb_error()
    return np.array(list(sums)), list(counts)


@pytest.mark.parametrize('last', [0, 1])
def test_noalloc_matches_the_allocating_level_pass(last):
    import torch
    L = noalloc_lib()
    pts = cells_box()
    n = pts.shape[0]
    cells = torch.from_numpy(pts.copy()).cuda()
    cap = n << 5
    thr = 1e-9
    ref_next = torch.zeros((cap, 12), dtype=torch.int8, device='cuda')
    torch.cuda.synchronize()
    ref_sums, ref_counts = existing_level(L, cells.data_ptr(), n, ref_next.data_ptr(), cap, last, thr)
    assert ref_counts[0] > 0 and ref_counts[2] > 0            # children evaluated, some through the fallback
    for _ in range(2):                                        # two calls in a row, sharing the scratch
        nxt = torch.full((cap, 12), 7, dtype=torch.int8, device='cuda')
        torch.cuda.synchronize()
        sums, counts = noalloc_level(L, cells.data_ptr(), n, nxt.data_ptr(), cap, last, thr)
        torch.cuda.synchronize()
        assert counts == ref_counts
        for a, b in zip(sums[0::2], ref_sums[0::2]):           # each sum's high part
            assert abs(a - b) <= 1e-13*abs(b), (a, b)
        assert np.all(np.abs((sums[0::2] + sums[1::2]) - (ref_sums[0::2] + ref_sums[1::2]))
                      <= 1e-13*np.abs(ref_sums[0::2]))
        if not last:
            k = ref_counts[1]
            assert k > 0 and torch.equal(nxt[:k].cpu(), ref_next[:k].cpu())


def test_noalloc_rejects_a_batch_beyond_its_scratch():
    import torch
    L = noalloc_lib()
    n = (1 << 18)//32 + 1                                      # one cell more than the scratch holds
    cells = torch.zeros((n, 12), dtype=torch.int8, device='cuda')
    sums = (C.c_double * 12)()
    counts = (C.c_longlong * 6)()
    rc = L.sqb_level_noalloc(GRAPH.encode(), H, K, cells.data_ptr(), n, ST, 1, 32.0, 1e-9, ABSERR, NEARF, DDSLACK,
                             1, 0, 1, None, 0, sums, counts, None)
    assert rc == -2 and b'split the cells' in L.sqb_error()
