"""Concurrent batches (sqb_hsum_batch) against one integral at a time (GPU).

Each integral of a batch is one sqb_hsum() on a worker thread with its own stream and buffers; its
arithmetic does not depend on the schedule, so every result field that is not a time must be
identical to the one-at-a-time run, whatever the worker count and order."""
import pytest

from sincfeyn_b200 import sq

pytestmark = pytest.mark.gpu

FIELDS = ('S', 'Ah', 'ref', 'prune', 'trunc', 'unres', 'nev', 'nq', 'kept_top', 'abskipped', 'unresdrop')


def same(a, b):
    """equal, NaN equal to NaN (S_4h is NaN where a run has no such level)"""
    if isinstance(a, list):
        return len(a) == len(b) and all(same(x, y) for x, y in zip(a, b))
    return a == b or (a != a and b != b)


def _jobs():
    jobs = []
    for h, N in ((1.0, 97), (0.8, 121)):
        for g in sq.select(['all2']) + ['v3_01', 'g3_07']:
            jobs.append((g, h, N, 1e-12))
    return jobs


def test_batch_equals_one_at_a_time():
    jobs = _jobs()
    one = [sq.hsum(g, h, N, eps) for g, h, N, eps in jobs]
    for workers in (1, 3, 8):
        res, ms = sq.hsum_batch(jobs, workers=workers)
        assert ms > 0
        for j, a, b in zip(jobs, one, res):
            for f in FIELDS:
                assert same(a[f], b[f]), (workers, j, f, a[f], b[f])


def test_batch_order_by_cost_and_tuner():
    jobs = [j + (-1, float(i % 5)) for i, j in enumerate(_jobs())]
    res, ms = sq.hsum_batch(jobs, workers=4)
    ref = [sq.hsum(g, h, N, eps) for g, h, N, eps, _, _ in jobs]
    assert all(same(a['S'], b['S']) for a, b in zip(res, ref))
    best, rates = sq.batch_tune(jobs[:6], (1, 2))
    assert best in (1, 2) and all(v > 0 for v in rates.values())


def test_batch_reports_a_bad_graph():
    with pytest.raises(sq.SqbError):
        sq.hsum_batch([('no_such_graph', 1.0, 97, 1e-12)], workers=2)
