"""The FP64 pass of g3_lbl in passes (GPU).  g3_lbl's point function is a flat sum of twelve independent
forest nodes; with split = 1 its level batches run as passes over groups of nodes (one per main node, the
zero-momentum subtractions in pairs) and a final pass (kgen.split_plan).  Every operation and its order are
those of the single function, so with the as-written kernels the whole sum is bit for bit the single-pass
one; the contracted kernels may fuse differently inside a pass, so there the sums agree to the three-loop
tolerance."""
import pytest

from sincfeyn_b200 import sq

pytestmark = pytest.mark.gpu
FIELDS = ('S', 'Ah', 'ref', 'prune', 'trunc', 'unres', 'nev', 'nq', 'kept_top', 'abskipped')


def same(a, b):
    if isinstance(a, list):
        return all(same(x, y) for x, y in zip(a, b))
    return a == b or (a != a and b != b)


def test_split_as_written_is_bitwise():
    one = sq.hsum('g3_lbl', 1.0, 97, 1e-12, 1, fma=0, split=0)
    many = sq.hsum('g3_lbl', 1.0, 97, 1e-12, 1, fma=0, split=1)
    assert many['f64_launches'] >= one['f64_launches']
    for f in FIELDS:
        assert same(one[f], many[f]), (f, one[f], many[f])


def test_split_contracted_within_tolerance():
    one = sq.hsum('g3_lbl', 1.0, 97, 1e-12, 1, split=0)
    many = sq.hsum('g3_lbl', 1.0, 97, 1e-12, 1, split=1)
    assert abs(many['nev'] - one['nev']) <= 1e-4*one['nev']
    assert abs(many['S'][0] - one['S'][0]) <= 1e-11*abs(one['S'][0])

