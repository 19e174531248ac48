"""The chosen precision form against the all-double-double form (GPU), on the headline workload's
configuration (h = 0.7, N = 139, eps = 1e-12): a D = 7 three-loop graph (g3_00, 6.6e9 points) and a D = 6
graph with fallback points (g3_01, 7.5e6 of them).

The chosen form evaluates every point in FP64 and recomputes in double-double only the points whose |.|
bound exceeds ABSERR (driver/eval.c:33-53); the all-dd form evaluates every point in double-double.  Their
values must agree within the three-loop tolerance 1e-11 relative (the error of the FP64 + dd result
stated against the all-dd run), in both FP64 builds (contracted and as written), and the all-dd form's
extra evaluations of FP64-resolved points must not move the evaluation count by more than the keep
decisions at ties (1e-4)."""
import pytest

from sincfeyn_b200 import sq

pytestmark = pytest.mark.gpu
H, N, EPS = 0.7, 139, 1e-12


@pytest.mark.parametrize('graph', ['g3_00', 'g3_01'])
def test_fp64_with_dd_fallback_against_all_dd(graph):
    alldd = sq.hsum(graph, H, N, EPS, alldd=1)
    ref = alldd['S'][0]
    for fma in (1, 0):
        r = sq.hsum(graph, H, N, EPS, fma=fma)
        rel = abs(r['S'][0] - ref)/abs(ref)
        print('%s fma=%d: |FP64+dd - all-dd| / |all-dd| = %.2e (fallback points %d of %d)' % (graph, fma, rel, r['nq'], r['nev']))
        assert rel <= 1e-11, (graph, fma, r['S'][0], ref)
        assert abs(r['nev'] - alldd['nev']) <= 1e-4*alldd['nev'], (graph, fma, r['nev'], alldd['nev'])
