"""Where the contracted FP64 form's point set differs, and why (GPU).

The contracted kernels round differently from the as-written ones by a few ulp of the |.| sum, so a
point whose value lies within that distance of the keep threshold thr = eps Ref 1e-2 can be kept in one
form and dropped in the other; its 2^D children are then evaluated in one form only.  This test lists
those points for v3_03 at h = 0.7, N = 139 (one of the integrals whose evaluation count differs between
the forms): it takes the kept cells after the step-2h level from each form's checkpoint, and for every
cell kept by one form only it evaluates the point with both FP64 kernels and checks that the two values
straddle the threshold and differ by no more than the kernels' rounding (16 ulp of the |.| sum)."""
import os

import numpy as np
import pytest

from sincfeyn_b200 import sq

pytestmark = pytest.mark.gpu


def kept_after_first_level(d, name, h, N, eps, fma):
    assert sq.hsum(name, h, N, eps, ckpt_every=600, ckpt_dir=d, ckpt_stop=1, fma=fma) is None
    ck = sq.ckpt_load(os.path.join(d, 'sincqed_%s.ckpt' % name))
    os.remove(os.path.join(d, 'sincqed_%s.ckpt' % name))
    return ck


def test_contracted_point_set_differs_only_at_the_threshold(tmp_path):
    name, h, N, eps = 'v3_03', 0.7, 139, 1e-12
    D = {g['name']: g['D'] for g in sq.graphs()}[name]
    a = kept_after_first_level(str(tmp_path), name, h, N, eps, 0)
    b = kept_after_first_level(str(tmp_path), name, h, N, eps, 1)
    # the same top level in both forms; its reference scale Ref (a sum of |f w|) differs by rounding
    assert a['kept_top'] == b['kept_top'] and abs(a['ref'] - b['ref']) <= 1e-12*a['ref']
    ka = {bytes(r[:D].tobytes()) for r in a['cur']}
    kb = {bytes(r[:D].tobytes()) for r in b['cur']}
    diff = sorted(ka ^ kb)
    assert len(diff) <= 1e-4*len(ka) + 4, len(diff)
    thr0, thr2 = eps*a['ref']*1e-2, eps*b['ref']*1e-2     # each form's keep threshold
    listing = []
    if diff:
        k = np.array([np.frombuffer(x, dtype=np.int8) for x in diff], dtype=np.float64)
        sf = np.exp(k*h)
        w = np.prod(sf*h, axis=1)
        f0, ab0 = sq.eval_points(name, sf, 0, 1)
        f2, _ = sq.eval_points(name, sf, 2, 1)
        for i, key in enumerate(diff):
            v0, v2 = abs(f0[i]*w[i]), abs(f2[i]*w[i])
            listing.append((tuple(int(x) for x in k[i]), 'as-written' if key in ka else 'contracted', v0/thr0, v2/thr2))
            # kept by exactly the form whose value reaches its threshold
            assert (v0 >= thr0) == (key in ka) and (v2 >= thr2) == (key in kb), listing[-1]
            # and within rounding of it: the two kernels' difference plus the two thresholds' difference
            tol = 16*np.finfo(float).eps*ab0[i]*w[i] + abs(thr0 - thr2)
            assert abs(v0 - thr0) <= tol and abs(v2 - thr2) <= tol, listing[-1]
    for k, kept_by, r0, r2 in listing:
        print('%s k=%s kept only by the %s form: |v|/thr = %.15f (as written), %.15f (contracted)' % (name, k, kept_by, r0, r2))
