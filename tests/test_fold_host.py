"""The symmetry fold's per-point rules on the CPU: sincfeyn_b200/csrc/sqorbit.cuh (the functions the
evaluation kernels, the level reduce and scatter and the predictor run on the device), compiled for the
host, against a restatement of the reference's symw() and symorbit() (driver/sum.c:29-46).

For the groups the reference finds for every graph (tests/golden/fold.json: generators closed under
composition in symadd()'s order, driver/sum.c:490-504) and seeded lattice points, many with repeated
coordinates so that stabilisers are not trivial: the compile-time-D and run-time-D orbit tests give the
reference's value (0, or the orbit size), and the orbit members come in the reference's order."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, 'sincfeyn_b200', 'csrc')
OUT = os.path.join(ROOT, 'tests', '_hostgen')

SRC = r'''
#include <string.h>
#include "sqorbit.cuh"
static sqb_sym_t mk(const signed char *g, int n){ sqb_sym_t s; memset(&s, 0, sizeof s); s.n = n; memcpy(s.g, g, (size_t)n*12); return s; }
template<int D> static int fixed(const sqb_sym_t &s, const int *k){ int kk[D]; for(int d = 0; d < D; d++) kk[d] = k[d]; return sqb_orbit<D>(s, kk); }
extern "C" int h_orbit(int D, const int *k, const signed char *g, int n){
    const sqb_sym_t s = mk(g, n);
    switch(D){ case 3: return fixed<3>(s, k); case 4: return fixed<4>(s, k); case 5: return fixed<5>(s, k);
               case 6: return fixed<6>(s, k); case 7: return fixed<7>(s, k); case 8: return fixed<8>(s, k);
               case 9: return fixed<9>(s, k); case 10: return fixed<10>(s, k); case 11: return fixed<11>(s, k); }
    return -1;
}
extern "C" int h_orbit_n(int D, const int *k, const signed char *g, int n){ return sqb_orbit_n(mk(g, n), k, D); }
extern "C" int h_members(int D, const int *k, const signed char *g, int n, int *out){
    const sqb_sym_t s = mk(g, n); int m = 0;
    for(int e = 0; e < n; e++) if(sqb_image_new(s, k, D, e)){ sqb_image(s, k, D, e, out + m*D); m++; }
    return m;
}
'''


@pytest.fixture(scope='module')
def lib():
    os.makedirs(OUT, exist_ok=True)
    cc = os.path.join(OUT, 'orbit_host.cc')
    so = os.path.join(OUT, 'orbit_host.so')
    deps = [os.path.join(CSRC, f) for f in ('sqorbit.cuh', 'sqdd.cuh', 'sqb_internal.h')]
    if not os.path.exists(so) or not os.path.exists(cc) or open(cc).read() != SRC or \
            any(os.path.getmtime(d) > os.path.getmtime(so) for d in deps):
        with open(cc, 'w') as f:
            f.write(SRC)
        subprocess.run(['g++', '-O1', '-std=c++17', '-shared', '-fPIC', '-I' + CSRC, '-o', so, cc], check=True)
    return C.CDLL(so)


def closure(gens, D):
    """symadd() for each generator in turn (driver/sum.c:490-504): products a o b with both indices
    running over the growing list"""
    G = [list(range(D))]
    for p in gens:
        if p in G:
            continue
        H = G + [p]
        a = 0
        while a < len(H):
            b = 0
            while b < len(H):
                c = [H[a][H[b][i]] for i in range(D)]
                if c not in H:
                    H.append(c)
                b += 1
            a += 1
        G = H
    return G


def symw(k, G):
    stab = 1
    for g in G[1:]:
        img = [k[g[i]] for i in range(len(k))]
        if img < k:
            return 0
        if img == k:
            stab += 1
    return len(G)//stab


def symorbit(k, G):
    out = [list(k)]
    for g in G[1:]:
        img = [k[g[i]] for i in range(len(k))]
        if img not in out:
            out.append(img)
    return out


def test_orbit_rules_match_the_reference(lib):
    with open(os.path.join(ROOT, 'tests', 'golden', 'fold.json')) as f:
        groups = json.load(f)['groups']
    rng = np.random.default_rng(7)
    checked = 0
    for name, grp in sorted(groups.items()):
        gens = [[int(x) for x in part.split(',')] for part in grp['desc'].split(';')]
        D = len(gens[0])
        G = closure(gens, D)
        assert len(G) == grp['order'], name
        g = np.zeros((len(G), 12), dtype=np.int8)
        g[:, :D] = np.array(G)
        gp = g.ctypes.data_as(C.POINTER(C.c_byte))
        for t in range(60):
            k = [int(x) for x in rng.integers(-2, 3, size=D)] if t % 2 else [int(x) for x in rng.integers(-72, 73, size=D)]
            ka = (C.c_int * D)(*k)
            want = symw(k, G)
            assert lib.h_orbit(D, ka, gp, len(G)) == want, (name, k)
            assert lib.h_orbit_n(D, ka, gp, len(G)) == want, (name, k)
            out = (C.c_int * (D*len(G)))()
            m = lib.h_members(D, ka, gp, len(G), out)
            orb = symorbit(k, G)
            assert m == len(orb) and [list(out[i*D:(i + 1)*D]) for i in range(m)] == orb, (name, k)
            if want:
                assert want == len(orb)
            checked += 1
    assert checked >= 100*60
