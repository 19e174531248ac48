"""The checkpoint file (SQCK4) on the CPU: the evaluator's reader and writer (sqb_ckpt_save/load) against
the reference's own (driver/checkpoint.c:59-120, built into oracle/_ref/libsqck.so behind a C shim).

  - a file written by the evaluator is read by the reference with every field intact, and the reverse;
  - both writers produce the same bytes for the same state;
  - a truncated or foreign file is refused by the evaluator's reader, as by the reference's."""
import ctypes as C
import os
import shutil

import numpy as np
import pytest

from sincfeyn_b200 import sq

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBSQCK = os.path.join(ROOT, 'oracle', '_ref', 'libsqck.so')


class Res(C.Structure):
    _fields_ = [('S', C.c_double * 3), ('Ah', C.c_double), ('ref', C.c_double), ('prune', C.c_double),
                ('trunc', C.c_double), ('unres', C.c_double), ('t', C.c_double),
                ('nev', C.c_long), ('nq', C.c_long), ('kept_top', C.c_long)]


class Vec(C.Structure):
    _fields_ = [('p', C.POINTER(C.c_byte)), ('n', C.c_long), ('cap', C.c_long)]


class RefCkpt(C.Structure):
    """ckpt_t of the reference (driver/sq.h:84-93)"""
    _fields_ = [('lev', C.c_int), ('next', C.c_long), ('s', C.c_double), ('a', C.c_double), ('drop', C.c_double),
                ('u', C.c_double), ('ne', C.c_long), ('q', C.c_long), ('Slev', C.c_double * 16), ('nl', C.c_int),
                ('R', Res), ('cur', Vec), ('nxt', Vec), ('es', C.c_double * 5), ('cnt', C.c_long * 3),
                ('esok', C.c_int), ('vs', C.c_void_p), ('vcap', C.c_long), ('vn', C.c_long), ('vsz', C.c_int)]


@pytest.fixture(scope='module')
def ref():
    if not os.path.exists(LIBSQCK):
        pytest.skip('oracle/_ref/libsqck.so not built (make -C oracle)')
    L = C.CDLL(LIBSQCK)
    args = [C.c_char_p, C.c_char_p, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.POINTER(RefCkpt)]
    L.ref_ckpt_save.argtypes = args
    L.ref_ckpt_load.argtypes = args
    L.ref_ckpt_free.argtypes = [C.POINTER(RefCkpt)]
    assert L.ref_ckpt_sizeof() == C.sizeof(RefCkpt)
    return L


def state(seed, mid):
    rng = np.random.default_rng(seed)
    d = dict(name='g3_07', h=0.7, eps=1e-12, N=139, top=2, dim=7, k=72, lev=0, next=311 if mid else 0,
             s=rng.normal(), a=rng.random(), drop=rng.random()*1e-9, u=rng.random()*1e-30, ne=int(rng.integers(1e9)),
             q=int(rng.integers(1e6)), Slev=list(rng.normal(size=16)), nl=2, S=[0.0, 0.0, 0.0], Ah=0.0,
             ref=rng.random(), prune=rng.random()*1e-10, trunc=rng.random()*1e-12, unres=0.0, t=123.25,
             nev=int(rng.integers(1e10)), nq=int(rng.integers(1e7)), kept_top=int(rng.integers(1e6)),
             es=[rng.normal()*1e-3, rng.normal()*1e-4, 0.0, 0.0, 0.0], cnt=[0, int(rng.integers(1e5)), 0], esok=1,
             vsz=16, vcap=0, vn=0)
    d['Slev'][2:] = [0.0]*14
    d['cur'] = rng.integers(-72, 73, size=(1000, 12)).astype(np.int8)
    d['cur'][:, 7:11] = 0
    d['cur'][:, 11] = rng.integers(0, 6, size=1000)
    d['nxt'] = d['cur'][:37].copy() if mid else np.zeros((0, 12), np.int8)
    d['ncur'], d['nnxt'] = len(d['cur']), len(d['nxt'])
    return d


def to_ref(d):
    c = RefCkpt()
    keep = []
    for f in ('lev', 'next', 's', 'a', 'drop', 'u', 'ne', 'q', 'nl', 'esok', 'vcap', 'vn', 'vsz'):
        setattr(c, f, d[f])
    for f in ('Slev', 'es', 'cnt'):
        for i, x in enumerate(d[f]):
            getattr(c, f)[i] = x
    for f in ('Ah', 'ref', 'prune', 'trunc', 'unres', 't', 'nev', 'nq', 'kept_top'):
        setattr(c.R, f, d[f])
    for i, x in enumerate(d['S']):
        c.R.S[i] = x
    for f in ('cur', 'nxt'):
        a = np.ascontiguousarray(d[f], dtype=np.int8).reshape(-1)
        keep.append(a)
        v = getattr(c, f)
        v.p = a.ctypes.data_as(C.POINTER(C.c_byte))
        v.n = v.cap = len(d[f])
    return c, keep


def from_ref(c):
    d = {f: getattr(c, f) for f in ('lev', 'next', 's', 'a', 'drop', 'u', 'ne', 'q', 'nl', 'esok', 'vcap', 'vn', 'vsz')}
    for f in ('Slev', 'es', 'cnt'):
        d[f] = list(getattr(c, f))
    for f in ('Ah', 'ref', 'prune', 'trunc', 'unres', 't', 'nev', 'nq', 'kept_top'):
        d[f] = getattr(c.R, f)
    d['S'] = list(c.R.S)
    for f in ('cur', 'nxt'):
        v = getattr(c, f)
        d[f] = np.ctypeslib.as_array(v.p, shape=(v.n*12,)).reshape(v.n, 12).copy() if v.n else np.zeros((0, 12), np.int8)
    return d


def same(a, b):
    for f, x in b.items():
        if f in ('name', 'h', 'eps', 'N', 'top', 'dim', 'k', 'ncur', 'nnxt'):
            continue
        if isinstance(x, np.ndarray):
            np.testing.assert_array_equal(a[f], x)
        else:
            assert a[f] == x, f


def ref_args(d, tmp):
    return (str(tmp).encode(), d['name'].encode(), d['h'], d['N'], d['eps'], d['top'], d['dim'], d['k'])


@pytest.mark.parametrize('mid', [False, True], ids=['level-end', 'mid-level'])
def test_checkpoints_cross_read(ref, tmp_path, mid):
    d = state(11 + mid, mid)
    ours = tmp_path / 'ours'
    theirs = tmp_path / 'theirs'
    ours.mkdir()
    theirs.mkdir()
    fn = 'sincqed_%s.ckpt' % d['name']
    sq.ckpt_save(str(ours / fn), d)
    # the reference reads the evaluator's file
    c = RefCkpt()
    assert ref.ref_ckpt_load(*ref_args(d, ours), C.byref(c)) == 1
    same(from_ref(c), d)
    ref.ref_ckpt_free(C.byref(c))
    # the reference writes the same state: the same bytes, and the evaluator reads it back
    rc, keep = to_ref(d)
    assert ref.ref_ckpt_save(*ref_args(d, theirs), C.byref(rc)) == 0
    assert (ours / fn).read_bytes() == (theirs / fn).read_bytes()
    back = sq.ckpt_load(str(theirs / fn))
    same(back, d)
    assert (back['name'], back['h'], back['N'], back['eps'], back['top'], back['dim'], back['k']) == \
        (d['name'], d['h'], d['N'], d['eps'], d['top'], d['dim'], d['k'])


def test_damaged_and_foreign_files_are_refused(ref, tmp_path):
    d = state(5, False)
    fn = tmp_path / ('sincqed_%s.ckpt' % d['name'])
    sq.ckpt_save(str(fn), d)
    good = fn.read_bytes()
    assert sq.ckpt_load(str(tmp_path / 'absent.ckpt')) is None
    fn.write_bytes(good[:len(good) - 7])              # truncated in the last field
    with pytest.raises(sq.SqbError):
        sq.ckpt_load(str(fn))
    c = RefCkpt()
    assert ref.ref_ckpt_load(*ref_args(d, tmp_path), C.byref(c)) == 0
    fn.write_bytes(b'SQCK5\0\0\0' + good[8:])          # the five-loop format (MAXD 14)
    with pytest.raises(sq.SqbError):
        sq.ckpt_load(str(fn))
    # the reference ignores a checkpoint of another run (header differs): h
    fn.write_bytes(good)
    args = list(ref_args(d, tmp_path))
    args[2] = 0.8
    assert ref.ref_ckpt_load(*args, C.byref(c)) == 0
    shutil.rmtree(tmp_path, ignore_errors=True)
