"""Test infrastructure: Python access to the oracle, i.e. the reference built by oracle/Makefile into
oracle/_ref/.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs use it,
as the checker; the evaluator never does.

  * run(binary, h, N, eps, graphs, top=None, env=None): runs `<binary> run h N [eps] [top] GRAPH...` (the
    reference's CLI, driver/main.c:205-251) and parses its results file (driver/main.c:66-73);
  * fd / fq / fv: the reference's own kernels at given points (refshim.cc over libsqref.so, built with
    -ffp-contract=off so their double half rounds as the evaluator's FP64 kernels do).
"""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, '_ref')
SINCQED = os.path.join(REF_DIR, 'sincqed')
SINCQED_EXACT = os.path.join(REF_DIR, 'sincqed-exact')
SINCQED_DROPIN = os.path.join(REF_DIR, 'sincqed-dropin')
LIBSQREF = os.path.join(REF_DIR, 'libsqref.so')
LIBSQREF_PI6 = os.path.join(REF_DIR, 'libsqref_pi6.so')   # the pi6 class alone
BOXSUM = os.path.join(REF_DIR, 'boxsum_gl')

COLS = ['name', 'volkov', 'L', 'D', 'w', 'h', 'N', 'eps', 'top', 'value', 'err', 'disc', 'prune', 'trunc',
        'round', 'S_2h', 'evals', 'time_s', 'ref', 'diff']


def available(path=SINCQED):
    return os.path.exists(path)


def parse_results(text):
    """Rows of a reference results file; the Volkov string has spaces, so columns are taken from the right
    of the value column (the first signed number of 20+ characters, as driver/main.c:249 finds it)."""
    rows = []
    for line in text.splitlines():
        if not line.strip() or line.startswith('#'):
            continue
        tok = line.split()
        iv = next(i for i in range(1, len(tok)) if tok[i][0] in '+-' and len(tok[i]) >= 20 and 'e' in tok[i])
        r = dict(name=tok[0], volkov=' '.join(tok[1:iv - 7]), L=int(tok[iv - 7]), D=int(tok[iv - 6]),
                 w=int(tok[iv - 5]), h=float(tok[iv - 4]), N=int(tok[iv - 3]), eps=float(tok[iv - 2]),
                 top=int(tok[iv - 1]), value=float(tok[iv]), err=float(tok[iv + 1]), disc=float(tok[iv + 2]),
                 prune=float(tok[iv + 3]), trunc=float(tok[iv + 4]), round=float(tok[iv + 5]))
        r['S_2h'] = float(tok[iv + 6]) if tok[iv + 6] != '-' else float('nan')
        r['evals'] = int(tok[iv + 7])
        r['time_s'] = float(tok[iv + 8])
        rows.append(r)
    return rows


def run(binary, h, N, eps, graphs, top=None, env=None, timeout=3600, threads=None):
    """Run the reference CLI; returns (rows, stdout)."""
    with tempfile.TemporaryDirectory() as d:
        res = os.path.join(d, 'results.txt')
        e = dict(os.environ)
        e.update(SINCQED_LOG='-', SINCQED_RESULTS=res, SINCQED_CKPT='0', SINCQED_PROGRESS='0')
        if threads:
            e['OMP_NUM_THREADS'] = str(threads)
        if env:
            e.update(env)
        args = [binary, 'run', repr(float(h)), str(int(N)), repr(float(eps))]
        if top is not None:
            args.append(str(int(top)))
        args += list(graphs)
        out = subprocess.run(args, cwd=d, env=e, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                             timeout=timeout)
        if out.returncode:
            raise RuntimeError('%s failed (%d):\n%s' % (binary, out.returncode, out.stdout[-3000:]))
        with open(res) as f:
            return parse_results(f.read()), out.stdout


_libs = {}


def lib(path=None):
    """the kernels' shim library (default libsqref.so; LIBSQREF_PI6 for the pi6 class)"""
    path = path or LIBSQREF
    if path not in _libs:
        L = C.CDLL(path)
        L.sqref_info.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
        for fn in (L.sqref_fd, L.sqref_fv):
            fn.argtypes = [C.c_char_p, C.c_long, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.sqref_fq.argtypes = [C.c_char_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p]
        L.sqref_name.restype = C.c_char_p
        L.sqref_volkov.restype = C.c_char_p
        L.sqref_volkov.argtypes = [C.c_char_p]
        _libs[path] = L
    return _libs[path]


def names(path=None):
    L = lib(path)
    return [L.sqref_name(i).decode() for i in range(L.sqref_count())]


def info(name, path=None):
    a = (C.c_int * 6)()
    if not lib(path).sqref_info(name.encode(), a):
        raise KeyError(name)
    return dict(L=a[0], D=a[1], weight=a[2], n=a[3], fixed=a[4], has_fv=bool(a[5]))


def fd(name, sf, sqab=1, path=None):
    sf = np.ascontiguousarray(sf, dtype=np.float64)
    f = np.empty(sf.shape[0]); ab = np.empty(sf.shape[0])
    if not lib(path).sqref_fd(name.encode(), sf.shape[0], sf.ctypes.data, int(sqab), f.ctypes.data, ab.ctypes.data):
        raise KeyError(name)
    return f, ab


def fv(name, sf, sqab=1):
    sf = np.ascontiguousarray(sf, dtype=np.float64)
    f = np.empty(sf.shape[0]); ab = np.empty(sf.shape[0])
    if not lib().sqref_fv(name.encode(), sf.shape[0], sf.ctypes.data, int(sqab), f.ctypes.data, ab.ctypes.data):
        return None
    return f, ab


def fq(name, sf, path=None):
    """double-double value and |.| sum as (n, 2) arrays of (hi, lo)"""
    sf = np.ascontiguousarray(sf, dtype=np.float64)
    f = np.empty((sf.shape[0], 2)); ab = np.empty((sf.shape[0], 2))
    if not lib(path).sqref_fq(name.encode(), sf.shape[0], sf.ctypes.data, f.ctypes.data, ab.ctypes.data):
        raise KeyError(name)
    return f, ab
