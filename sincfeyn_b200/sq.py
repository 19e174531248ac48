"""Python mirror of the evaluator's C ABI (include/sincfeyn_b200.h), over ctypes.

The library is sincfeyn_b200/lib/libsqb200.so, built in-tree by sincfeyn_b200.build.  There is no other
implementation behind these functions: if the library is missing, or the CUDA device cannot be used,
they raise.

    import sincfeyn_b200.sq as sq
    r = sq.hsum('g2_00', 1.0, 97, 1e-12)          # the reference's hsum() for one graph
    rows = sq.run(1.0, 97, 1e-12, ['all2'])       # `sincqed run 1.0 97 1e-12 all2`, one row per graph
"""
import ctypes as C
import math
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'lib', 'libsqb200.so')
_lib = None


class Opts(C.Structure):
    """sqb_opts_t: the reference's environment settings that reach the hot path (driver/main.c:176-185)."""
    _fields_ = [('abserr0', C.c_double), ('abrel', C.c_double), ('nearf', C.c_double), ('ddslack', C.c_double),
                ('abskip', C.c_int), ('abcheck', C.c_int), ('dropunres', C.c_int), ('growskip', C.c_int),
                ('alldd', C.c_int), ('device', C.c_int), ('max_children', C.c_long), ('verbose', C.c_int),
                ('ckpt_every', C.c_double), ('ckpt_dir', C.c_char_p), ('ckpt_stop', C.c_int), ('fma', C.c_int),
                ('split', C.c_int), ('sym', C.c_char_p), ('predict', C.c_double), ('group', C.c_int)]


class Result(C.Structure):
    """sqb_result_t: res_t of the reference (driver/sq.h:111) plus the log counters and timings."""
    _fields_ = [('S', C.c_double * 3), ('Ah', C.c_double), ('ref', C.c_double), ('prune', C.c_double),
                ('trunc', C.c_double), ('unres', C.c_double), ('t', C.c_double),
                ('nev', C.c_long), ('nq', C.c_long), ('kept_top', C.c_long),
                ('es1', C.c_double), ('es2', C.c_double), ('esok', C.c_int),
                ('abskipped', C.c_long), ('unresdrop', C.c_long), ('zero', C.c_int),
                ('t_top', C.c_double), ('t_levels', C.c_double), ('nlev', C.c_int),
                ('lev_evals', C.c_long * 16), ('lev_ms', C.c_double * 16),
                ('f64_ms', C.c_double), ('dd_ms', C.c_double), ('f64_launches', C.c_long), ('launches', C.c_long),
                ('sym_order', C.c_int), ('sym_desc', C.c_char * 256), ('sym_worst', C.c_double),
                ('sym_msg', C.c_char * 512), ('pskip', C.c_long)]


class ScaleResult(C.Structure):
    """sqb_scale_result_t: the scaling test of one graph (driver/main.c:76-115)."""
    _fields_ = [('n', C.c_int), ('fixed', C.c_int), ('ndir', C.c_long), ('slow', C.c_int), ('worst', C.c_double),
                ('worst_dir', C.c_long), ('worst_e', C.c_int * 16), ('worst_g', C.c_double * 3),
                ('listed_e', (C.c_int * 16) * 12), ('listed_g', (C.c_double * 3) * 12)]


class Job(C.Structure):
    """sqb_job_t: one integral of a batch."""
    _fields_ = [('graph', C.c_char_p), ('h', C.c_double), ('N', C.c_int), ('eps', C.c_double), ('top', C.c_int),
                ('cost', C.c_double)]


class SqbError(RuntimeError):
    pass


# sqb_sym_eval_fn: (ctx, n, k[n*D], f[n], ab[n]) -> 0
SYM_EVAL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_long, C.POINTER(C.c_int), C.POINTER(C.c_double),
                          C.POINTER(C.c_double))


def lib():
    """The loaded C-ABI library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SqbError('%s is missing: build it with `python -m sincfeyn_b200.build`' % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        L.sqb_default_opts.argtypes = [C.POINTER(Opts)]
        L.sqb_hsum.argtypes = [C.c_char_p, C.c_double, C.c_int, C.c_double, C.c_int, C.POINTER(Opts), C.POINTER(Result)]
        L.sqb_hsum.restype = C.c_int
        L.sqb_error.restype = C.c_char_p
        L.sqb_graph_count.restype = C.c_int
        L.sqb_graph_name.argtypes = [C.c_int]
        L.sqb_graph_name.restype = C.c_char_p
        L.sqb_graph_volkov.argtypes = [C.c_char_p]
        L.sqb_graph_volkov.restype = C.c_char_p
        L.sqb_graph_info.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
        L.sqb_graph_flops.argtypes = [C.c_char_p, C.c_int]
        L.sqb_graph_flops.restype = C.c_double
        L.sqb_eval_points.argtypes = [C.c_char_p, C.c_long, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.sqb_eval_points.restype = C.c_int
        L.sqb_device_info.restype = C.c_char_p
        L.sqb_kernel_timing.argtypes = [C.c_int]
        L.sqb_probe_fp64.argtypes = [C.c_int, C.c_long]
        L.sqb_probe_fp64.restype = C.c_double
        L.gpu_info.restype = C.c_char_p
        L.sqb_hsum_batch.argtypes = [C.POINTER(Job), C.c_int, C.POINTER(Opts), C.c_int, C.POINTER(Result),
                                     C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.sqb_batch_tune.argtypes = [C.POINTER(Job), C.c_int, C.POINTER(Opts), C.POINTER(C.c_int), C.c_int,
                                     C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.sqb_sym_find.argtypes = [C.c_int, SYM_EVAL_FN, C.c_void_p, C.c_char_p, C.POINTER(C.c_int), C.c_char_p,
                                   C.c_int, C.POINTER(C.c_double), C.c_char_p, C.c_int]
        L.sqb_sym_find.restype = C.c_int
        _lib = L
    return _lib


def default_opts(**kw):
    o = Opts()
    lib().sqb_default_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v.encode() if isinstance(v, str) else v)
    return o


CKPT_STOPPED = 2


class Checkpoint(C.Structure):
    """sqb_ckpt_t: the reference's checkpoint (SQCK4), field for field."""
    _fields_ = [('name', C.c_char * 32), ('h', C.c_double), ('eps', C.c_double), ('N', C.c_int), ('top', C.c_int),
                ('dim', C.c_int), ('k', C.c_int), ('lev', C.c_int), ('next', C.c_long),
                ('s', C.c_double), ('a', C.c_double), ('drop', C.c_double), ('u', C.c_double),
                ('ne', C.c_long), ('q', C.c_long), ('Slev', C.c_double * 16), ('nl', C.c_int),
                ('S', C.c_double * 3), ('Ah', C.c_double), ('ref', C.c_double), ('prune', C.c_double),
                ('trunc', C.c_double), ('unres', C.c_double), ('t', C.c_double),
                ('nev', C.c_long), ('nq', C.c_long), ('kept_top', C.c_long),
                ('ncur', C.c_long), ('cur', C.POINTER(C.c_byte)), ('nnxt', C.c_long), ('nxt', C.POINTER(C.c_byte)),
                ('es', C.c_double * 5), ('cnt', C.c_long * 3), ('esok', C.c_int),
                ('vsz', C.c_int), ('vcap', C.c_long), ('vn', C.c_long), ('vs', C.c_void_p)]


def ckpt_load(path):
    """Read a checkpoint file: None if absent; a dict of its fields, the cell lists as (n, 12) int8 arrays."""
    L = lib()
    L.sqb_ckpt_load.argtypes = [C.c_char_p, C.POINTER(Checkpoint)]
    L.sqb_ckpt_free.argtypes = [C.POINTER(Checkpoint)]
    c = Checkpoint()
    rc = L.sqb_ckpt_load(path.encode(), C.byref(c))
    if rc == 0:
        return None
    if rc < 0:
        raise SqbError('%s: damaged or not SQCK4' % path)
    d = {f: getattr(c, f) for f, _ in Checkpoint._fields_ if f not in ('cur', 'nxt', 'vs')}
    d['name'] = c.name.decode()
    for f in ('Slev', 'S', 'es', 'cnt'):
        d[f] = list(d[f])
    for f, n in (('cur', c.ncur), ('nxt', c.nnxt)):
        d[f] = np.ctypeslib.as_array(getattr(c, f), shape=(n * 12,)).reshape(n, 12).copy() if n else np.zeros((0, 12), np.int8)
    L.sqb_ckpt_free(C.byref(c))
    return d


def ckpt_save(path, d):
    """Write a checkpoint from a dict shaped like ckpt_load()'s (the predictor table empty)."""
    L = lib()
    L.sqb_ckpt_save.argtypes = [C.c_char_p, C.POINTER(Checkpoint)]
    c = Checkpoint()
    keep = []
    for f, _ in Checkpoint._fields_:
        if f in ('cur', 'nxt'):
            a = np.ascontiguousarray(d[f], dtype=np.int8).reshape(-1)
            keep.append(a)
            setattr(c, f, a.ctypes.data_as(C.POINTER(C.c_byte)))
        elif f == 'name':
            c.name = d['name'].encode()
        elif f == 'vs':
            c.vs = None
        elif f in ('Slev', 'S', 'es', 'cnt'):
            arr = getattr(c, f)
            for i, x in enumerate(d[f]):
                arr[i] = x
        elif f in d:
            setattr(c, f, d[f])
    c.vcap = 0
    if L.sqb_ckpt_save(path.encode(), C.byref(c)):
        raise SqbError('could not write %s' % path)


def graphs():
    """[{name, volkov, L, D, weight, n, fixed}] of the graphs compiled into the library, in registry order."""
    L = lib()
    out = []
    for i in range(L.sqb_graph_count()):
        name = L.sqb_graph_name(i)
        info = (C.c_int * 6)()
        L.sqb_graph_info(name, info)
        out.append(dict(name=name.decode(), volkov=L.sqb_graph_volkov(name).decode(), L=info[0], D=info[1],
                        weight=info[2], n=info[3], fixed=info[4]))
    return out


def flops(name, ab=1):
    """Algorithmic FP64 flops per point of the graph's double path (with or without the |.| sums)."""
    return lib().sqb_graph_flops(name.encode(), int(ab))


def default_top(h):
    """driver/main.c:211-215 (SINCQED_TOPSTEP = 3)."""
    top = 1
    while top < 2 and (1 << (top + 1)) * h <= 3.0 * (1 + 1e-9):
        top += 1
    return top


def hsum(graph, h, N, eps, top=-1, **opts):
    """The hierarchical Sinc sum of one graph; returns the result fields as a dict."""
    o = default_opts(**opts)
    r = Result()
    rc = lib().sqb_hsum(graph.encode(), float(h), int(N), float(eps), int(top), C.byref(o), C.byref(r))
    if rc == CKPT_STOPPED and opts.get('ckpt_stop'):
        return None
    if rc:
        raise SqbError('%s: %s' % (graph, lib().sqb_error().decode()))
    return _result_dict(r)


def _result_dict(r):
    d = {f: getattr(r, f) for f, _ in Result._fields_}
    d['sym_desc'] = r.sym_desc.decode()
    d['sym_msg'] = r.sym_msg.decode()
    d['S'] = list(r.S)
    d['lev_evals'] = list(r.lev_evals)[:r.nlev]
    d['lev_ms'] = list(r.lev_ms)[:r.nlev]
    return d


def _jobs(jobs):
    """[(graph, h, N, eps[, top[, cost]])] -> a sqb_job_t array (top -1: the default)"""
    arr = (Job * len(jobs))()
    for i, j in enumerate(jobs):
        g, h, N, eps = j[:4]
        arr[i] = Job(g.encode(), float(h), int(N), float(eps), int(j[4]) if len(j) > 4 else -1,
                     float(j[5]) if len(j) > 5 else 0.0)
    return arr


def hsum_batch(jobs, workers=4, **opts):
    """Many integrals concurrently (sqb_hsum_batch): jobs = [(graph, h, N, eps[, top[, cost]])].
    Returns (results in job order as hsum() dicts, device milliseconds of the whole batch)."""
    arr = _jobs(jobs)
    n = len(jobs)
    res = (Result * max(1, n))()
    rcs = (C.c_int * max(1, n))()
    ms = C.c_double()
    o = default_opts(**opts)
    rc = lib().sqb_hsum_batch(arr, n, C.byref(o), int(workers), res, rcs, C.byref(ms))
    if rc:
        raise SqbError('batch: %d failed: %s' % (rc, lib().sqb_error().decode()))
    return [_result_dict(res[i]) for i in range(n)], ms.value


def hsum_group(jobs, **opts):
    """Several integrals of one graph as one group (sqb_hsum_group): jobs = [(graph, h, N, eps[, top])], at
    most 8, all of the same graph; their refinement levels run as shared launches.  Returns the results
    in job order as hsum() dicts (each bit for bit the hsum() result)."""
    arr = _jobs(jobs)
    n = len(jobs)
    res = (Result * max(1, n))()
    rcs = (C.c_int * max(1, n))()
    o = default_opts(**opts)
    L = lib()
    L.sqb_hsum_group.argtypes = [C.POINTER(Job), C.c_int, C.POINTER(Opts), C.POINTER(Result), C.POINTER(C.c_int)]
    rc = L.sqb_hsum_group(arr, n, C.byref(o), res, rcs)
    if rc:
        raise SqbError('group: %d failed: %s' % (rc, L.sqb_error().decode()))
    return [_result_dict(res[i]) for i in range(n)]


def batch_tune(jobs, candidates=(1, 2, 4, 6, 8), **opts):
    """The batch tuner (sqb_batch_tune): runs the calibration jobs twice per candidate worker count;
    returns (best worker count, {count: points per second of device time, the better run})."""
    arr = _jobs(jobs)
    cand = (C.c_int * len(candidates))(*candidates)
    rate = (C.c_double * len(candidates))()
    best = C.c_int()
    o = default_opts(**opts)
    rc = lib().sqb_batch_tune(arr, len(jobs), C.byref(o), cand, len(candidates), rate, C.byref(best))
    if rc:
        raise SqbError('tune: %s' % lib().sqb_error().decode())
    return best.value, {c: rate[i] for i, c in enumerate(candidates)}


def select(selectors):
    """Graph names matched by names, Volkov strings or groups (driver/graphs.c:15-29), in order."""
    gs = graphs()

    def hit(g, s):
        n = g['name']
        if s in (n, g['volkov']):
            return True
        return {'all2': g['L'] == 2, 'all3': g['L'] == 3 and not n.startswith('w3_'), 'all4': g['L'] == 4,
                'q3': n.startswith('g3_') and n != 'g3_lbl', 'vp3': n.startswith('v3_'),
                'vp4': n.startswith('v4_') or n.startswith('w4_'), 'lbl': n == 'g3_lbl',
                'synth': n.startswith('syn_')}.get(s, False)
    out = []
    for s in selectors:
        for g in gs:
            if hit(g, s) and g['name'] not in out:
                out.append(g['name'])
    return out


def run(h, N, eps, selectors, top=-1, **opts):
    """`sincqed run h N eps [top] GRAPH...`: per graph its value (weight * S_h) and error columns, as the
    reference's run_graph() computes them (driver/main.c:40-75)."""
    if top < 0:
        top = default_top(h)
    info = {g['name']: g for g in graphs()}
    rows = []
    for name in select(selectors):
        r = hsum(name, h, N, eps, top, **opts)
        w = info[name]['weight']
        S0, S1 = r['S'][0], r['S'][1]
        d2 = abs(S1 - S0) if not math.isnan(S1) else float('nan')
        disc = 2 * d2 * d2 / r['Ah'] if r['Ah'] > 0 else 0.0
        err = w * (disc + r['prune'] + r['trunc'] + r['unres'])
        rows.append(dict(name=name, D=info[name]['D'], weight=w, value=w * S0, err=err, disc=w * disc,
                         prune=w * r['prune'], trunc=w * r['trunc'], round=w * r['unres'],
                         S_2h=w * S1, evals=r['nev'], quad=r['nq'], kept=r['kept_top'], time=r['t'], raw=r))
    return rows


def sym_find(D, evaluate, spec='auto'):
    """The symmetry fold's group search (sqb_sym_find) with a Python evaluator: evaluate(k) takes an
    (n, D) int array of lattice nodes and returns (f, ab) arrays of n values.  spec as Opts.sym.
    Returns dict(order, elems (order x D), desc, worst, msg)."""
    err = []

    def cb(_ctx, n, k, f, ab):
        try:
            kk = np.ctypeslib.as_array(k, shape=(n * D,)).reshape(n, D).copy()
            fv, av = evaluate(kk)
            np.ctypeslib.as_array(f, shape=(n,))[:] = fv
            np.ctypeslib.as_array(ab, shape=(n,))[:] = av
            return 0
        except Exception as e:  # reported after the call
            err.append(e)
            return -1
    fn = SYM_EVAL_FN(cb)
    el = (C.c_int * (64 * 12))()
    desc = C.create_string_buffer(1024)
    msg = C.create_string_buffer(2048)
    worst = C.c_double()
    n = lib().sqb_sym_find(int(D), fn, None, spec.encode() if spec else None, el, desc, len(desc), C.byref(worst),
                           msg, len(msg))
    if n < 0:
        raise SqbError('symmetry search failed: %r' % (err[0] if err else 'evaluator'))
    elems = np.array(el[:], dtype=np.int64).reshape(64, 12)[:n, :D]
    return dict(order=n, elems=elems, desc=desc.value.decode(), worst=worst.value, msg=msg.value.decode())


def scale_test(graph, kappa=24.0, seed=1, E=1):
    """`sincqed scale GRAPH kappa seed` for one graph on the device: None for a graph without a raw point
    function (VP), else a dict with the directions tested, the slow ones (first twelve listed with |g| at
    kappa/3, 2kappa/3, kappa) and the worst ratio with its direction."""
    L = lib()
    L.sqb_scale_test.argtypes = [C.c_char_p, C.c_double, C.c_uint, C.c_int, C.POINTER(ScaleResult)]
    r = ScaleResult()
    rc = L.sqb_scale_test(graph.encode(), float(kappa), int(seed), int(E), C.byref(r))
    if rc == 1:
        return None
    if rc:
        raise SqbError('%s: %s' % (graph, L.sqb_error().decode()))
    return _scale_dict(r)


def _scale_dict(r):
    free = [i for i in range(r.n) if i != r.fixed]
    return dict(n=r.n, fixed=r.fixed, ndir=r.ndir, slow=r.slow, worst=r.worst, worst_dir=r.worst_dir,
                worst_e=[r.worst_e[i] for i in free], worst_g=list(r.worst_g),
                listed=[([r.listed_e[j][i] for i in free], list(r.listed_g[j])) for j in range(min(r.slow, 12))])


def scale_setup(n, fixed, kappa=24.0, seed=1, E=1):
    """The scaling test's host half (sqb_scale_setup): the base point x0[n] and the factor table
    xs[3, 2E+1] for a caller that evaluates the point function itself."""
    L = lib()
    L.sqb_scale_setup.argtypes = [C.c_int, C.c_int, C.c_double, C.c_uint, C.c_int, C.c_void_p, C.c_void_p]
    x0 = np.zeros(n)
    xs = np.zeros(3 * (2 * E + 1))
    L.sqb_scale_setup(int(n), int(fixed), float(kappa), int(seed), int(E), x0.ctypes.data, xs.ctypes.data)
    return x0, xs


def scale_summary(n, fixed, E, g):
    """The scaling test's summary (sqb_scale_summary) of values g[3 d + q] over the (2E+1)^(n-1)
    directions, as scale_test() returns it."""
    L = lib()
    L.sqb_scale_summary.argtypes = [C.c_int, C.c_int, C.c_int, C.c_long, C.c_void_p, C.POINTER(ScaleResult)]
    g = np.ascontiguousarray(g, dtype=np.float64)
    r = ScaleResult()
    L.sqb_scale_summary(int(n), int(fixed), int(E), g.size // 3, g.ctypes.data, C.byref(r))
    return _scale_dict(r)


def eval_points(graph, sf, prec=0, ab=1):
    """The graph kernel at the points sf (n x D) on the device.  prec 0: FP64 (f, ab) arrays, every
    operation rounded as written; prec 2: FP64 with contraction (fused multiply-adds); prec 1:
    double-double, (f, ab) as (n, 2) arrays of (hi, lo)."""
    sf = np.ascontiguousarray(sf, dtype=np.float64)
    n = sf.shape[0]
    if prec in (0, 2):
        f = np.empty(n)
        a = np.empty(n)
    else:
        f = np.empty((n, 2))
        a = np.empty((n, 2))
    rc = lib().sqb_eval_points(graph.encode(), n, sf.ctypes.data, int(prec), int(ab), f.ctypes.data, a.ctypes.data)
    if rc:
        raise SqbError('%s: %s' % (graph, lib().sqb_error().decode()))
    return f, a


def device_info():
    return lib().sqb_device_info().decode()


def preload(graph=None):
    """Load the device code of a graph's kernels (None: all graphs) before timing or at start-up."""
    L = lib()
    L.sqb_preload.argtypes = [C.c_char_p]
    n = L.sqb_preload(graph.encode() if graph else None)
    if n < 0:
        raise SqbError('preload failed')
    return n


def kernel_timing(on=True):
    """Bracket the evaluation kernels with events; hsum() results then carry f64_ms and dd_ms."""
    lib().sqb_kernel_timing(1 if on else 0)


def probe_fp64(fma=True, iters=1 << 16):
    """The device's measured FP64 rate in TFLOP/s (FMA = 2 flops)."""
    r = lib().sqb_probe_fp64(1 if fma else 0, int(iters))
    if r < 0:
        raise SqbError('FP64 probe failed')
    return r
