#!/usr/bin/env python3
"""Test infrastructure: the reference's own GPU kernels against this evaluator's, on one B200.

The reference's GPU build (oracle/Makefile `refgpu`: its driver/gpu_kernel.h kernels written by its
tools/gpugen.py, compiled for sm_100a with -fmad=false as its Makefile:180-235 does) exports one
GG_<graph> plug-in descriptor per graph (driver/gpu.h:17-21), and so does sincfeyn_b200/lib/libsqb200.so.
Both launchers take the same arguments, so the two kernels run here on the same device buffers:

  kernels   for each graph, 2^22 seeded nodes (int16 k uniform in [-K, K], h = 0.7, K = 72, every node with
            its |.| sums): the reference's gk_<graph> through its GG_<graph>, this evaluator's FP64 kernel
            as written (GG_<graph>) and contracted (sqb_plugin_launch form 2); CUDA events on one stream,
            3 warm-up launches, the median of 10; the values compared (the as-written kernels must agree
            bit for bit) and the algorithmic FP64 rate of each;
  runs      whole `run` commands through each program: the reference GPU build (oracle/_ref/sincqed-gpu:
            its driver, its kernels, its SIMD double-double fallback on the host) and this evaluator's
            command line (sincfeyn_b200/bin/sincqed), wall time and the results' time and evaluations.

    python oracle/refgpu_bench.py [--graphs g3_00,g3_07,...] [--runs] [--out FILE]

Prints one JSON line per measurement.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)
REFGPU_LIB = os.path.join(HERE, '_ref', 'libsqrefgpu.so')
REFGPU_BIN = os.path.join(HERE, '_ref', 'sincqed-gpu')
OURS_BIN = os.path.join(ROOT, 'sincfeyn_b200', 'bin', 'sincqed')

LAUNCH = C.CFUNCTYPE(None, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                     C.c_void_p, C.c_void_p, C.c_int, C.c_int)


class GpuDesc(C.Structure):
    """sq_gpu_t of driver/gpu.h:20"""
    _fields_ = [('name', C.c_char_p), ('D', C.c_int), ('launch', LAUNCH)]


def gg(lib, name):
    return GpuDesc.in_dll(lib, 'GG_' + name)


def time_launches(fn, stream, warm=3, reps=10):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts), min(ts)


def kernels(graphs, npts=1 << 22, h=0.7, K=72, seed=1):
    import numpy as np
    import torch
    from sincfeyn_b200 import sq
    ref = C.CDLL(REFGPU_LIB)
    ours = sq.lib()
    ours.sqb_plugin_launch.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_long, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    ours.sqb_plugin_launch.restype = C.c_int
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    ex = torch.tensor([math.exp(k*h) for k in range(-K, K + 1)], dtype=torch.float64, device='cuda')
    info = {g['name']: g for g in sq.graphs()}
    out = []
    for g in graphs:
        D = info[g]['D']
        rng = np.random.default_rng(seed)
        k = torch.from_numpy(rng.integers(-K, K + 1, size=(npts, D)).astype(np.int16)).cuda()
        res = {}
        for form in ('reference', 'ours_as_written', 'ours_contracted'):
            of = torch.zeros(npts, dtype=torch.float64, device='cuda')
            oab = torch.zeros(npts, dtype=torch.float64, device='cuda')
            if form == 'reference':
                d = gg(ref, g)
                assert d.D == D
                fn = lambda d=d, of=of, oab=oab: d.launch(sp, npts, k.data_ptr(), None, ex.data_ptr(), K, h,
                                                          of.data_ptr(), oab.data_ptr(), 0, 0)
            else:
                f_ = 0 if form == 'ours_as_written' else 2

                def fn(f_=f_, of=of, oab=oab):
                    rc = ours.sqb_plugin_launch(g.encode(), f_, sp, npts, k.data_ptr(), None, ex.data_ptr(), K, h,
                                                of.data_ptr(), oab.data_ptr(), 0, 0)
                    if rc:
                        raise RuntimeError(ours.sqb_error())
            med, mn = time_launches(fn, stream)
            res[form] = (med, mn, of.cpu().numpy(), oab.cpu().numpy())
        fl = sq.flops(g, 1)*npts
        rf, ra = res['reference'][2], res['reference'][3]
        row = {'graph': g, 'D': D, 'points': npts, 'h': h, 'K': K, 'flops_per_point': sq.flops(g, 1)}
        for form, (med, mn, f, a) in res.items():
            row[form] = {'ms': med, 'ms_min': mn, 'points_s': npts/(med*1e-3), 'tflops': fl/(med*1e-3)/1e12}
            if form != 'reference':
                fin = np.isfinite(rf)
                row[form]['bitwise_equal_f'] = float(np.mean(f[fin] == rf[fin]))
                row[form]['max_abs_diff_over_ab'] = float(np.max(np.abs(f[fin] - rf[fin])/np.maximum(ra[fin], 1e-300)))
                row[form]['speedup_vs_reference'] = res['reference'][0]/med
        out.append(row)
        print(json.dumps(row), flush=True)
    return out


def run_cmd(binary, h, N, eps, sel, env=None):
    with tempfile.TemporaryDirectory() as d:
        res = os.path.join(d, 'r.txt')
        e = dict(os.environ, SINCQED_LOG='-', SINCQED_RESULTS=res, SINCQED_CKPT='0', SINCQED_PROGRESS='0')
        e.update(env or {})
        t0 = time.perf_counter()
        p = subprocess.run([binary, 'run', repr(h), str(N), repr(eps)] + sel, cwd=d, env=e, stdout=subprocess.PIPE,
                           stderr=subprocess.STDOUT, text=True, timeout=3600)
        wall = time.perf_counter() - t0
        if p.returncode:
            raise RuntimeError('%s failed: %s' % (binary, p.stdout[-2000:]))
        import refpy
        with open(res) as f:
            rows = refpy.parse_results(f.read())
    return wall, rows


def runs(cases):
    out = []
    for h, N, eps, sel in cases:
        row = {'run': 'run %g %d %g %s' % (h, N, eps, ' '.join(sel))}
        for label, binary in (('reference_gpu', REFGPU_BIN), ('ours', OURS_BIN)):
            wall, rows = run_cmd(binary, h, N, eps, sel)
            row[label] = {'wall_s': wall, 'time_s': sum(r['time_s'] for r in rows), 'evals': sum(r['evals'] for r in rows),
                          'values': {r['name']: r['value'] for r in rows}}
        row['wall_ratio'] = row['reference_gpu']['wall_s']/row['ours']['wall_s']
        row['max_rel_diff'] = max(abs(row['ours']['values'][g] - v)/abs(v) for g, v in row['reference_gpu']['values'].items())
        out.append(row)
        print(json.dumps(row), flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--graphs', default='g3_00,g3_07,g3_01,g3_lbl,g2_00,v3_01')
    ap.add_argument('--npoints', type=int, default=1 << 22)
    ap.add_argument('--runs', action='store_true', help='whole runs: all2 at h=1.0 and g3_00 at h=0.7')
    ap.add_argument('--no-kernels', action='store_true')
    ap.add_argument('--out', default=None)
    a = ap.parse_args()
    allout = {}
    if not a.no_kernels:
        allout['kernels'] = kernels(a.graphs.split(','), a.npoints)
    if a.runs:
        allout['runs'] = runs([(1.0, 97, 1e-12, ['all2']), (0.7, 139, 1e-12, ['g3_00'])])
    if a.out:
        with open(a.out, 'w') as f:
            json.dump(allout, f, indent=1)


if __name__ == '__main__':
    main()
