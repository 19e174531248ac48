#!/usr/bin/env python3
"""Writes the golden fixtures in tests/golden/ from the reference itself (oracle/_ref, built by
oracle/Makefile from the reference sources).  Run from the repository root after `make -C oracle`:

    python tests/golden/make_golden.py

Fixtures
  all2_h1.0_N97_eps1e-12.json   `sincqed run 1.0 97 1e-12 all2`, the reference CPU build as shipped
                                (symmetry fold on) and the -ffp-contract=off build with SINCQED_SYM=0 (the
                                unfolded point set the GPU evaluates, driver/sum.c:571): every column of
                                every results line
  boxsum_gl.json                the reference's pointwise known-answer program
                                (mathematica/check/boxsum_gl.c): term values at k = 0 and k = (1,-1,2,0),
                                h = 1, and full-box sums at h = 1, K = 6, for the five two-loop kernels
  pointwise_<class>.npz         400 (g3: 128, v4/w4/pi6: 32) seeded nodes per graph, sigma = e^z, z ~ U[-3,3] (the protocol of
                                tests/check_onept.sh): fd with SQ_AB = 1 and 0 and fq (hi, lo) of the
                                reference kernels
  pointwise_synth.npz           the same for the synthetic integrands syn_d5, syn_d8, syn_d11 (64 nodes each),
                                evaluated by the oracle build (the synthetic sources compiled with the
                                reference's double-double type and oracle/sqsynth.h)
  synth_runs.json               the reference's hsum() on the synthetic integrands, -ffp-contract=off build,
                                SINCQED_SYM=0 and SINCQED_KEEPBT=1 (one boundary table, the exact grow):
                                syn_d5 at h = 1.0 (N = 61) and h = 0.7 (N = 87), syn_d8 at h = 1.0 (N = 61)
  scale.json                    `sincqed scale SEL kappa seed` of the -ffp-contract=off build, one thread
                                (directions in order): the stdout lines per graph, kappa = 24 for all2, g3_00,
                                g3_07, g3_lbl, v3_00 and kappa = 3 (slow directions listed) for g2_00, g3_07
  predict.json                  the last-level predictor, SINCQED_PREDICT=1 (driver/sum.c:64-69, 379-422), the
                                -ffp-contract=off build with SINCQED_KEEPBT=1: runs unfolded (SINCQED_SYM=0) and
                                one folded, with the log's count of final-level points left out
  fold.json                     the symmetry fold (driver/sum.c:21-46, 464-592), -ffp-contract=off build:
                                the group line the reference prints for every graph of g2 g3 v3 v4 w4
                                (`run 2.0 13 1e-4 GRAPH`, SINCQED_SYM unset = auto; the search's nodes only
                                need K >= 6), and folded sums (SINCQED_SYM unset, SINCQED_KEEPBT=1) with
                                top = 2 so that kept orbits go on to a second refinement level
  all2_mixed_h.json             all2 at h = 1.0, 0.9, 0.8, 0.7 (N = 2 ceil(48/h) + 1, eps = 1e-12), the
                                -ffp-contract=off build with SINCQED_SYM=0 and SINCQED_KEEPBT=1: the two-loop
                                part of the mixed batch
  vp4_sample.json               four-loop lepton-loop kernels (kernels/v4, kernels/w4), a sample of D = 6..9 with
                                the sets I(a), I(b), I(c) of docs/LEPTON_LOOPS.md, at h = 1.0 (N = 97) and 0.9
                                (N = 107), eps = 1e-12, -ffp-contract=off build, SINCQED_SYM=0, SINCQED_KEEPBT=1
                                (hours on 8 cores; resumable, see vp4())
  all3_h0.7_N139_eps1e-12.json  `sincqed run 0.7 139 1e-12 GRAPH` for the 41 three-loop integrals (the headline
                                workload), -ffp-contract=off build, SINCQED_SYM=0, SINCQED_KEEPBT=1, default
                                top = 2: every results column, the fallback count and the host wall time
                                (an hour or more on 8 cores; resumable, see all3())

    python tests/golden/make_golden.py [all2 boxsum pointwise synth fold scale predict all3 mixed2 vp4]
    (default: all but all3, mixed2 and vp4)
"""
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))
import refpy  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def with_log(rows, out):
    """add the log line's fallback count and kept top-level cells (driver/main.c:58-65) to the rows"""
    for r in rows:
        m = re.search(r'^%s .* evals (\d+) quad (\d+) kept (\d+)' % re.escape(r['name']), out, re.M)
        r['quad'], r['kept_top'] = int(m.group(2)), int(m.group(3))
    return rows


def all2():
    d = {'command': 'run 1.0 97 1e-12 all2'}
    rows, out = refpy.run(refpy.SINCQED, 1.0, 97, 1e-12, ['all2'])
    d['reference'] = with_log(rows, out)
    rows, out = refpy.run(refpy.SINCQED_EXACT, 1.0, 97, 1e-12, ['all2'], env={'SINCQED_SYM': '0'})
    d['reference_exact_unfolded'] = with_log(rows, out)
    for r in d['reference'] + d['reference_exact_unfolded']:
        r.pop('time_s', None)
    with open(os.path.join(OUT, 'all2_h1.0_N97_eps1e-12.json'), 'w') as f:
        json.dump(d, f, indent=1)


def boxsum():
    out = subprocess.run([refpy.BOXSUM, '1.0', '6'], stdout=subprocess.PIPE, text=True, check=True).stdout
    d = {}
    for line in out.splitlines():
        m = re.match(r'(\w+) term0 (\S+) term1 (\S+)', line)
        if m:
            d.setdefault(m.group(1), {}).update(term0=float(m.group(2)), term1=float(m.group(3)))
        m = re.match(r'(\w+) box h=1.0 K=6 (\S+)', line)
        if m:
            d.setdefault(m.group(1), {}).update(box_h1_K6=float(m.group(2)))
    d['_source'] = 'mathematica/check/boxsum_gl.c run as `boxsum_gl 1.0 6` (QREAL_DOUBLE)'
    with open(os.path.join(OUT, 'boxsum_gl.json'), 'w') as f:
        json.dump(d, f, indent=1)


def pointwise(cls, prefixes, npts=400, path=None):
    rng = np.random.default_rng(12345)
    arrays = {}
    for name in refpy.names(path):
        if not name.startswith(prefixes):
            continue
        D = refpy.info(name, path)['D']
        sf = np.exp(rng.uniform(-3, 3, size=(npts, D)))
        f1, a1 = refpy.fd(name, sf, 1, path)
        f0, a0 = refpy.fd(name, sf, 0, path)
        q, qa = refpy.fq(name, sf, path)
        arrays[name + '.sf'] = sf
        arrays[name + '.fd1'] = np.stack([f1, a1], 1)
        arrays[name + '.fd0'] = np.stack([f0, a0], 1)
        arrays[name + '.fq'] = np.concatenate([q, qa], 1)
    np.savez_compressed(os.path.join(OUT, 'pointwise_%s.npz' % cls), **arrays)


SYNTH_RUNS = [('syn_d5', 1.0, 61), ('syn_d5', 0.7, 87), ('syn_d8', 1.0, 61)]


def synth():
    pointwise('synth', ('syn_',), 64)
    d = {'env': {'SINCQED_SYM': '0', 'SINCQED_KEEPBT': '1'}, 'eps': 1e-12, 'runs': []}
    for name, h, N in SYNTH_RUNS:
        rows, out = refpy.run(refpy.SINCQED_EXACT, h, N, 1e-12, [name], env=d['env'])
        r = with_log(rows, out)[0]
        r.pop('time_s', None)
        r.update(h=h, N=N)
        d['runs'].append(r)
    with open(os.path.join(OUT, 'synth_runs.json'), 'w') as f:
        json.dump(d, f, indent=1)


FOLD_GROUP_RUN = (2.0, 13, 1e-4)
FOLD_RUNS = [('v2_00', 1.0, 97, 2), ('g3_07', 1.0, 97, 2), ('g3_25', 1.0, 97, 2), ('g3_08', 1.0, 97, 2),
             ('v3_00', 1.0, 97, 2), ('v3_03', 1.0, 97, 2), ('v3_p4Vm', 1.0, 97, 2), ('g3_lbl', 1.5, 65, 2)]
_SYMLINE = re.compile(r'^# (\S+): symmetry fold sigma=(.*) \(group of order (\d+)\), '
                      r'max \|f\(k\)-f\(k sigma\)\|/sum\|terms\| over 200 nodes (\S+)$', re.M)


SCALE_RUNS = [('all2', 24, 1), ('g3_00', 24, 1), ('g3_07', 24, 1), ('g3_lbl', 24, 1), ('v3_00', 24, 1),
              ('g2_00', 3, 2), ('g3_07', 3, 5)]      # kappa = 3: slow directions (ratio ~ e^-1) to list


def scale():
    d = {'E': 1, 'runs': []}
    env = dict(os.environ, OMP_NUM_THREADS='1', SINCQED_LOG='-', SINCQED_RESULTS='-')
    env.pop('SCALE_E', None)
    for sel, kappa, seed in SCALE_RUNS:
        out = subprocess.run([refpy.SINCQED_EXACT, 'scale', sel, str(kappa), str(seed)], env=env,
                             stdout=subprocess.PIPE, text=True, check=True, timeout=3600).stdout
        run, cur = {'sel': sel, 'kappa': kappa, 'seed': seed, 'lines': {}}, []
        for line in out.splitlines():
            if line.startswith('  slow direction'):
                cur.append(line)
            elif 'scale test kappa=' in line or '(no scale test' in line:
                run['lines'][line.split()[0]] = cur + [line]
                cur = []
        d['runs'].append(run)
    with open(os.path.join(OUT, 'scale.json'), 'w') as f:
        json.dump(d, f, indent=1)


PREDICT_RUNS = [('g2_01', 0.7, 139, '0'), ('g2_03', 0.7, 139, '0'), ('v2_00', 0.7, 139, '0'), ('g3_07', 0.7, 139, '0'),
                ('v3_01', 0.7, 139, '0'), ('g3_25', 1.0, 97, '0'), ('g3_07', 0.7, 139, None)]


def predict():
    d = {'alpha': 1.0, 'eps': 1e-12, 'runs': []}
    for name, h, N, sym in PREDICT_RUNS:
        env = {'SINCQED_PREDICT': '1', 'SINCQED_KEEPBT': '1'}
        if sym is not None:
            env['SINCQED_SYM'] = sym
        rows, out = refpy.run(refpy.SINCQED_EXACT, h, N, 1e-12, [name], top=2, env=env)
        r = with_log(rows, out)[0]
        r.pop('time_s', None)
        m = re.search(r'^# %s predictor alpha \S+: skipped (\d+) final-level points' % re.escape(name), out, re.M)
        r.update(h=h, N=N, top=2, fold=sym is None, pskip=int(m.group(1)))
        d['runs'].append(r)
    with open(os.path.join(OUT, 'predict.json'), 'w') as f:
        json.dump(d, f, indent=1)


def fold():
    h, N, eps = FOLD_GROUP_RUN
    d = {'group_run': {'h': h, 'N': N, 'eps': eps}, 'groups': {}, 'runs': [], 'env': {'SINCQED_KEEPBT': '1'}}
    names = [n for n in refpy.names() if n.split('_')[0] in ('g2', 'v2', 'g3', 'v3', 'w3', 'v4', 'w4')]
    for i in range(0, len(names), 16):
        _, out = refpy.run(refpy.SINCQED_EXACT, h, N, eps, names[i:i + 16])
        for m in _SYMLINE.finditer(out):
            d['groups'][m.group(1)] = {'desc': m.group(2), 'order': int(m.group(3)), 'worst': m.group(4)}
    d['searched'] = names
    for name, h, N, top in FOLD_RUNS:
        rows, out = refpy.run(refpy.SINCQED_EXACT, h, N, 1e-12, [name], top=top, env=d['env'])
        r = with_log(rows, out)[0]
        r.pop('time_s', None)
        d['runs'].append(r)
    with open(os.path.join(OUT, 'fold.json'), 'w') as f:
        json.dump(d, f, indent=1)


MIX_H = (1.0, 0.9, 0.8, 0.7)


def mixed2():
    """all2 at each h of the mixed batch (N = 2 ceil(48/h) + 1, eps = 1e-12, default top): the
    -ffp-contract=off build, SINCQED_SYM=0, SINCQED_KEEPBT=1"""
    import math
    d = {'env': {'SINCQED_SYM': '0', 'SINCQED_KEEPBT': '1'}, 'eps': 1e-12, 'runs': []}
    for h in MIX_H:
        N = 2*math.ceil(48/h - 1e-9) + 1
        rows, out = refpy.run(refpy.SINCQED_EXACT, h, N, 1e-12, ['all2'], env=d['env'])
        for r in with_log(rows, out):
            r.pop('time_s', None)
            r.update(h=h, N=N)
            d['runs'].append(r)
    with open(os.path.join(OUT, 'all2_mixed_h.json'), 'w') as f:
        json.dump(d, f, indent=1)


VP4_H = ((1.0, 97), (0.9, 107))
# a dimension-stratified sample of kernels/v4 and kernels/w4 (D = 6, 7, 8, 9; the cheapest D = 9 graph at
# h = 2.0), the lepton-loop sets I(a), I(b), I(c) of docs/LEPTON_LOOPS.md:5-17, and two large integrands with
# many cells near the fallback at h = 1.0 (v4_65, w4_04Sm: 38 % and 21 % of their evaluations with the |.|
# sums), whose contracted level kernel takes each batch in two sweeps
VP4_SAMPLE = {1.0: ['w4_00Sc', 'v4_00', 'w4_00Sm', 'w4_00Vm', 'w4_0iSc', 'w4_0iSm', 'w4_0iVm', 'v4_02', 'v4_14',
                    'v4_65', 'w4_04Sm'],
              0.9: ['w4_00Sc', 'v4_00', 'w4_00Sm', 'w4_0iSc', 'w4_0iSm', 'v4_02']}     # D = 6..8 at h = 0.9
VP4_FILE = os.path.join(OUT, 'vp4_sample.json')


def vp4():
    """`sincqed run h N 1e-12 GRAPH` for VP4_SAMPLE at h = 1.0 (N = 97; D = 6..9) and 0.9 (N = 107; D = 6..8, the
    D = 9 graph alone being hours of CPU time there), default top = 1:
    the -ffp-contract=off build, SINCQED_SYM=0, SINCQED_KEEPBT=1, one graph per process (checkpoints every
    15 min; the file is rewritten after every run and runs already in it are kept)"""
    d = {'env': {'SINCQED_SYM': '0', 'SINCQED_KEEPBT': '1'}, 'eps': 1e-12, 'threads': os.cpu_count(),
         'cpu': _cpu_model(), 'runs': []}
    if os.path.exists(VP4_FILE):
        with open(VP4_FILE) as f:
            d['runs'] = json.load(f)['runs']
    done = {(r['name'], r['h']) for r in d['runs']}
    ck = os.path.join(tempfile.gettempdir(), 'sincfeyn_golden_ckpt')
    os.makedirs(ck, exist_ok=True)
    for h, N in VP4_H:
        for g in VP4_SAMPLE[h]:
            if (g, h) in done:
                continue
            env = dict(d['env'], SINCQED_CKPT='900', SINCQED_CKPT_DIR=ck)
            rows, out = refpy.run(refpy.SINCQED_EXACT, h, N, 1e-12, [g], env=env, timeout=12*3600)
            r = with_log(rows, out)[0]
            r.update(h=h, N=N)
            d['runs'].append(r)
            with open(VP4_FILE, 'w') as f:
                json.dump(d, f, indent=1)
            print('%s h=%g %+.16e evals %d %.1f s' % (g, h, r['value'], r['evals'], r['time_s']), flush=True)


ALL3 = (0.7, 139, 1e-12)
ALL3_FILE = os.path.join(OUT, 'all3_h0.7_N139_eps1e-12.json')


def all3():
    """`sincqed run 0.7 139 1e-12 GRAPH` for each of the 41 integrals of all3 (default top = 2, K = 72): the
    -ffp-contract=off build, SINCQED_SYM=0 (the unfolded point set) and SINCQED_KEEPBT=1 (one boundary
    table: the exact grow), one graph per process with checkpoints every 15 min so that a stopped run
    resumes.  The file is rewritten after every graph, and graphs already in it are not run again.  Each
    row keeps the reference's wall time on this host (time_s) with the host's thread count and CPU."""
    h, N, eps = ALL3
    d = {'command': 'run 0.7 139 1e-12 GRAPH', 'h': h, 'N': N, 'eps': eps, 'top': 2,
         'env': {'SINCQED_SYM': '0', 'SINCQED_KEEPBT': '1'}, 'binary': 'sincqed-exact (-ffp-contract=off)',
         'threads': os.cpu_count(), 'cpu': _cpu_model(), 'rows': []}
    if os.path.exists(ALL3_FILE):
        with open(ALL3_FILE) as f:
            d['rows'] = json.load(f)['rows']
    done = {r['name'] for r in d['rows']}
    ck = os.path.join(tempfile.gettempdir(), 'sincfeyn_golden_ckpt')
    os.makedirs(ck, exist_ok=True)
    for g in _set_members('all3'):
        if g in done:
            continue
        env = dict(d['env'], SINCQED_CKPT='900', SINCQED_CKPT_DIR=ck)
        rows, out = refpy.run(refpy.SINCQED_EXACT, h, N, eps, [g], env=env, timeout=6*3600)
        r = with_log(rows, out)[0]
        d['rows'].append(r)
        with open(ALL3_FILE, 'w') as f:
            json.dump(d, f, indent=1)
        print('%s %+.16e evals %d %.1f s' % (g, r['value'], r['evals'], r['time_s']), flush=True)
    d['set_sum'] = sum(r['value'] for r in d['rows'])          # the value column includes the mirror weight
    d['reference_time_s'] = sum(r['time_s'] for r in d['rows'])
    with open(ALL3_FILE, 'w') as f:
        json.dump(d, f, indent=1)


def _set_members(sel):
    """the integrals of a loop-order group in the reference's registry order: its `list` output filtered
    by the selector rule of driver/graphs.c:19-21 (allL: L = L, all3 without the w3_ checks)"""
    assert sel in ('all2', 'all3')
    env = dict(os.environ, SINCQED_LOG='-', SINCQED_RESULTS='-')
    out = subprocess.run([refpy.SINCQED_EXACT, 'list'], env=env, stdout=subprocess.PIPE, text=True,
                         check=True).stdout
    L = 'L=' + sel[-1]
    return [t[0] for t in (l.split() for l in out.splitlines() if l.startswith('  '))
            if len(t) > 1 and t[1] == L and not t[0].startswith('w3_')]


def _cpu_model():
    try:
        with open('/proc/cpuinfo') as f:
            return next(l.split(':', 1)[1].strip() for l in f if l.startswith('model name'))
    except (OSError, StopIteration):
        return None


if __name__ == '__main__':
    parts = sys.argv[1:] or ['all2', 'boxsum', 'pointwise', 'synth', 'fold', 'scale', 'predict']
    if 'all3' in parts:
        all3()
    if 'mixed2' in parts:
        mixed2()
    if 'vp4' in parts:
        vp4()
    if 'all2' in parts:
        all2()
    if 'boxsum' in parts:
        boxsum()
    if 'pointwise' in parts:
        pointwise('g2', ('g2_', 'v2_'))
        pointwise('v3', ('v3_', 'w3_'))
        pointwise('g3', ('g3_',), 128)
        pointwise('v4', ('v4_',), 32)
        pointwise('w4', ('w4_',), 32)
        pointwise('pi6', ('w4_p6',), 32, refpy.LIBSQREF_PI6)
    if 'synth' in parts:
        synth()
    if 'fold' in parts:
        fold()
    if 'scale' in parts:
        scale()
    if 'predict' in parts:
        predict()
