#!/usr/bin/env python3
"""Benchmark of the evaluator on its headline workload: the three-loop set (all3: 41 integrals, 72
diagrams) at h = 0.7, N = 139 (K rounded up to 72, top = 2), eps = 1e-12, FP64 with the double-double
fallback on the device.  Metric: integrand points per second and time-to-sum.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is the whole set: its 41 integrals as one concurrent batch through the public C ABI
(sqb_hsum_batch: host parameters in, host results out; each integral's top-level grow and dilation, then
every refinement level on the device; the worker count from the batch tuner, run once before the warm-up).
W warm-up steps, then K timed steps; the step's device time is the set's time-to-sum.  The same integrals
then run one at a time, each kernel timed alone, for the level-pass throughput and the FP64 roofline.
With N ranks (torchrun) the integrals are dealt round-robin to the ranks (strong scaling, no collective on
the data path); the time is the maximum over ranks.

JSON line (rank 0):
  value      points/s of the device-resident refinement levels: evaluated children / device time of the
             level passes (cell lists already in HBM when each pass starts; CUDA events on the library's
             stream), one integral at a time over the whole set
  e2e        points/s of a step: all evaluated points of the set / device time of the batch, every
             host<->device copy inside; ms_per_step and time_to_sum_s are that device time (mean of the K
             steps); one_at_a_time the same integrals through sqb_hsum one after another
  roofline   the FP64 evaluation kernels (sqb_k_f64<graph>): algorithmic flops per point (+ - * / of the
             kernel's double path, counted by the code generator; skipped |.| sums counted as skipped) over
             their event-timed launches, against this device's FP64 FMA rate measured by a probe kernel
  cpu_baseline  the reference's own OpenMP CPU build (oracle/_ref/sincqed) on this host's cores, on a
             bounded sample of the same workload (integrals of D = 5, 6, 6, 7), with its rate per D
  precision  the error of the results: a sample's FP64 + dd values against all-double-double GPU runs of
             the same integrals (two D = 7 graphs; --alldd-full: the whole set) with both forms' times, the
             set sum against the analytic A1^(6), and every integral against the reference CPU run of the
             workload (the committed fixture tests/golden/all3_h0.7_N139_eps1e-12.json)
  fold       the same batch with the symmetry fold (sym='auto': each integrand's group of axis
             permutations, as the reference CPU build finds it): time-to-sum, evaluated points, the largest
             relative difference from the unfolded values, the group orders
`--impl reference` times the reference CPU build on the same metric (rank 0 only), one integral of the CPU
sample per step.

Other measurements (one GPU, each prints its own JSON lines; not the headline):
  --workload mixed   all2 + all3 at h = 1.0, 0.9, 0.8, 0.7 (184 integrals): one at a time against the
                     tuned concurrent batch (sqb_hsum_batch), results compared
  --workload synth   the synthetic Sinc-sum microbenchmark (d = 5, 8, 11; h = 1.0, 0.7) and its
                     precision table (FP64 only, FP64 + dd, all-dd, the reference's hsum)
  --workload vp4     the four-loop lepton-loop set (kernels/v4, kernels/w4) at h = 1.0 and 0.9, with the
                     exactly known set values (--fold: with the symmetry fold; --predict alpha: with the
                     last-level predictor)
  --workload single  one integral (--graph) warm, then timed once: a small command for profilers
  --workload points  one launch of a graph's evaluation kernel on --npoints seeded nodes (--prec)
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

H, N_PTS, EPS = 0.7, 139, 1e-12
SET = 'all3'
# the CPU sample: three-loop integrals of D = 5, 6, 6 and 7 at the workload's (h, N, eps); by points it is
# mostly D = 7, as the set is (12 of its 41 integrals, about nine tenths of its points)
CPU_SAMPLE = ['g3_07', 'v3_01', 'g3_01', 'g3_00']
# the precision sample: FP64 + dd against all-dd, two D = 7 graphs among them
ALLDD_SAMPLE = ['v3_01', 'g3_07', 'g3_01', 'g3_00', 'g3_12']
PROFILE_TRAFFIC = os.path.join(ROOT, 'profiles', 'fp64_kernel_traffic.json')
BATCH_CANDIDATES = (2, 4, 8)     # worker streams tried by the batch tuner


def env_rank():
    return int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1)), int(os.environ.get('LOCAL_RANK', 0))


def assign(integrals, rank, world):
    """Round-robin deal of the set's integrals to the ranks (each integral exactly once)."""
    return [x for i, x in enumerate(integrals) if i % world == rank]


def reduce_max_sum(vals_max, vals_sum, world):
    """Max over ranks of vals_max and sum of vals_sum (torch.distributed all_reduce; identity at world 1)."""
    if world == 1:
        return list(vals_max), list(vals_sum)
    import torch
    import torch.distributed as dist
    dev = 'cuda' if dist.get_backend() == 'nccl' else 'cpu'
    a = torch.tensor(vals_max, dtype=torch.float64, device=dev)
    b = torch.tensor(vals_sum, dtype=torch.float64, device=dev)
    dist.all_reduce(a, op=dist.ReduceOp.MAX)
    dist.all_reduce(b, op=dist.ReduceOp.SUM)
    return a.cpu().tolist(), b.cpu().tolist()


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, power, throttle reasons)."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile('w+', suffix='.csv', delete=False)
        try:
            self.p = subprocess.Popen(['nvidia-smi', '-i', str(index), '--query-gpu=' + self.Q, '--format=csv,noheader,nounits',
                                       '-lms', '200'], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [l.split(', ') for l in self.f.read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace('.', '').isdigit()]
        if not sm:
            return None
        reasons = set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.strip() == 'Active':
                    reasons.add(n)
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': float(rows[0][2]), 'samples': len(sm),
                'power_w_max': max(float(r[3]) for r in rows if len(r) > 3 and r[3].replace('.', '').isdigit()),
                'reasons': sorted(reasons)}


def cpu_reference(graphs, threads):
    """The reference CPU build (oracle/_ref/sincqed, symmetry fold on as shipped) on these integrals, one
    process each; returns (evals, seconds, per-graph rows)."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import refpy
    if not refpy.available():
        raise RuntimeError('oracle/_ref/sincqed is not built')
    ev, sec, rows = 0, 0.0, []
    for g in graphs:
        t0 = time.perf_counter()
        r, _ = refpy.run(refpy.SINCQED, H, N_PTS, EPS, [g], threads=threads)
        dt = time.perf_counter() - t0
        ev += r[0]['evals']
        sec += dt
        rows.append({'graph': g, 'evals': r[0]['evals'], 'seconds': round(dt, 3), 'value': r[0]['value']})
    return ev, sec, rows


def run_reference(args, rank):
    """--impl reference: the reference's CPU implementation of the path (oracle/_ref/sincqed, its OpenMP build,
    all host threads), same metric.  A step of ours is the whole set (minutes of CPU time per integral of
    D = 7, an hour or more for the set); a step here is one integral of the CPU sample in turn, which keeps
    the run to minutes: the warm-up steps run its cheapest integral."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    seq = [CPU_SAMPLE[i % len(CPU_SAMPLE)] for i in range(args.steps)]
    cpu_reference([CPU_SAMPLE[0]]*args.warmup, threads)
    ev, sec, rows = cpu_reference(seq, threads)
    v = ev/sec
    line = {'impl': 'reference', 'metric': 'integrand points/s (time-to-sum) of the three-loop set at h=0.7',
            'value': v, 'unit': 'points/s', 'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': 1e3*sec/args.steps, 'higher_is_better': True, 'scaling': 'strong', 'vs_baseline': None,
            'dtype': 'f64+dd', 'data': 'the reference kernels (kernels/g3, kernels/v3), no external data',
            'config': {'workload': 'all3 at h=%g N=%d eps=%g: a sample, one integral per step cycling over %s (D = 5, 6, 6, 7)'
                                   % (H, N_PTS, EPS, ','.join(CPU_SAMPLE)),
                       'cpu': 'oracle/_ref/sincqed (reference CPU build, OpenMP)'},
            'cpu_baseline': {'value': v, 'unit': 'points/s', 'cores': threads, 'kind': 'reference',
                             'sample': '%d integrals cycling over %s' % (args.steps, ','.join(CPU_SAMPLE)),
                             'rows': rows},
            'e2e': {'value': v, 'unit': 'points/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


MIX_H = (1.0, 0.9, 0.8, 0.7)
MIX_SETS = ('all2', 'all3')


def mixed_jobs(sq):
    """The mixed batch: every two- and three-loop integral at h = 1.0, 0.9, 0.8, 0.7, N = 2 ceil(48/h) + 1,
    eps = 1e-12 (184 integrals of D = 3..7); cost estimate (2/h)^D for the largest-first order."""
    info = {g['name']: g for g in sq.graphs()}
    jobs = []
    for h in MIX_H:
        N = 2*math.ceil(48/h - 1e-9) + 1
        for g in sq.select(list(MIX_SETS)):
            jobs.append((g, h, N, EPS, -1, (2.0/h)**info[g]['D']))
    return jobs


def run_mixed(args, sq, L):
    """--workload mixed: the batch one integral at a time (one worker), as a concurrent batch (the tuned
    worker count, each integral alone) and grouped (each graph's four h as one group, sqb_hsum_group: its
    refinement levels in shared launches over the four integrals, tiles from a device queue); device time
    of each whole batch, points/s, and the runs' values, which must be identical (each integral's
    arithmetic does not depend on the schedule).  The tuner runs a calibration sample (every 8th graph's
    four integrals) twice per candidate (workers, grouped or not) and picks the fastest."""
    import torch
    jobs = mixed_jobs(sq)
    for g in sorted({j[0] for j in jobs}):
        sq.preload(g)
    graphs = sorted({j[0] for j in jobs})
    sample = [j for j in jobs if j[0] in graphs[::8]]
    # warm-up and tuning: the calibration sample twice per candidate
    rates = {}
    best, best_rate = None, -1.0
    for grp in (0, 1):
        b, r = sq.batch_tune(sample, (1, 2, 4, 8, 12, 16), group=grp)
        for w, v in r.items():
            rates['%s%d' % ('group_' if grp else '', w)] = v
            if v > best_rate:
                best, best_rate = (w, grp), v
    torch.cuda.synchronize()
    clocks = Clocks(0)
    seq, ms_seq = sq.hsum_batch(jobs, workers=1)
    bat, ms_bat = sq.hsum_batch(jobs, workers=best[0])
    grp, ms_grp = sq.hsum_batch(jobs, workers=best[0], group=1)
    tuned, ms_tuned = (grp, ms_grp) if best[1] else (bat, ms_bat)
    clk = clocks.stop()
    nev = sum(r['nev'] for r in seq)

    def ident(x, y):
        return all(all(a == b or (a != a and b != b) for a, b in zip(p['S'], q['S'])) and p['nev'] == q['nev']
                   for p, q in zip(x, y))
    info = {g['name']: g for g in sq.graphs()}
    per_h = {}
    for j, r in zip(jobs, tuned):
        per_h.setdefault(j[1], [0.0, 0])
        per_h[j[1]][0] += r['S'][0]*info[j[0]]['weight']
        per_h[j[1]][1] += r['nev']
    line = {'workload': 'mixed', 'metric': 'integrand points/s of the mixed batch (all2+all3 x h=1.0,0.9,0.8,0.7)',
            'value': nev/(ms_tuned*1e-3), 'unit': 'points/s', 'n_gpus': 1, 'higher_is_better': True,
            'integrals': len(jobs), 'points': nev,
            'one_at_a_time': {'workers': 1, 'device_s': ms_seq*1e-3, 'points_s': nev/(ms_seq*1e-3)},
            'concurrent': {'workers': best[0], 'device_s': ms_bat*1e-3, 'points_s': nev/(ms_bat*1e-3),
                           'speedup_vs_one_at_a_time': ms_seq/ms_bat},
            'grouped': {'workers': best[0], 'device_s': ms_grp*1e-3, 'points_s': nev/(ms_grp*1e-3),
                        'speedup_vs_one_at_a_time': ms_seq/ms_grp,
                        'note': 'each graph\'s four h as one sqb_hsum_group: shared level launches, tiles from a device queue'},
            'identical_results': ident(seq, bat) and ident(seq, grp),
            'tuner': {'sample': '%d integrals (every 8th graph, its four h)' % len(sample), 'points_s': rates,
                      'chosen': {'workers': best[0], 'grouped': bool(best[1])}},
            'sums_by_h': {str(h): {'sum': v[0], 'points': v[1]} for h, v in sorted(per_h.items())},
            'clocks': clk, 'dtype': 'f64+dd', 'data': 'the reference kernels (kernels/g2, g3, v3)',
            'config': {'workload': 'all2+all3 at h in %s, N=2ceil(48/h)+1, eps=%g, default top' % (list(MIX_H), EPS)}}
    print(json.dumps(line), flush=True)


# the lepton-loop sets with exactly known values (docs/LEPTON_LOOPS.md:5-17; Laporta, Table 2)
VP4_SETS = [('I(a) Pi2^3', lambda n: n == 'v4_00', 0.000876865858890),
            ('I(b) Pi2+Pi4', lambda n: n.startswith('w4_00'), 0.015325282902013),
            ('I(c) Pi4 with Pi2 inside', lambda n: n.startswith('w4_0i'), 0.011130913987517),
            ('II(a) Pi4 in 2-loop vertices', lambda n: n[:5] in ('w4_01', 'w4_02', 'w4_03', 'w4_04', 'w4_05',
                                                               'w4_06', 'w4_07'), -0.420482262508962),
            ('II(b)+II(c)+III Pi2 insertions', lambda n: n.startswith('v4_') and n != 'v4_00', -0.027675 - 0.073452 + 1.417687)]
VP4_H = ((1.0, 97), (0.9, 107))


def run_vp4(args, sq, L):
    """--workload vp4: the four-loop lepton-loop kernels (kernels/v4, kernels/w4: 118 integrals, D = 6..9)
    at h = 1.0 (N = 97) and 0.9 (N = 107), eps = 1e-12, as one concurrent batch per h; the device time,
    points/s, and each lepton-loop set's sum against its exact value."""
    import torch
    names = [n for n in sq.select(['vp4']) if not n.startswith('w4_p6')]     # kernels/v4 and kernels/w4 (not pi6)
    info = {g['name']: g for g in sq.graphs()}
    for g in names:
        sq.preload(g)
    workers = args.workers or 6
    torch.cuda.synchronize()
    clocks = Clocks(0)
    out = []
    for h, N in VP4_H:
        if args.vp4_h and h not in args.vp4_h:
            continue
        jobs = [(g, h, N, EPS, -1, (2.0/h)**info[g]['D']) for g in names]
        kw = dict(({'sym': 'auto'} if args.fold else {}), **({'predict': args.predict} if args.predict > 0 else {}))
        res, ms = sq.hsum_batch(jobs, workers=workers, **kw)
        nev = sum(r['nev'] for r in res)
        val = {g: r['S'][0]*info[g]['weight'] for g, r in zip(names, res)}
        sets = []
        for label, pick, exact in VP4_SETS:
            mem = [g for g in names if pick(g)]
            s = sum(val[g] for g in mem)
            sets.append({'set': label, 'graphs': len(mem), 'sum': s, 'exact': exact, 'diff': s - exact})
        slow = sorted(zip(names, res), key=lambda x: -x[1]['t'])[:5]
        row = {'h': h, 'N': N, 'integrals': len(jobs), 'workers': workers, 'fold': bool(args.fold),
               'predict': args.predict, 'predicted_out': sum(r['pskip'] for r in res),
               'device_s': ms*1e-3, 'points': nev,
               'points_s': nev/(ms*1e-3), 'fallback': sum(r['nq'] for r in res), 'sets': sets,
               'slowest': [[g, round(r['t'], 2), r['nev']] for g, r in slow],
               'values': {g: val[g] for g in names}}
        out.append(row)
        print(json.dumps(row), flush=True)
    print(json.dumps({'workload': 'vp4', 'clocks': clocks.stop(), 'cases': len(out)}), flush=True)


def run_single(args, sq, L):
    """--workload single: one integral (--graph, at the headline's h, N, eps) once warm, then once timed; a
    small, fixed command for profilers.  --workload points: one launch of the graph's FP64 kernel
    (--prec 0 as written, 2 contracted) or double-double kernel (--prec 1) on --npoints seeded nodes."""
    import numpy as np
    g = args.graph
    sq.preload(g)
    if args.workload == 'points':
        D = {x['name']: x['D'] for x in sq.graphs()}[g]
        sf = np.exp(np.random.default_rng(1).uniform(-3, 3, size=(args.npoints, D)))
        f, _ = sq.eval_points(g, sf, args.prec, 1)
        print(json.dumps({'workload': 'points', 'graph': g, 'prec': args.prec, 'points': args.npoints,
                          'sum_abs_f': float(np.nansum(np.abs(f if args.prec != 1 else f[:, 0])))}), flush=True)
        return
    h = args.h or H
    N = args.N or (2*math.ceil(48/h - 1e-9) + 1 if args.h else N_PTS)
    kw = {'split': args.split}
    sq.hsum(g, h, N, EPS, **kw)
    L.sqb_timer_start()
    r = sq.hsum(g, h, N, EPS, **kw)
    ms = L.sqb_timer_stop()
    a1, a0 = sq.flops(g, 1), sq.flops(g, 0)
    fl = (r['nev'] - r['abskipped'])*a1 + r['abskipped']*a0
    print(json.dumps({'workload': 'single', 'graph': g, 'h': h, 'N': N, 'split': args.split, 'ms': ms,
                      'points': r['nev'], 'value': r['S'][0], 'f64_ms': r['f64_ms'], 'f64_launches': r['f64_launches'],
                      'f64_tflops': fl/(r['f64_ms']*1e-3)/1e12 if r['f64_ms'] else None,
                      'levels_ms': sum(r['lev_ms']), 'top_ms': 1e3*r['t_top']}), flush=True)


SYN_D = (5, 8, 11)
SYN_H = (1.0, 0.7)
GOLDEN_SYNTH = os.path.join(ROOT, 'tests', 'golden', 'synth_runs.json')
FLOPS_JSON = os.path.join(ROOT, 'sincfeyn_b200', 'lib', 'flops.json')


def run_synth(args, sq, L):
    """--workload synth: the synthetic Sinc-sum microbenchmark (d = 5, 8, 11; h = 1.0, 0.7; N =
    2 ceil(30/h) + 1; eps = 1e-12).  Per case: points/s and FP64 rate of the FP64+dd form, and the
    precision table: the value in FP64 only (no fallback: the fallback bound set to infinity), FP64+dd,
    all double-double (not d = 11 at h = 1.0), against the reference's hsum() on the host-double-double oracle build
    where a golden run exists (d = 5 both h, d = 8 at h = 1.0)."""
    import torch
    with open(FLOPS_JSON) as f:
        fl = json.load(f)
    gold = {}
    if os.path.exists(GOLDEN_SYNTH):
        with open(GOLDEN_SYNTH) as f:
            for r in json.load(f)['runs']:
                gold[(r['name'], r['h'])] = r['value']
    peak = sq.probe_fp64(True)
    for d in SYN_D:
        sq.preload('syn_d%d' % d)
    # warm-up: the smallest case in every form (device buffers, pinned staging)
    for kw in ({}, {'abserr0': 1e300}, {'alldd': 1}):
        sq.run(1.0, 61, EPS, ['syn_d5'], **kw)
    rows = []
    torch.cuda.synchronize()
    clocks = Clocks(0)
    for d in SYN_D:
        name = 'syn_d%d' % d
        for h in SYN_H:
            N = 2*math.ceil(30/h - 1e-9) + 1
            row = {'d': d, 'h': h, 'N': N}
            for form, kw in (('fp64dd', {}), ('fp64', {'abserr0': 1e300}), ('alldd', {'alldd': 1})):
                if form == 'alldd' and d > 8 and h > 0.8:      # d = 11 at h = 1.0: 4e11 points, minutes in dd
                    continue
                L.sqb_timer_start()
                r = sq.run(h, N, EPS, [name], **kw)[0]
                ms = L.sqb_timer_stop()
                raw = r['raw']
                row[form] = {'value': r['value'], 'evals': r['evals'], 'fallback': r['quad'], 'device_s': ms*1e-3,
                             'points_s': r['evals']/(ms*1e-3)}
                if form == 'fp64dd':
                    a1, a0, tr = fl[name]['ab1'], fl[name]['ab0'], fl[name].get('tr', 0)
                    fk = (r['evals'] - raw['abskipped'])*a1 + raw['abskipped']*a0
                    row['fp64_kernel'] = {'ms': raw['f64_ms'], 'flops_per_point': a1, 'exp_log_per_point': tr,
                                          'arith_tflops': fk/(raw['f64_ms']*1e-3)/1e12 if raw['f64_ms'] else None,
                                          'exp_log_per_s': r['evals']*tr/(raw['f64_ms']*1e-3) if raw['f64_ms'] else None,
                                          'dd_ms': raw['dd_ms']}
            ref = gold.get((name, h))
            base = ref if ref is not None else (row['alldd']['value'] if 'alldd' in row else None)
            row['reference_value'] = ref
            row['error_vs'] = 'reference hsum (host dd oracle)' if ref is not None else ('all-dd GPU run' if base else None)
            for form in ('fp64dd', 'fp64', 'alldd'):
                if form in row and base:
                    row[form]['rel_err'] = abs(row[form]['value'] - base)/abs(base)
            rows.append(row)
            print(json.dumps(row), flush=True)
    clk = clocks.stop()
    line = {'workload': 'synth', 'metric': 'synthetic Sinc-sum points/s, FP64+dd', 'unit': 'points/s',
            'peak_fp64_tflops': peak, 'clocks': clk, 'cases': len(rows),
            'config': {'workload': 'syn_d{5,8,11} at h in %s, N=2ceil(30/h)+1, eps=%g' % (list(SYN_H), EPS)}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3, help='timed steps, each the whole set as one batch')
    ap.add_argument('--warmup', type=int, default=3, help='untimed steps before them (at least 3)')
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline sample')
    ap.add_argument('--no-alldd', action='store_true', help='skip the all-double-double comparison')
    ap.add_argument('--alldd-full', action='store_true', help='all-double-double comparison on the whole set (~6 min)')
    ap.add_argument('--no-fold', action='store_true', help='skip the batch with the symmetry fold')
    ap.add_argument('--fold', action='store_true', help='--workload vp4: with the symmetry fold (sym=auto)')
    ap.add_argument('--predict', type=float, default=0.0, help='--workload vp4: the last-level predictor with this alpha')
    ap.add_argument('--workers', type=int, default=0, help='batch workers for --workload vp4 (default 6)')
    ap.add_argument('--vp4-h', type=float, action='append', help='--workload vp4: only these h (repeatable)')
    ap.add_argument('--graph', default='g3_00', help='--workload single/points: the graph')
    ap.add_argument('--prec', type=int, default=2, help='--workload points: 0 FP64 as written, 2 contracted, 1 dd')
    ap.add_argument('--npoints', type=int, default=1 << 22, help='--workload points: number of nodes')
    ap.add_argument('--split', type=int, default=0, help='--workload single: 1 = the FP64 pass of a graph with '
                    'node passes in passes (0: one kernel)')
    ap.add_argument('--h', type=float, default=0.0, help='--workload single: h (default 0.7)')
    ap.add_argument('--N', type=int, default=0, help='--workload single: N (default 2ceil(48/h)+1)')
    ap.add_argument('--workload', default='all3', choices=['all3', 'mixed', 'synth', 'vp4', 'single', 'points'],
                    help='all3: the headline line; mixed: the mixed batch, one-at-a-time vs concurrent; '
                         'synth: the synthetic microbenchmark and its precision table; vp4: the four-loop '
                         'lepton-loop set at h=1.0 and 0.9 (one GPU)')
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world, local = env_rank()
    if args.workload != 'all3':
        if rank == 0 and args.impl == 'ours':
            from sincfeyn_b200 import sq
            import ctypes as C
            L = sq.lib()
            L.sqb_timer_stop.restype = C.c_double
            sq.kernel_timing(True)
            {'mixed': run_mixed, 'synth': run_synth, 'vp4': run_vp4, 'single': run_single,
             'points': run_single}[args.workload](args, sq, L)
        return
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
    if args.impl == 'reference':
        run_reference(args, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    from sincfeyn_b200 import sq
    torch.cuda.set_device(local)
    names = sq.select([SET])
    D_OF = {x['name']: x['D'] for x in sq.graphs()}
    mine = assign(names, rank, world)
    L = sq.lib()
    import ctypes as C
    L.sqb_timer_stop.restype = C.c_double
    L.sqb_l2_flush.argtypes = [C.c_size_t]
    # the batch runs without per-kernel events (they synchronise the host once per level batch); the
    # one-at-a-time pass below turns them on for the roofline
    sq.kernel_timing(False)
    # the device code of every graph of the set is loaded before the timed region (CUDA loads a kernel
    # on its first launch otherwise); the one-time cost is reported as load_s
    t_load = time.perf_counter()
    for g in names:
        sq.preload(g)
    t_load = time.perf_counter() - t_load
    # cost estimate for the largest-first order: children per cell times flops per point
    jobs = [(g, H, N_PTS, EPS, -1, float(2**D_OF[g])*sq.flops(g, 1)) for g in mine]
    # the batch tuner (untimed): every 4th integral of this rank's share twice per candidate worker count;
    # the sample leaves out the costliest integral, which alone would set its time whatever the count
    top = max(j[5] for j in jobs)
    workers, tune_rates = sq.batch_tune([j for j in jobs if j[5] < top][::4], BATCH_CANDIDATES, device=local)
    # W warm-up steps: the whole share as one batch, untimed
    for _ in range(args.warmup):
        sq.hsum_batch(jobs, workers=workers, device=local)
    peak = sq.probe_fp64(True)
    flops = {g: (sq.flops(g, 1), sq.flops(g, 0)) for g in names}
    weight = {x['name']: x['weight'] for x in sq.graphs()}
    h0 = (C.c_ulonglong(), C.c_ulonglong())
    L.sqb_copy_bytes(C.byref(h0[0]), C.byref(h0[1]))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    # the timed region: K steps, each this rank's whole share of the set as one concurrent batch through
    # the C ABI (sqb_hsum_batch: host parameters in, host results out), its device time by CUDA events;
    # L2 flushed before every step
    step_ms, walls, bres, same_steps = [], [], None, True
    for _ in range(args.steps):
        L.sqb_l2_flush(256 << 20)
        t_wall = time.perf_counter()
        res, ms = sq.hsum_batch(jobs, workers=workers, device=local)
        walls.append(time.perf_counter() - t_wall)
        step_ms.append(ms)
        if bres is None:
            bres = res
        else:
            same_steps = same_steps and all(_same(a['S'][0], b['S'][0]) and a['nev'] == b['nev'] for a, b in zip(res, bres))
    torch.cuda.synchronize()
    clk = clocks.stop()
    h1 = (C.c_ulonglong(), C.c_ulonglong())
    L.sqb_copy_bytes(C.byref(h1[0]), C.byref(h1[1]))
    nev = sum(r['nev'] for r in bres)
    launches = sum(r['launches'] for r in bres)*args.steps
    bvals = {j[0]: r['S'][0] for j, r in zip(jobs, bres)}
    # the same integrals one at a time, each kernel timed alone: the level-pass throughput and the FP64
    # roofline (a kernel that shares the device with other streams would read slow)
    sq.kernel_timing(True)
    one_ms, lev_ms, lev_ev, f64_ms, f64_n, fl, results, same = 0.0, 0.0, 0, 0.0, 0, 0.0, [], True
    for g in mine:
        L.sqb_l2_flush(256 << 20)
        L.sqb_timer_start()
        r = sq.hsum(g, H, N_PTS, EPS, device=local)
        ms = L.sqb_timer_stop()
        one_ms += ms
        lev_ms += sum(r['lev_ms'])
        lev_ev += sum(r['lev_evals'])
        f64_ms += r['f64_ms']
        f64_n += r['f64_launches']
        a1, a0 = flops[g]
        fl += (r['nev'] - r['abskipped'])*a1 + r['abskipped']*a0
        same = same and _same(r['S'][0], bvals[g])
        results.append([g, D_OF[g], r['S'][0]*weight[g], r['nev'], r['nq'], round(ms, 2), round(1e3*r['t_top'], 2),
                        round(sum(r['lev_ms']), 2)])
    sq.kernel_timing(False)
    # the same batch with the symmetry fold (sym='auto', the reference CPU build's default): the same kept
    # tree and values to rounding, fewer evaluations; reported beside the headline, not in it
    fold_ms, fnev, fdiff, groups, fold_err = 0.0, 0, 0.0, {}, None
    if not args.no_fold:
        try:
            L.sqb_l2_flush(256 << 20)
            fres, fold_ms = sq.hsum_batch(jobs, workers=workers, device=local, sym='auto')
            fnev = sum(r['nev'] for r in fres)
            for j, fr, br in zip(jobs, fres, bres):
                groups[j[0]] = fr['sym_order']
                if br['S'][0] == br['S'][0] and br['S'][0] != 0:
                    fdiff = max(fdiff, abs(fr['S'][0] - br['S'][0])/abs(br['S'][0]))
        except sq.SqbError as e:                   # reported beside the headline, which stands without it
            fold_ms, fold_err = 0.0, str(e)[:200]
    torch.cuda.synchronize()
    batch_ms = statistics.mean(step_ms)
    wall = statistics.mean(walls)
    mx, sm = reduce_max_sum([batch_ms, min(step_ms), max(step_ms), one_ms, wall, fold_ms, fdiff],
                            [lev_ms, lev_ev, nev, f64_ms, f64_n, fl, launches, h1[0].value - h0[0].value,
                             h1[1].value - h0[1].value, 0 if same and same_steps else 1, fnev], world)
    batch_ms, step_min, step_max, one_ms, wall, fold_ms, fdiff = mx
    lev_ms, lev_ev, nev, f64_ms, f64_n, fl, launches, h2d, d2h, ndiff, fnev = sm
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    achieved = fl/(f64_ms*1e-3)/1e12 if f64_ms > 0 else None
    traffic = None
    if os.path.exists(PROFILE_TRAFFIC):
        with open(PROFILE_TRAFFIC) as f:
            prof = json.load(f)
        if f64_n:
            traffic = prof['dram_bytes_per_point']*(lev_ev/max(1, f64_n))
    line = {
        'metric': 'integrand points/s (time-to-sum) of the three-loop set at h=0.7',
        'value': lev_ev/(lev_ms*1e-3) if lev_ms > 0 else None, 'unit': 'points/s',
        'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': batch_ms,
        'higher_is_better': True, 'scaling': 'strong', 'vs_baseline': None, 'dtype': 'f64+dd',
        'data': 'the reference kernels (kernels/g3, kernels/v3) as integrands; no external data',
        'precision_form': 'FP64 pass contracted (fused multiply-adds), double-double fallback and level sums',
        'config': {'workload': '%s (%d integrals) h=%g N=%d eps=%g top=2, FP64 + double-double fallback'
                               % (SET, len(names), H, N_PTS, EPS),
                   'step': 'the whole set (all %d integrals) as one concurrent batch through sqb_hsum_batch' % len(names),
                   'l2': 'flushed (256 MiB memset) before every step and before every one-at-a-time integral',
                   'kernels': 'device code of the set\'s kernels loaded before the timed region (load_s %.2f s, once per process)' % t_load,
                   'parallelism': 'integrals dealt round-robin over %d GPU(s); on each, one concurrent batch of %d worker streams'
                                  % (world, workers)},
        'time_to_sum_s': batch_ms*1e-3,
        'time_to_sum_steps_s': {'mean': batch_ms*1e-3, 'min': step_min*1e-3, 'max': step_max*1e-3},
        'e2e': {'value': nev/(batch_ms*1e-3), 'unit': 'points/s', 'h2d_bytes_per_step': int(h2d/args.steps),
                'd2h_bytes_per_step': int(d2h/args.steps), 'wall_s_per_step': wall,
                'note': 'the whole set per step through the C ABI (host parameters in, host results out)'},
        'batch': {'workers': workers, 'tuner_points_s': tune_rates, 'device_s': batch_ms*1e-3},
        'one_at_a_time': {'device_s': one_ms*1e-3, 'points_s': nev/(one_ms*1e-3),
                          'same_values_as_batch': ndiff == 0},
        'fold': None if args.no_fold else {'unavailable': fold_err} if fold_err or not fold_ms else {
            'time_to_sum_s': fold_ms*1e-3, 'points': int(fnev), 'speedup_vs_unfolded': batch_ms/fold_ms,
            'max_rel_diff_vs_unfolded': fdiff, 'group_orders': groups if world == 1 else None,
            'note': 'the same concurrent batch with the symmetry fold found automatically (sym=auto); '
                    'not the headline, whose point set is the unfolded tree'},
        'roofline': {'bound': 'fp64', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
                     'frac': achieved/peak if achieved else None, 'traffic': traffic,
                     'kernel': 'sqb_k_f64<graph> (FP64 evaluation), timed one integral at a time',
                     'peak_source': 'measured FP64 FMA rate (probe kernel, this device)',
                     'flops_per_launch': fl/max(1, f64_n), 'launches': int(f64_n)},
        'gpu_launches': int(launches),
        'load_s': t_load,
        'clocks': clk,
        'points': int(nev), 'level_points': int(lev_ev),
    }
    if world == 1:
        line['precision'] = precision_table(args, sq, L, names, {g: v*weight[g] for g, v in bvals.items()}, line)
    if world == 1 and not args.no_cpu:
        try:
            ev, sec, rows = cpu_reference(CPU_SAMPLE, os.cpu_count() or 1)
            per_d = {}
            for r in rows:
                x = per_d.setdefault(D_OF[r['graph']], [0, 0.0])
                x[0] += r['evals']
                x[1] += r['seconds']
            line['cpu_baseline'] = {'value': ev/sec, 'unit': 'points/s', 'cores': os.cpu_count() or 1, 'kind': 'reference',
                                    'sample': 'reference CPU build (OpenMP, all host threads) on %s (D = %s) at h=%g N=%d '
                                              'eps=%g, one integral at a time (%.1f s)'
                                              % (','.join(r['graph'] for r in rows),
                                                 ','.join(str(D_OF[r['graph']]) for r in rows), H, N_PTS, EPS, sec),
                                    'points_s_by_D': {str(d): v[0]/v[1] for d, v in sorted(per_d.items())},
                                    'rows': rows}
        except Exception as e:                      # the oracle binary is test infrastructure; report why
            line['cpu_baseline'] = {'value': None, 'unavailable': str(e)[:200]}
    line['per_integral'] = {'columns': ['graph', 'D', 'value', 'evals', 'fallback', 'ms', 'top_ms', 'levels_ms'],
                            'rows': results}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def _same(a, b):
    return a == b or (a != a and b != b)


A1_6 = 1.181241456587          # the analytic three-loop coefficient (docs/REPRODUCE.md:98-100)
GOLDEN_ALL3 = os.path.join(ROOT, 'tests', 'golden', 'all3_h0.7_N139_eps1e-12.json')


def precision_table(args, sq, L, names, values, line):
    """The error of the results: per integral of a sample (two D = 7 graphs among them; --alldd-full: the whole
    set) the FP64 + double-double value against the all-double-double GPU run of the same integral, with
    both forms' times; the set's sum against the analytic A1^(6); and, where the reference CPU run of the
    workload is among the committed fixtures, every integral against it."""
    out = {'form': line['precision_form']}
    sample = names if args.alldd_full else ALLDD_SAMPLE
    if not args.no_alldd:
        t, vals = {}, {}
        try:
            for form, kw in (('fp64dd', {}), ('fp64dd_as_written', {'fma': 0}), ('alldd', {'alldd': 1})):
                sq.hsum(sample[0], H, N_PTS, EPS, **kw)                 # warm: this form's kernels and buffers
                t[form] = 0.0
                for g in sample:
                    L.sqb_l2_flush(256 << 20)
                    L.sqb_timer_start()
                    r = sq.hsum(g, H, N_PTS, EPS, **kw)
                    t[form] += L.sqb_timer_stop()*1e-3
                    vals.setdefault(g, {})[form] = r['S'][0]
            rel = {g: abs(v['fp64dd'] - v['alldd'])/abs(v['alldd']) for g, v in vals.items()}
            rel_w = {g: abs(v['fp64dd_as_written'] - v['alldd'])/abs(v['alldd']) for g, v in vals.items()}
            out['vs_alldd'] = {'sample': 'all %d integrals' % len(sample) if args.alldd_full else sample,
                               'rel_err_fp64dd': rel, 'rel_err_fp64dd_as_written': rel_w,
                               'max_rel_err': max(rel.values()), 'fp64dd_s': t['fp64dd'],
                               'fp64dd_as_written_s': t['fp64dd_as_written'], 'alldd_s': t['alldd'],
                               'speedup': t['alldd']/t['fp64dd'],
                               'note': 'one integral at a time, each form warmed first, L2 flushed before each integral'}
            line['vs_alldd'] = {'sample': out['vs_alldd']['sample'], 'speedup': t['alldd']/t['fp64dd'],
                                'fp64dd_s': t['fp64dd'], 'alldd_s': t['alldd']}
        except sq.SqbError as e:                   # reported beside the headline, which stands without it
            out['vs_alldd'] = {'unavailable': str(e)[:200]}
    total = sum(values.values())
    out['set_sum'] = {'value': total, 'A1_6': A1_6, 'diff': total - A1_6,
                      'note': 'the sum of weight x value over the 41 integrals; the Sinc sum at h=0.7 with top=2 '
                              'differs from the analytic value by its discretisation and pruning errors'}
    if os.path.exists(GOLDEN_ALL3):
        with open(GOLDEN_ALL3) as f:
            gold = {r['name']: r for r in json.load(f)['rows']}
        common = [g for g in names if g in gold and g in values]
        if common:
            rel = {g: abs(values[g] - gold[g]['value'])/abs(gold[g]['value']) if gold[g]['value'] else abs(values[g])
                   for g in common}
            worst = max(rel, key=rel.get)
            ref_sum = sum(gold[g]['value'] for g in common)
            out['vs_reference_cpu'] = {'integrals': len(common), 'max_rel': rel[worst], 'worst': worst,
                                       'reference_set_sum': ref_sum if len(common) == len(names) else None,
                                       'source': 'tests/golden/all3_h0.7_N139_eps1e-12.json (sincqed-exact, SINCQED_SYM=0, '
                                                 'SINCQED_KEEPBT=1)'}
    return out


if __name__ == '__main__':
    main()
