"""Build of the evaluator: generated per-graph CUDA, the runtime, the C-ABI library and the CLI.

    python -m sincfeyn_b200.build --kernels DIR [--classes "g2 g3 v3"] [-j N]

Inputs are the generated sincFeyn kernel sources (kernels/<class>/<g>.c of the reference tree, the same
files its tools/gpugen.py reads): DIR is that kernels/ directory, given by --kernels or SQB_KERNELS.  Outputs, all in-tree and git-ignored:
  sincfeyn_b200/_build/gen/   kgen output (<g>.cuh), the per-graph translation units, the registry;
  sincfeyn_b200/_build/obj/   objects;
  sincfeyn_b200/lib/libsqb200.so   the C ABI (include/sincfeyn_b200.h), every graph's sm_100a kernels;
  sincfeyn_b200/bin/sincqed        the command line;
  sincfeyn_b200/lib/flops.json     algorithmic FP64 flops per point of every graph (SQ_AB = 1 and 0).
A step is redone only when one of its inputs is newer than its output.  Without a kernel tree (e.g. on
a host that only runs the prebuilt library) the build keeps what is there.
"""
import argparse
import concurrent.futures as cf
import json
import os
import re
import shutil
import subprocess
import sys

from .codegen import kgen

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, 'csrc')
BUILD = os.path.join(PKG, '_build')
GEN = os.path.join(BUILD, 'gen')
OBJ = os.path.join(BUILD, 'obj')
LIB = os.path.join(PKG, 'lib')
BIN = os.path.join(PKG, 'bin')
INC = os.path.join(ROOT, 'include')
DEFAULT_KERNELS = os.environ.get('SQB_KERNELS')     # the reference's kernels/ directory (no default)
DEFAULT_CLASSES = os.environ.get('SQB_CLASSES', 'g2 g3 v3 v4 w4 pi6')

NVCC = os.environ.get('NVCC', 'nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
# -fmad=false: the kernels' cancellations must round as written (no contraction), exactly as the
# reference CPU code compiled without contraction; the double-double code uses explicit intrinsics.
# -Xfatbin -compress-all: the device code of 200 graphs in two builds each is stored compressed in the
# library (about a third of the size; the driver expands a kernel's code when it loads it)
NVFLAGS = ARCH + ['-O3', '-lineinfo', '-fmad=false', '-std=c++17', '-Xcompiler', '-fPIC',
                  '-diag-suppress', '177,550', '-Xfatbin', '-compress-all', '-I' + CSRC, '-I' + INC]
# the second unit of every graph: its FP64 kernel with contraction (fused multiply-adds), for the fast form
NVFLAGS_FMA = [f if f != '-fmad=false' else '-fmad=true' for f in NVFLAGS]
CXX = 'g++'   # the system compiler (an environment CXX may lack libgomp.spec)
CXXFLAGS = ['-O2', '-fPIC', '-fopenmp', '-std=c++17', '-I' + CSRC, '-I' + INC, '-I/usr/local/cuda/include']

LIBSO = os.path.join(LIB, 'libsqb200.so')
CLI = os.path.join(BIN, 'sincqed')
FLOPS = os.path.join(LIB, 'flops.json')


def _newer(out, ins):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(i) > t for i in ins if os.path.exists(i))


def _flags_stamp():
    """A file holding the contracted units' compile policy (flags, spill limit, occupancy candidates): an
    input of every such unit, rewritten -- so newer than the objects -- only when the policy changes.  A
    first stamp is dated to the epoch: objects already built are taken to follow the policy."""
    path = os.path.join(BUILD, 'fma_policy.txt')
    text = json.dumps({'flags': NVFLAGS_FMA, 'spill_max': SPILL_MAX, 'sweeps_flops': SWEEPS_FLOPS}) + '\n'
    old = open(path).read() if os.path.exists(path) else None
    if old != text:
        os.makedirs(BUILD, exist_ok=True)
        with open(path, 'w') as f:
            f.write(text)
        if old is None:
            os.utime(path, (0, 0))
    return path


def _run(cmd, log=None):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode:
        raise RuntimeError('build step failed (%d): %s\n%s' % (r.returncode, ' '.join(cmd), r.stdout[-4000:]))
    return r.stdout


SYNTH = os.path.join(PKG, 'synth')
OCC = os.path.join(LIB, 'occupancy.json')

# The contracted FP64 kernel's occupancy, chosen per graph at build time from the compiler's own report:
# three resident CTAs per SM (registers capped at 168 for 128 threads) where that costs at most SPILL_MAX
# bytes of spill stores, else the uncapped allocation.  Measured on the B200 at h = 0.7: the capped
# kernels of the D = 7 three-loop graphs run 7-9 % faster, while g3_lbl, which would spill kilobytes,
# runs slower capped.
SPILL_MAX = 128
# The contracted unit's level kernel takes a batch's tiles in two sweeps (SQB_SWEEPS = 2: the children of
# cells that skip the |.| sums, then the others) for integrands of at least SWEEPS_FLOPS algorithmic flops
# per point with cells of at least 32 children: measured on the B200 at 50 % skipped cells, the two forms of
# such a point function interleaved on one SM run 1.3-1.6x slower than either alone (v4_65, 5,520 flops;
# w4_07Vm, 9,313; g3_lbl, 25,307), while g3_00's (2,137) do not.
SWEEPS_FLOPS = 4000
# the point function's spill stores: the contracted unit calls it (sqb_fcall, one copy per kernel); the
# exact unit inlines it into sqb_k_f64
_PTXAS_SPILL = re.compile(r'Function properties for (_Z9sqb_fcall|_Z9sqb_k_f64)\S*\s*\n\s*(\d+) bytes stack frame, (\d+) bytes spill stores')


def _spill(out):
    """The largest spill-store count ptxas reports for the point function (its calls if there are any,
    else the FP64 kernels); -1 if it reports none."""
    found = [(m.group(1), int(m.group(3))) for m in _PTXAS_SPILL.finditer(out)]
    calls = [v for k, v in found if k == '_Z9sqb_fcall']
    vals = calls or [v for k, v in found]
    return max(vals) if vals else -1


def _compile_graph(tu, o, tuf, of, name, do_exact, do_fma, sweeps=1):
    """Both units of one graph.  A graph whose contracted point function spills even at the uncapped
    allocation (g3_lbl: ~1 KB of stack per thread) is built without the level-mode tile sums in both units:
    their shared memory would take L1 from the stack it spills to (measured: g3_lbl 15 % slower with them)."""
    info = None
    if do_fma:
        sw = ['-DSQB_SWEEPS=2'] if sweeps > 1 else []
        out = _run([NVCC] + NVFLAGS_FMA + sw + ['-DSQB_MINB=3', '-Xptxas', '-v', '-I' + GEN, '-c', tuf, '-o', of])
        spill = _spill(out)
        info = {'min_blocks': 3, 'spill_stores_at_3': spill, 'fused': 1, 'sweeps': sweeps}
        if spill < 0 or spill > SPILL_MAX:
            out = _run([NVCC] + NVFLAGS_FMA + sw + ['-Xptxas', '-v', '-I' + GEN, '-c', tuf, '-o', of])
            spill1 = _spill(out)
            info = {'min_blocks': 1, 'spill_stores_at_3': spill, 'spill_stores_at_1': spill1, 'fused': 1, 'sweeps': sweeps}
            if spill1 < 0 or spill1 > SPILL_MAX:
                _run([NVCC] + NVFLAGS_FMA + sw + ['-DSQB_FUSE=0', '-I' + GEN, '-c', tuf, '-o', of])
                info['fused'] = 0
    elif os.path.exists(OCC):
        with open(OCC) as f:
            info = json.load(f).get(name)
    if do_exact:
        fuse = [] if not info or info.get('fused', 1) else ['-DSQB_FUSE=0']
        _run([NVCC] + NVFLAGS + fuse + ['-I' + GEN, '-c', tu, '-o', o])
    return name, info


def kernel_sources(kdir, classes):
    """the reference's kernels of these classes, then the synthetic integrands of sincfeyn_b200/synth"""
    out = []
    if not kdir:
        return out
    for c in classes.split():
        d = os.path.join(kdir, c)
        if os.path.isdir(d):
            out += sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith('.c'))
    if out:
        out += sorted(os.path.join(SYNTH, f) for f in os.listdir(SYNTH) if f.endswith('.c'))
    return out


def generate(srcs):
    """kgen every kernel; returns [(name, D, cuh path, tu path)] in registry order (first name wins,
    as driver/graphs.c:8-12)."""
    os.makedirs(GEN, exist_ok=True)
    me = [os.path.abspath(kgen.__file__)]
    graphs, seen = [], set()
    for src in srcs:
        base = os.path.splitext(os.path.basename(src))[0]
        cuh = os.path.join(GEN, base + '.cuh')
        if _newer(cuh, [src] + me):
            # rewritten only when the text changes, so that a generator change that leaves a graph's
            # output as it was does not recompile that graph
            k, text = kgen.emit(src)
            if not os.path.exists(cuh) or open(cuh).read() != text:
                with open(cuh, 'w') as f:
                    f.write(text)
        with open(cuh) as f:
            m = re.search(r'^SQ_GRAPH(?:_SPLIT)?\((\w+), "((?:[^"\\]|\\.)*)", (\d+), (\d+),', f.read(), re.M)
        name, D = m.group(1), int(m.group(4))
        if name in seen:
            continue
        seen.add(name)
        tu = os.path.join(GEN, 'k_%s.cu' % name)
        text = '#include "sqkern.cuh"\n#include "%s"\n' % os.path.basename(cuh)
        # the contracted FP64 kernel: its own unit and namespace (sqkern.cuh, SQ_GRAPH)
        tuf = os.path.join(GEN, 'kf_%s.cu' % name)
        textf = '#define SQB_FMA_TU 1\n#define SQG_NS(n) sqgf_##n\n' + text
        for path, t in ((tu, text), (tuf, textf)):
            if not os.path.exists(path) or open(path).read() != t:
                with open(path, 'w') as f:
                    f.write(t)
        graphs.append((name, D, cuh, tu))
    return graphs


def write_registry(graphs, flops):
    reg = os.path.join(GEN, 'registry.cu')
    L = ['/* generated by sincfeyn_b200/build.py: the graphs of this library */',
         '#include "sqb_internal.h"', '#include "sincfeyn_b200.h"', '#include <string.h>']
    for name, D, _, _ in graphs:
        L.append('extern "C" const sqb_graph_t SQB_%s;' % name)
    L.append('extern "C" const sqb_graph_t *const SQB_ALL[] = {')
    L += ['    &SQB_%s,' % n for n, _, _, _ in graphs] + ['    0 };', 'extern "C" const int SQB_NALL = %d;' % len(graphs)]
    # the reference's per-graph plug-in descriptors GG_<name> (driver/gpu_kernel.h:39, Makefile:231-234)
    L.append('extern "C" void sqb_gg_launch(const sqb_graph_t *g, void *st, long n, const short *k, const unsigned char *skip,'
             ' const double *EX, int K, double H, double *of, double *oab, int cmode, int cst);')
    for name, D, _, _ in graphs:
        L.append('static void gl_%s(sq_stream_t st, long n, const short *k, const unsigned char *skip, const double *EX, int K,'
                 ' double H, double *of, double *oab, int cmode, int cst){ sqb_gg_launch(&SQB_%s, (void*)st, n, k, skip, EX, K, H,'
                 ' of, oab, cmode, cst); }' % (name, name))
        L.append('extern "C" const sq_gpu_t GG_%s = {"%s", %d, gl_%s};' % (name, name, D, name))
    L.append('extern "C" const sq_gpu_t *GPU_ALL[] = {')
    L += ['    &GG_%s,' % n for n, _, _, _ in graphs] + ['    0 };']
    L.append('static const struct { const char *name; double ab1, ab0; } FLOPS[] = {')
    for name, _, _, _ in graphs:
        f = flops.get(name, {})
        L.append('    {"%s", %.1f, %.1f},' % (name, f.get('ab1', 0), f.get('ab0', 0)))
    L += ['    {0, 0, 0} };',
          'extern "C" double sqb_graph_flops(const char *name, int ab){',
          '    for(int i = 0; FLOPS[i].name; i++) if(!strcmp(FLOPS[i].name, name)) return ab ? FLOPS[i].ab1 : FLOPS[i].ab0;',
          '    return 0; }']
    text = '\n'.join(L) + '\n'
    if not os.path.exists(reg) or open(reg).read() != text:
        with open(reg, 'w') as f:
            f.write(text)
    return reg


def count_flops(graphs):
    """Compile every generated kernel over the counting type on the host and count one point."""
    src = os.path.join(GEN, 'count.cc')
    exe = os.path.join(BUILD, 'count')
    L = ['/* generated by sincfeyn_b200/build.py: algorithmic flop counter */',
         '#include <stdio.h>', '#include "sqcount.h"', 'long sq_flops, sq_trans;',
         '#define SQ_TABLE static const', '#define SQ_FUNC', '#define SQ_FUNC_K', '#define SQ_CHUNK', '#define SQ_CHUNK_DD', '#define RABS(x) sq_rabs(x)',
         '#define SQ_EXP(x) sq_exp(x)', '#define SQ_LOG(x) sq_log(x)', '#define SQG_NS(n) sqg_##n',
         '#define SQ_GRAPH_SPLIT(NAME, VOLKOV, L, D, W, NP, FIX, NPARTS) SQ_GRAPH(NAME, VOLKOV, L, D, W, NP, FIX)',
         '#define SQ_SCALE(NAME)',
         '#define SQ_GRAPH(NAME, VOLKOV, L, D, W, NP, FIX) \\',
         'static void count_##NAME(void){ sq_count sf[D], ab; for(int d = 0; d < D; d++) sf[d] = sq_count(0.7 + 0.37*d); \\',
         '  sq_flops = 0; sq_trans = 0; sqg_##NAME::K<sq_count, 1>::f_##NAME(sf, &ab); long a1 = sq_flops, t1 = sq_trans; \\',
         '  sq_flops = 0; sqg_##NAME::K<sq_count, 0>::f_##NAME(sf, &ab); long a0 = sq_flops; \\',
         '  printf("%s\\"%s\\": {\\"ab1\\": %ld, \\"ab0\\": %ld, \\"tr\\": %ld}", first ? "" : ",\\n", #NAME, a1, a0, t1); first = 0; }',
         'static int first = 1;']
    for name, D, cuh, _ in graphs:
        L.append('#include "%s"' % os.path.basename(cuh))
    L.append('int main(void){ printf("{\\n");')
    L += ['  count_%s();' % n for n, _, _, _ in graphs]
    L.append('  printf("\\n}\\n"); return 0; }')
    text = '\n'.join(L) + '\n'
    if not os.path.exists(src) or open(src).read() != text:
        with open(src, 'w') as f:
            f.write(text)
    if _newer(exe, [src, os.path.join(CSRC, 'sqcount.h')] + [g[2] for g in graphs]):
        _run([CXX, '-O0', '-std=c++17', '-I' + CSRC, '-I' + GEN, '-o', exe, src])
    if _newer(FLOPS, [exe]):
        out = _run([exe])
        os.makedirs(LIB, exist_ok=True)
        with open(FLOPS, 'w') as f:
            f.write(out)
    with open(FLOPS) as f:
        return json.load(f)


def generate_only(kernels=DEFAULT_KERNELS, classes='pi6'):
    """Run the code generator on classes that the library is not built with (default: pi6), so that their
    generated headers can be checked on the host; returns the graph names (none without sources)."""
    srcs = [f for f in kernel_sources(kernels, classes) if not f.startswith(SYNTH)]
    return [g[0] for g in generate(srcs)] if srcs else []


def build(kernels=DEFAULT_KERNELS, classes=DEFAULT_CLASSES, jobs=None, verbose=True):
    """Generate and compile whatever is out of date; returns the library path."""
    srcs = kernel_sources(kernels, classes)
    if not srcs:
        if os.path.exists(LIBSO):
            return LIBSO
        raise RuntimeError('no kernel sources under %s and no prebuilt %s: give the reference\'s kernels/ '
                           'directory (--kernels DIR or SQB_KERNELS)' % (kernels, LIBSO))
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    graphs = generate(srcs)
    flops = count_flops(graphs)
    reg = write_registry(graphs, flops)
    hdrs = [os.path.join(CSRC, f) for f in ('sqkern.cuh', 'sqdd.cuh', 'sqscale.cuh', 'sqorbit.cuh', 'sqb_internal.h', 'sqb_rt.h')] + \
           [os.path.join(INC, 'sincfeyn_b200.h')]
    khdrs = [os.path.join(CSRC, f) for f in ('sqkern.cuh', 'sqdd.cuh', 'sqscale.cuh', 'sqorbit.cuh', 'sqb_internal.h')]   # what a graph TU includes
    stamp = _flags_stamp()
    jobs_list = []
    for name, D, cuh, tu in graphs:
        o = os.path.join(OBJ, 'k_%s.o' % name)
        of = os.path.join(OBJ, 'kf_%s.o' % name)
        tuf = os.path.join(GEN, 'kf_%s.cu' % name)
        do_fma = _newer(of, [tuf, cuh, stamp] + khdrs)
        do_exact = do_fma or _newer(o, [tu, cuh] + khdrs)
        if do_fma or do_exact:
            sweeps = 2 if D >= 5 and flops.get(name, {}).get('ab1', 0) >= SWEEPS_FLOPS else 1
            jobs_list.append(lambda a=(tu, o, tuf, of, name, do_exact, do_fma, sweeps): _compile_graph(*a))
    rt_o = os.path.join(OBJ, 'runtime.o')
    if _newer(rt_o, [os.path.join(CSRC, 'runtime.cu')] + hdrs):
        jobs_list.append([NVCC] + NVFLAGS + ['-Xcompiler', '-fopenmp', '-c', os.path.join(CSRC, 'runtime.cu'), '-o', rt_o])
    tg_o = os.path.join(OBJ, 'topgrid.o')
    if _newer(tg_o, [os.path.join(CSRC, 'topgrid.cu')] + hdrs):
        jobs_list.append([NVCC] + NVFLAGS + ['-c', os.path.join(CSRC, 'topgrid.cu'), '-o', tg_o])
    pr_o = os.path.join(OBJ, 'predict.o')
    if _newer(pr_o, [os.path.join(CSRC, 'predict.cu')] + hdrs):
        jobs_list.append([NVCC] + NVFLAGS + ['-c', os.path.join(CSRC, 'predict.cu'), '-o', pr_o])
    na_o = os.path.join(OBJ, 'noalloc.o')
    if _newer(na_o, [os.path.join(CSRC, 'noalloc.cu')] + hdrs):
        jobs_list.append([NVCC] + NVFLAGS + ['-c', os.path.join(CSRC, 'noalloc.cu'), '-o', na_o])
    reg_o = os.path.join(OBJ, 'registry.o')
    if _newer(reg_o, [reg] + hdrs):
        jobs_list.append([NVCC] + NVFLAGS + ['-c', reg, '-o', reg_o])
    eng_o = os.path.join(OBJ, 'engine.o')
    if _newer(eng_o, [os.path.join(CSRC, 'engine.cpp')] + hdrs):
        jobs_list.append([CXX] + CXXFLAGS + ['-c', os.path.join(CSRC, 'engine.cpp'), '-o', eng_o])
    ck_o = os.path.join(OBJ, 'ckpt.o')
    if _newer(ck_o, [os.path.join(CSRC, 'ckpt.cpp')] + hdrs):
        jobs_list.append([CXX] + CXXFLAGS + ['-c', os.path.join(CSRC, 'ckpt.cpp'), '-o', ck_o])
    bat_o = os.path.join(OBJ, 'batch.o')
    if _newer(bat_o, [os.path.join(CSRC, 'batch.cpp')] + hdrs):
        jobs_list.append([CXX] + CXXFLAGS + ['-pthread', '-c', os.path.join(CSRC, 'batch.cpp'), '-o', bat_o])
    sym_o = os.path.join(OBJ, 'sym.o')
    if _newer(sym_o, [os.path.join(CSRC, 'sym.cpp'), os.path.join(CSRC, 'sqb_rand.h')] + hdrs):
        jobs_list.append([CXX] + CXXFLAGS + ['-c', os.path.join(CSRC, 'sym.cpp'), '-o', sym_o])
    sc_o = os.path.join(OBJ, 'scale.o')
    if _newer(sc_o, [os.path.join(CSRC, 'scale.cpp'), os.path.join(CSRC, 'sqb_rand.h')] + hdrs):
        jobs_list.append([CXX] + CXXFLAGS + ['-c', os.path.join(CSRC, 'scale.cpp'), '-o', sc_o])
    n = jobs or min(len(jobs_list) or 1, os.cpu_count() or 4)
    if verbose and jobs_list:
        print('sincfeyn_b200: compiling %d objects with %d jobs' % (len(jobs_list), n), file=sys.stderr)
    occ = {}
    if os.path.exists(OCC):
        with open(OCC) as f:
            occ = json.load(f)
    with cf.ThreadPoolExecutor(max_workers=n) as ex:
        for f in [ex.submit(c) if callable(c) else ex.submit(_run, c) for c in jobs_list]:
            r = f.result()
            if isinstance(r, tuple) and r[1] is not None:
                occ[r[0]] = r[1]
    with open(OCC, 'w') as f:
        json.dump(occ, f, indent=0, sort_keys=True)
    objs = [os.path.join(OBJ, 'k_%s.o' % g[0]) for g in graphs] + \
           [os.path.join(OBJ, 'kf_%s.o' % g[0]) for g in graphs] + [rt_o, tg_o, pr_o, na_o, reg_o, eng_o, bat_o, ck_o, sym_o, sc_o]
    if _newer(LIBSO, objs):
        _run([NVCC] + ARCH + ['-shared', '-o', LIBSO] + objs + ['-Xcompiler', '-fopenmp', '-lgomp', '-lpthread'])
    main_cpp = os.path.join(CSRC, 'main.cpp')
    if _newer(CLI, [main_cpp, LIBSO, os.path.join(INC, 'sincfeyn_b200.h')]):
        _run([CXX, '-O2', '-std=c++17', '-I' + INC, '-o', CLI, main_cpp, '-L' + LIB, '-lsqb200',
              '-Wl,-rpath,$ORIGIN/../lib'])
    return LIBSO


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument('--kernels', default=DEFAULT_KERNELS)
    ap.add_argument('--classes', default=DEFAULT_CLASSES)
    ap.add_argument('-j', '--jobs', type=int, default=None)
    ap.add_argument('--clean', action='store_true')
    a = ap.parse_args(argv)
    if a.clean:
        shutil.rmtree(BUILD, ignore_errors=True)
    print(build(a.kernels, a.classes, a.jobs))


if __name__ == '__main__':
    main()
