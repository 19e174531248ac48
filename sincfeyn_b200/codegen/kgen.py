#!/usr/bin/env python3
"""kgen -- the kernel code generator: one generated sincFeyn graph kernel (kernels/<class>/<g>.c)
into device code for this evaluator.  It replaces the reference's tools/gpugen.py for the same kernel
sources, with a different construction.

A kernel file holds two complete copies of the integrand: a double half and a QREAL half
(driver/common.h:5-22, e.g. kernels/g2/g2_00.c:7-231 and :232-462).  The QREAL half is scalar C written
against the macros REAL, FN(x) and RABS(x) and the thread-local flag SQ_AB, with no calls other than its
own functions (pt_, f_, vp_, helper p_/nd_, chunk functions bk_/ab_).  kgen wraps that half, unchanged in
its arithmetic, into a class template

    template<class SqReal_, int SQ_AB> struct K { static ... pt_<g>(...); static ... f_<g>(...); };

so that one text compiles as
  * FP64 device code with SQ_AB a compile-time constant (K<double,1> and K<double,0>: the skip variant
    loses the |.| companion sums entirely instead of branching over them),
  * double-double device code (K<sqdd,1>) for the precision fallback and the all-dd form,
  * host C++ over a counting number type (K<sq_count,..>), which gives the algorithmic flop count of
    the double path per point for each SQ_AB (+ - * / each 1, as in scripts/plot5_cost.py:11).

The graph descriptor `const graph_t G_<g>={name,volkov,L,D,weight,n,fixed,...}` (driver/common.h:38)
and the Gauss-Legendre tables are carried over as data.

    python3 -m sincfeyn_b200.codegen.kgen KERNEL.c OUT.cuh
"""
import re
import sys

_DESC = re.compile(r'^const graph_t G_(\w+)=\{"([^"]*)","([^"]*)",(\d+),(\d+),(\d+),(\d+),(\d+),', re.M)
_GL = re.compile(r'^static const double (GL[XW]_\w+)\[(\d+)\]=\{([^}]*)\}(?:, (GL[XW]_\w+)\[(\d+)\]=\{([^}]*)\})?;', re.M)
_TAB1 = re.compile(r'^static const double (\w+)\[(\d+)\]=\{([^}]*)\};$', re.M)
_FDEF = re.compile(r'^static (REAL|void) FN\((\w+)\)\(', re.M)


class KernelSource:
    """The parts of one generated kernel file that the evaluator needs."""

    def __init__(self, path):
        with open(path) as f:
            txt = f.read()
        self.path = path
        m = _DESC.search(txt)
        if not m:
            raise ValueError('%s: no graph descriptor' % path)
        self.name, self.volkov = m.group(1), m.group(3)
        self.L, self.D, self.weight, self.n, self.fixed = (int(m.group(i)) for i in range(4, 9))
        self.gl = []
        for g in _GL.finditer(txt):
            self.gl.append((g.group(1), int(g.group(2)), g.group(3)))
            if g.group(4):
                self.gl.append((g.group(4), int(g.group(5)), g.group(6)))
        for g in _TAB1.finditer(txt):                 # single-table lines (the synthetic integrands)
            if g.group(1) not in [t[0] for t in self.gl]:
                self.gl.append((g.group(1), int(g.group(2)), g.group(3)))
        i = txt.index('#define REAL QREAL')
        j = txt.index('#define FN(x) x##_q', i) + len('#define FN(x) x##_q')
        k = txt.index('#undef REAL', j)
        self.qhalf = txt[j:k]
        self.funcs = [(m.group(1), m.group(2)) for m in _FDEF.finditer(self.qhalf)]
        if ('REAL', 'f_' + self.name) not in self.funcs:
            raise ValueError('%s: no f_%s in the QREAL half' % (path, self.name))

    def chunk(self, fname):
        return re.match(r'(bk|ab)_', fname) is not None

    def body(self, chunk_attr='SQ_CHUNK', func_attr='SQ_FUNC'):
        """The QREAL half with each function turned into a static member of the class template; the chunk
        functions (bk_/ab_) get chunk_attr, the others func_attr."""
        def repl(m):
            ret, fname = m.group(1), m.group(2)
            attr = chunk_attr if self.chunk(fname) else func_attr
            return 'static %s %s FN(%s)(' % (attr, ret, fname)
        b = _FDEF.sub(repl, self.qhalf)
        rest = re.sub(r'static (%s|%s)' % (chunk_attr, func_attr), '', b)
        if re.search(r'\bstatic\b', rest):
            raise ValueError('%s: unexpected static in the QREAL half' % self.path)
        return b


def emit(src):
    """Header text for one graph: namespace SQG_NS(<name>) (a macro of the including unit, normally
    sqg_<name>) with the tables and two copies of the class
    template -- K, whose chunk functions are SQ_CHUNK and whose other functions (pt_, vp_, helpers) are
    SQ_FUNC_K (the FP64 evaluation: all inlined, so that the argument arrays stay in registers), and KD, whose chunk functions are SQ_CHUNK_DD (double-double:
    real calls, which keeps the compile of the large kernels bounded) -- then SQ_GRAPH(...), which the
    including translation unit defines (kernels and registry entry, or flop counter)."""
    k = KernelSource(src)
    out = ['/* generated by sincfeyn_b200/codegen/kgen.py from %s (QREAL half, arithmetic unchanged) */'
           % re.sub(r'^.*?(kernels/)', r'\1', src),
           'namespace SQG_NS(%s) {' % k.name]
    for name, n, vals in k.gl:
        out.append('SQ_TABLE double %s[%d] = {%s};' % (name, n, vals))
    out += ['#define REAL SqReal_', '#define FN(x) x',
            'template<class SqReal_, int SQ_AB> struct K {',
            k.body('SQ_CHUNK', 'SQ_FUNC_K').strip('\n'),
            '};']
    if any(k.chunk(f) for _, f in k.funcs):
        out += ['template<class SqReal_, int SQ_AB> struct KD {',
                k.body('SQ_CHUNK_DD').strip('\n'),
                '};']
    else:
        out += ['template<class SqReal_, int SQ_AB> using KD = K<SqReal_, SQ_AB>;']
    out += ['#undef REAL', '#undef FN', '}',
            'SQ_GRAPH(%s, "%s", %d, %d, %d, %d, %d)' % (k.name, k.volkov.replace('"', '\\"'),
                                                        k.L, k.D, k.weight, k.n, k.fixed)]
    return k, '\n'.join(out) + '\n'


def main(argv):
    if len(argv) != 2:
        sys.exit('usage: kgen.py KERNEL.c OUT.cuh')
    k, text = emit(argv[0])
    with open(argv[1], 'w') as f:
        f.write(text)


if __name__ == '__main__':
    main(sys.argv[1:])
