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
        # the descriptor's remaining fields: fd, fq, ptd, ptq[, fv]; a graph with a raw QREAL point function
        # (ptq) has the scaling test (driver/main.c:197; VP graphs have 0 there)
        rest = txt[m.end():txt.index('}', m.end())].split(',')
        self.has_ptq = len(rest) > 3 and rest[3].strip() == 'pt_%s_q' % self.name
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
        if self.has_ptq and ('REAL', 'pt_' + self.name) not in self.funcs:
            raise ValueError('%s: the descriptor names pt_%s_q, the QREAL half has no pt_%s' % (path, self.name, self.name))

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


_PT_DEF = re.compile(r'^static REAL FN\((pt_\w+)\)\(const REAL \*x, const REAL Vx, REAL \*ab\)\{$', re.M)


def split_plan(k, max_parts=12):
    max_parts = min(max_parts, 16)         # sqkern.cuh launches at most sixteen passes
    """A point function that is a flat sum of independent forest nodes can be evaluated in passes.

    Returns None, or (groups, text) for the graph's FP64 split: the QREAL half's pt_<g> holds a header
    (x0..x{n-1}), node sections (each opened by a `/* node` comment, using only the header and its own
    names: checked), `REAL tot=0, tota=0;`, one accumulation block per node ending in `tot+=r` or
    `tot-=r; tota+=ra; }`, and `*ab=tota; return tot;`; its f_<g> calls it once, from a one-point
    Gauss-Legendre loop.  Pass P evaluates the nodes of group P and applies their accumulation blocks to
    the running (tot, tota) of the point, kept in memory between passes; the final pass applies f_'s
    own arithmetic to them.  Every operation and its order are those of the unsplit function, so the
    values are the same.  The groups are consecutive nodes, about equal in text size."""
    q = k.qhalf
    m = _PT_DEF.search(q)
    if not m:
        return None
    pt = m.group(1)
    body_start = m.end()
    end = q.index('\n}\n', body_start)
    lines = q[body_start:end].split('\n')[1:]
    heads = [n for n, l in enumerate(lines) if l.strip().startswith('/* node')]
    tots = [n for n, l in enumerate(lines) if l.strip() == 'REAL tot=0, tota=0;']
    if len(heads) < 8 or len(tots) != 1 or lines[-1].strip() != '*ab=tota; return tot;':
        return None
    header = lines[:heads[0]]
    if not all(re.match(r'\s*const REAL x\d+=x\[\d+\];$', l) for l in header):
        return None
    secs = [lines[heads[a]:(heads[a + 1] if a + 1 < len(heads) else tots[0])] for a in range(len(heads))]
    blocks, cur = [], []
    for l in lines[tots[0] + 1:-1]:
        cur.append(l)
        if re.search(r'tot[+-]=r; tota\+=ra; \}$', l.strip()):
            blocks.append(cur)
            cur = []
    if cur or len(blocks) != len(secs):
        return None
    defs = [set(re.findall(r'\b([A-Za-z_]\w*)(?=\[[^]]*\]*\s*(?:=|,|;))|(?:REAL|,)\s*([A-Za-z_]\w*)\s*[=;,\[]', '\n'.join(sec)))
            for sec in secs]
    names = [set(a or b for a, b in d) for d in defs]
    hdr = set(re.findall(r'const REAL (x\d+)=', '\n'.join(header)))
    for a, sec in enumerate(secs):
        used = set(re.findall(r'\b([A-Za-z_]\w*)\b', '\n'.join(sec)))
        for b, nb in enumerate(names):
            if b != a and (used & (nb - names[a]) - hdr):
                return None
    # the f_ function: one call of pt, inside a one-point loop
    fm = re.search(r'^static REAL FN\((f_%s)\)\(const REAL \*sf, REAL \*ab\)\{\n(.*?)\n\}$' % re.escape(k.name), q, re.M | re.S)
    if not fm:
        return None
    fbody = fm.group(2)
    call = 'FN(%s)(s,0,&a)' % pt
    if fbody.count(call) != 1 or not re.search(r'for\(int g=0;g<1;g\+\+\)', fbody) or q.count('FN(%s)(' % pt) != 2:
        return None
    # consecutive groups of about equal text size
    size = [sum(len(l) for l in sec) for sec in secs]
    target = sum(size)/max_parts
    groups, g, acc = [], [], 0
    for a in range(len(secs)):
        g.append(a); acc += size[a]
        if acc >= target and len(groups) < max_parts - 1:
            groups.append(g); g, acc = [], 0
    if g:
        groups.append(g)
    out = []
    for P, grp in enumerate(groups):
        out.append('static SQ_FUNC_K void FN(ptp%d_%s)(const REAL *x, const REAL Vx, REAL *tot_, REAL *tota_){' % (P, k.name))
        out += header
        for a in grp:
            out += secs[a]
        out.append('  REAL tot=*tot_, tota=*tota_;')
        for a in grp:
            out += blocks[a]
        out.append('  *tot_=tot; *tota_=tota;')
        out.append('}')
        fp = fbody.replace('REAL acc=0, aa=0, a;', '')
        fp = fp.replace('const REAL wg=(REAL)GLW_%s[g]; acc+=wg*%s; aa+=wg*a; }' % (k.name, call),
                        'FN(ptp%d_%s)(s,0,tot_,tota_); }' % (P, k.name))
        fp = fp[:fp.index('const REAL nrm=')] if 'const REAL nrm=' in fp else None
        if fp is None or 'FN(ptp' not in fp:
            return None
        out.append('static SQ_FUNC_K void FN(fpart%d_%s)(const REAL *sf, REAL *tot_, REAL *tota_){' % (P, k.name))
        out.append(fp.rstrip())
        out.append('}')
    fin = fbody.replace(call, '(a=TA_, TT_)')
    out.append('static SQ_FUNC_K REAL FN(ffin_%s)(const REAL *sf, const REAL TT_, const REAL TA_, REAL *ab){' % k.name)
    out.append(fin)
    out.append('}')
    # pass P by a template parameter (only the selected pass is compiled into a kernel)
    out.append('template<int P> static SQ_FUNC_K void FN(fpart_%s)(const REAL *sf, REAL *tot_, REAL *tota_){' % k.name)
    for P in range(len(groups)):
        out.append('  %sif constexpr(P == %d) FN(fpart%d_%s)(sf, tot_, tota_);' % ('else ' if P else '', P, P, k.name))
    out.append('}')
    return groups, '\n'.join(out)


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
    plan = split_plan(k)
    out += ['#define REAL SqReal_', '#define FN(x) x',
            'template<class SqReal_, int SQ_AB> struct K {',
            k.body('SQ_CHUNK', 'SQ_FUNC_K').strip('\n')]
    if plan:
        out += ['/* the same point function in %d passes over groups of its nodes (kgen.split_plan) */' % len(plan[0]),
                plan[1]]
    out += ['};']

    if any(k.chunk(f) for _, f in k.funcs):
        out += ['template<class SqReal_, int SQ_AB> struct KD {',
                k.body('SQ_CHUNK_DD').strip('\n'),
                '};']
    else:
        out += ['template<class SqReal_, int SQ_AB> using KD = K<SqReal_, SQ_AB>;']
    out += ['#undef REAL', '#undef FN', '}']
    if plan:
        out.append('SQ_GRAPH_SPLIT(%s, "%s", %d, %d, %d, %d, %d, %d)' % (k.name, k.volkov.replace('"', '\\"'),
                                                                    k.L, k.D, k.weight, k.n, k.fixed, len(plan[0])))
    else:
        out.append('SQ_GRAPH(%s, "%s", %d, %d, %d, %d, %d)' % (k.name, k.volkov.replace('"', '\\"'),
                                                            k.L, k.D, k.weight, k.n, k.fixed))
    if k.has_ptq:
        out.append('SQ_SCALE(%s)' % k.name)
    return k, '\n'.join(out) + '\n'


def main(argv):
    if len(argv) != 2:
        sys.exit('usage: kgen.py KERNEL.c OUT.cuh')
    k, text = emit(argv[0])
    with open(argv[1], 'w') as f:
        f.write(text)


if __name__ == '__main__':
    main(sys.argv[1:])
