#!/usr/bin/env python3
"""Test infrastructure (oracle build only): prepare one generated sincFeyn kernel source for the
oracle build of the reference, the way the reference's own build prepares it.

The reference Makefile pipes every kernel through an awk filter (Makefile:157-162, `KPREP`) before
compiling it.  That filter changes what the kernel computes, so an oracle build that skipped it would
not be the reference.  This script restates its three edits:

  1. in the double half only (text before `#define REAL QREAL`), every accumulation of a |.|
     companion sum written as `; n_<id>_Wa[..]..+=` on a line gets an `if(SQ_AB) ` guard
     (Makefile:161), so SQ_AB = 0 skips it;
  2. with the double-double fallback (the reference default, DD=1, compiled as C++), the graph
     descriptor `const graph_t G_` becomes `extern const graph_t G_` (Makefile:162; a namespace-scope
     const has internal linkage in C++);
  3. the QREAL half is preceded by `#pragma GCC optimize ("<QOPT>")` (Makefile:160, QOPT=O1).

    python3 kprep.py [--qopt O1] [--no-dd] KERNEL.c > out.cc
"""
import re
import sys

_WA = re.compile(r'; n_[A-Za-z0-9_]+_Wa(\[[^]]*\])+\+=')


def guard_line(line):
    """Insert `if(SQ_AB) ` after the `; ` of every |.|-sum accumulation on this line."""
    out, pos = [], 0
    for m in _WA.finditer(line):
        out.append(line[pos:m.start() + 2])
        out.append('if(SQ_AB) ')
        pos = m.start() + 2
    out.append(line[pos:])
    return ''.join(out)


def prepare(src, qopt='O1', dd=True):
    lines = src.split('\n')
    out, in_q = [], False
    for line in lines:
        if line.startswith('#define REAL QREAL'):
            in_q = True
            if qopt:
                out.append('#pragma GCC optimize ("%s")' % qopt)
        if not in_q and '_Wa[' in line:
            line = guard_line(line)
        if dd and line.startswith('const graph_t G_'):
            line = 'extern ' + line
        out.append(line)
    return '\n'.join(out)


def main(argv):
    qopt, dd, files = 'O1', True, []
    i = 0
    while i < len(argv):
        a = argv[i]
        if a == '--qopt':
            qopt = argv[i + 1]
            i += 2
            continue
        if a == '--no-dd':
            dd = False
        else:
            files.append(a)
        i += 1
    if len(files) != 1:
        sys.exit('usage: kprep.py [--qopt O1] [--no-dd] KERNEL.c')
    with open(files[0]) as f:
        sys.stdout.write(prepare(f.read(), qopt, dd))


if __name__ == '__main__':
    main(sys.argv[1:])
