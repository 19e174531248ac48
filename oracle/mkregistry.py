#!/usr/bin/env python3
"""Test infrastructure (oracle build only): the graph list of an oracle build of the reference.

The reference generates `register_graphs()` from the `const graph_t G_<name>` lines of the kernel
sources (Makefile:145-152); graphs are added in file order and the first one of a name wins
(driver/graphs.c:8-12).  This writes the same list for the kernel files given on the command line.

    python3 mkregistry.py KERNEL.c ... > registry.c
"""
import re
import sys

names = []
for fn in sys.argv[1:]:
    with open(fn) as f:
        for line in f:
            m = re.match(r'const graph_t (G_[A-Za-z0-9_]+)', line)
            if m:
                names.append(m.group(1))
out = ['/* graphs of this oracle build (oracle/mkregistry.py) */', '#include "sq.h"']
out += ['extern const graph_t %s;' % n for n in names]
out.append('void register_graphs(void){')
out += ['    add_graph(&%s);' % n for n in names]
out.append('}')
sys.stdout.write('\n'.join(out) + '\n')
