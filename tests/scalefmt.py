"""The reference's printed lines of `sincqed scale` (driver/main.c:104-113, :197) from a scale result."""


def scale_lines(name, volkov, r, kappa):
    if r is None:
        return ['%-6s %-22s (no scale test for VP graphs)' % (name, volkov)]
    out = ['  slow direction e=(%s)  |g| at kappa/3,2/3,1: %.3e %.3e %.3e' % (''.join('%+d' % x for x in e), *g)
           for e, g in r['listed']]
    out.append('%-6s %-22s scale test kappa=%g: %d directions, %d slow (ratio>0.3), worst ratio %.3g (dir %d: e=(%s) '
               '|g| %.2e %.2e %.2e)' % (name, volkov, kappa, r['ndir'], r['slow'], r['worst'], r['worst_dir'],
                                        ''.join('%+d' % x for x in r['worst_e']), *r['worst_g']))
    return out
