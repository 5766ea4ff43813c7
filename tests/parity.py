"""Parity helpers: run one scenario through two cores and compare bitwise."""

import numpy as np

import helpers as H

pkg, sc = H.pkg, H.scenarios


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def first_difference(a, b):
    for f in ("x", "y", "vx", "vy"):
        ua, ub = bits(getattr(a, f)), bits(getattr(b, f))
        if not np.array_equal(ua, ub):
            i = int(np.nonzero(ua != ub)[0][0])
            return "node %d %s: %r vs %r" % (i, f, getattr(a, f)[i], getattr(b, f)[i])
    return None


def run_pair(setup, ocore, gcore, ticks, step=1, check_every=1):
    """setup(core) -> (nodes, sim). Ticks both and compares after every check."""
    na, sa = setup(ocore)
    nb, sb = setup(gcore)
    try:
        d = first_difference(na, nb)
        assert d is None, "after initialize: " + d
        t = 0
        while t < ticks:
            k = min(step, ticks - t)
            sa.tick(k)
            sb.tick(k)
            t += k
            if t % check_every == 0 or t == ticks:
                d = first_difference(na, nb)
                assert d is None, "tick %d: %s" % (t, d)
                assert sa.alpha() == sb.alpha()
        if sa.randomSource() is None:
            assert ocore.sim_get_lcg(sa.ctx.h) == gcore.sim_get_lcg(sb.ctx.h), "random stream position"
        else:  # each side drew from its own copy of the caller's function
            assert sa.randomSource()() == sb.randomSource()(), "random stream position"
    finally:
        sa.close()
        sb.close()
