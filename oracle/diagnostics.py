"""CPU restatement of the reference's beam diagnostics (test infrastructure
only): diagnostics.hpp:38-180, serial loops in the reference's order, on
[N, 3] host arrays of live particles."""

import math


def _csqrt(v):
    """C's sqrt: NaN for a negative argument (a rounding-level negative
    variance of a degenerate beam gives NaN, as in the reference)."""
    return math.sqrt(v) if v >= 0 else float("nan")


def kinetic_energies(p, m, c):
    """diagnostics.hpp:38-58: v = c p / sqrt(m^2 c^2 + p^2), (p/v - m) c^2."""
    out = []
    for pi, mi in zip(p, m):
        pn = math.sqrt(pi[0] ** 2 + pi[1] ** 2 + pi[2] ** 2)
        v = c * pn / math.sqrt(mi * mi * c * c + pn * pn)
        out.append((pn / v - mi) * c * c)
    return out


def total_charge(q):
    s = 0.0
    for qi in q:
        s += qi
    return s


def particle_momentum(p):
    s = [0.0, 0.0, 0.0]
    for pi in p:
        for d in range(3):
            s[d] += pi[d]
    return s


def rms_beam_size(x, axis):
    if len(x) == 0:
        return 0.0
    s = 0.0
    for xi in x:
        s += xi[axis] ** 2
    return math.sqrt(s / len(x))


def rms_beam_emittance(x, p, axis, beam_axis):
    n = len(x)
    if n == 0:
        return 0.0
    mx = mxp = mx2 = mxp2 = mxxp = 0.0
    for xi, pi in zip(x, p):
        xv = xi[axis]
        mx += xv
        mx2 += xv * xv
        xp = pi[axis] / pi[beam_axis] if pi[beam_axis] else 0.0
        mxp += xp
        mxp2 += xp * xp
        mxxp += xv * xp
    mx /= n
    mxp /= n
    mx2 /= n
    mxp2 /= n
    mxxp /= n
    return _csqrt(mx2 * mxp2 - mx ** 2 * mxp2 - mx2 * mxp ** 2
                  - (mxxp ** 2 - 2 * mxxp * mx * mxp))


def std_dev(values):
    """tools.hpp:303-322."""
    if not values:
        raise RuntimeError("attempted to take empty average")
    s = s2 = 0.0
    for v in values:
        s += v
        s2 += v * v
    mean = s / len(values)
    return _csqrt(s2 / len(values) - mean ** 2)


def rms_energy_spread(p, m, c):
    if len(p) == 0:
        return 0.0
    return std_dev(kinetic_energies(p, m, c))


def particle_current(q, v, length):
    s = [0.0, 0.0, 0.0]
    for qi, vi in zip(q, v):
        for d in range(3):
            s[d] += qi * vi[d]
    return [si / length for si in s]
