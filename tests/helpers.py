"""Shared helpers for the parity tests: seeded field data and QM31 circle points."""
import numpy as np

P = (1 << 31) - 1


def rng(seed):
    return np.random.default_rng(seed)


def m31(r, n):
    """n uniform M31 elements in [0, p)."""
    return r.integers(0, P, n, dtype=np.uint64).astype(np.uint32)


def m31_nonzero(r, n):
    return r.integers(1, P, n, dtype=np.uint64).astype(np.uint32)


def qm31_vals(r, n):
    return m31(r, 4 * n).reshape(n, 4)


# Pure-Python QM31 arithmetic for building test points (tiny, exact).
def _cm_mul(x, y):
    return ((x[0] * y[0] - x[1] * y[1]) % P, (x[0] * y[1] + x[1] * y[0]) % P)


def _cm_add(x, y):
    return ((x[0] + y[0]) % P, (x[1] + y[1]) % P)


def _cm_sub(x, y):
    return ((x[0] - y[0]) % P, (x[1] - y[1]) % P)


def _cm_inv(x):
    n = (x[0] * x[0] + x[1] * x[1]) % P
    ni = pow(n, P - 2, P)
    return (x[0] * ni % P, (-x[1]) * ni % P)


def q_mul(x, y):
    a, b = (x[0], x[1]), (x[2], x[3])
    c, d = (y[0], y[1]), (y[2], y[3])
    ac, bd = _cm_mul(a, c), _cm_mul(b, d)
    rbd = _cm_mul((2, 1), bd)
    re = _cm_add(ac, rbd)
    im = _cm_add(_cm_mul(a, d), _cm_mul(b, c))
    return (re[0], re[1], im[0], im[1])


def q_add(x, y):
    return tuple((a + b) % P for a, b in zip(x, y))


def q_sub(x, y):
    return tuple((a - b) % P for a, b in zip(x, y))


def q_inv(x):
    a, b = (x[0], x[1]), (x[2], x[3])
    den = _cm_sub(_cm_mul(a, a), _cm_mul((2, 1), _cm_mul(b, b)))
    di = _cm_inv(den)
    ra = _cm_mul(a, di)
    rb = _cm_mul(b, di)
    return (ra[0], ra[1], (-rb[0]) % P, (-rb[1]) % P)


ONE = (1, 0, 0, 0)


def random_circle_point(r):
    """A QM31 point on x^2 + y^2 = 1 from the rational parametrisation
    ((1 - t^2) / (1 + t^2), 2t / (1 + t^2))."""
    t = tuple(int(v) for v in m31(r, 4))
    t2 = q_mul(t, t)
    den = q_inv(q_add(ONE, t2))
    x = q_mul(q_sub(ONE, t2), den)
    y = q_mul(q_add(t, t), den)
    assert q_add(q_mul(x, x), q_mul(y, y)) == ONE
    return x, y


def random_qm31(r):
    return tuple(int(v) for v in m31(r, 4))
