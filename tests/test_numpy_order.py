"""The host's numpy / BLAS summation orders that the oracle and the kernels
restate: einsum('nij,nj->ni') and einsum('nij,nkj->nik') as (t0 + t2) + t1,
np.linalg.norm(axis=-1) as a left-to-right sum of squares, 3-vector dot and
row-major @ transposed-matrix as fma(a2,b2, fma(a1,b1, a0*b0)), and 3x3
matrix @ vector as fma(r2,x2, fma(r0,x0, r1*x1)).

These orders come from numpy and its bundled OpenBLAS and may depend on the
CPU's SIMD dispatch, so the same checks run twice: here (unmarked) and, marked
``gpu``, on the host of the GPU machine, whose reference runs the drop-in
tests there.
"""
from fractions import Fraction

import numpy as np
import pytest


def _fma(a, b, c):
    """Correctly rounded a*b + c (exact rational arithmetic, one rounding)."""
    return float(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c)))


def _dot_chain(a, b):
    return _fma(a[2], b[2], _fma(a[1], b[1], float(a[0]) * float(b[0])))


def _gemv_row(r, x):
    return _fma(r[2], x[2], _fma(r[0], x[0], float(r[1]) * float(x[1])))


def _check_orders(seed):
    rng = np.random.default_rng(seed)
    # wide exponent spread so that the orders give different roundings
    def draw(*shape):
        return rng.normal(size=shape) * np.exp2(rng.integers(-20, 20, size=shape))

    A = draw(64, 3, 3)
    x = draw(64, 3)
    got = np.einsum('nij,nj->ni', A, x)
    t = A * x[:, None, :]
    assert np.array_equal(got, (t[..., 0] + t[..., 2]) + t[..., 1]), "einsum('nij,nj->ni')"

    B = draw(64, 3, 3)
    got = np.einsum('nij,nkj->nik', A, B)
    t = A[:, :, None, :] * B[:, None, :, :]
    assert np.array_equal(got, (t[..., 0] + t[..., 2]) + t[..., 1]), "einsum('nij,nkj->nik')"

    for width in (3, 4):
        v = draw(64, width)
        s = v[:, 0] * v[:, 0]
        for c in range(1, width):
            s = s + v[:, c] * v[:, c]
        assert np.array_equal(np.linalg.norm(v, axis=-1), np.sqrt(s)), 'norm of %d-vectors' % width

    for _ in range(32):
        a, b = draw(3), draw(3)
        assert float(np.dot(a, b)) == _dot_chain(a, b), 'np.dot of 3-vectors'
        R, y = draw(3, 3), draw(3)
        assert np.array_equal(R @ y, [_gemv_row(R[i], y) for i in range(3)]), '3x3 @ vector'

    R = draw(3, 3)
    for rows in (3, 8, 300):
        P = draw(rows, 3)
        want = np.array([[_dot_chain(P[p], R[c]) for c in range(3)] for p in range(rows)])
        assert np.array_equal(P @ R.T, want), '(%d,3) @ R.T' % rows


@pytest.mark.parametrize('seed', [0, 1])
def test_summation_orders_on_this_host(seed):
    _check_orders(seed)


@pytest.mark.gpu
def test_summation_orders_on_the_gpu_host():
    _check_orders(2)
