"""The split form's decision bounds (csrc/expm_batched.cu, `powers`): the width
around |A^4|_1 and |A^6|_1 must hold any FP64 evaluation of those norms, in
any summation order, complex 4M included. Checked here against powers
computed in extended precision (64-bit mantissa, so its own error is 2^-11 of
the bound's scale) for FP64 products in two different summation orders
(numpy's BLAS and a plain k-ordered loop).
"""
import numpy as np
import pytest

U = 2.0 ** -53


def widths(n, a1, p2, p4, p6):
    """The bound of expm_batched.cu's `powers`, term for term."""
    un = n * U
    g = 4.0 * un / (1.0 - un)
    e2 = g * a1 * a1
    q2 = p2 + e2
    e4 = g * q2 * q2 + 2.0 * q2 * e2 + e2 * e2
    q4 = p4 + e4
    e6 = g * q2 * q4 + q2 * e4 + e2 * q4 + e2 * e4
    return 2.0 * (e4 + g * p4), 2.0 * (e6 + g * p6)


def norm1(x):
    return np.abs(x).sum(axis=0).max()


def kloop(a, b):
    """C = A B with each entry summed in k order, one rounding per step."""
    c = np.zeros((a.shape[0], b.shape[1]), dtype=a.dtype)
    for k in range(a.shape[1]):
        c = c + np.outer(a[:, k], b[k, :])
    return c


@pytest.mark.parametrize("n", [16, 48])
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("kind", ["gaussian", "cancelling"])
def test_bounds_hold_fp64_norms(n, cplx, kind):
    rng = np.random.default_rng(n + 10 * cplx)
    a = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    if kind == "cancelling":  # nearly nilpotent: |A^4| far below |A|^4
        a = np.triu(a, 1) + 1e-6 * a
    ld = np.clongdouble if cplx else np.longdouble
    al = a.astype(ld)
    a2l = al @ al
    a4l = a2l @ a2l
    a6l = a2l @ a4l
    n4_exact, n6_exact = norm1(a4l), norm1(a6l)
    for mul in (np.matmul, kloop):
        a2 = mul(a, a)
        a4 = mul(a2, a2)
        a6 = mul(a2, a4)
        p4, p6 = norm1(a4), norm1(a6)
        w4, w6 = widths(n, norm1(a), norm1(a2), p4, p6)
        # Each evaluation lies within half the width of the exact norm, so
        # the split value (a far smaller error) and the reference's FP64
        # value lie within the width of each other.
        assert abs(float(n4_exact) - p4) <= 0.5 * w4
        assert abs(float(n6_exact) - p6) <= 0.5 * w6
