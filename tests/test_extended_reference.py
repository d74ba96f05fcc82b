"""The extended-precision exponential (oracle/extended.py) that the GPU
forms' accuracy is measured against: it must be far more accurate than FP64
before it can tell two FP64 results apart."""
import math

import numpy as np
import pytest
import scipy.linalg

from oracle.extended import expm_extended, has_extended_precision, rel1_extended

pytestmark = pytest.mark.skipif(not has_extended_precision(), reason="long double is not the 80-bit format")


def sweep_matrix(rng, n, w):
    g = rng.standard_normal((n, n)) / math.sqrt(n)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    d = np.exp(rng.uniform(math.log(1e-3), 0.0, n))
    c = (q.T * d) @ q
    c = 0.5 * (c + c.T)
    return np.asfortranarray(-(g + 1j * w * c))


def test_closed_forms_in_long_double():
    t = np.longdouble(0.3)  # the double 0.3, which the input holds
    e = expm_extended(np.array([[0.0, -0.3], [0.3, 0.0]], dtype=np.longdouble).astype(np.float64))
    r = np.array([[np.cos(t), -np.sin(t)], [np.sin(t), np.cos(t)]])
    assert float(np.abs(e - r).max()) < 1e-18
    lam = 1.75
    e = expm_extended(np.array([[lam, 1.0], [0.0, lam]]))
    el = np.exp(np.longdouble(lam))
    assert float(abs(e[0, 0] - el) / el) < 1e-18 and float(abs(e[0, 1] - el) / el) < 1e-18


def test_agrees_with_scipy_on_a_well_conditioned_matrix():
    rng = np.random.default_rng(1)
    a = (rng.standard_normal((40, 40)) + 1j * rng.standard_normal((40, 40))) / 8.0
    assert rel1_extended(scipy.linalg.expm(a), expm_extended(a)) < 1e-14


@pytest.mark.parametrize("w", [1e2, 1e4, 1e6])
def test_is_far_inside_the_fp64_floor(w, orc):
    """Two long double evaluations with different scalings (s and s + 1
    squarings, different Taylor arguments) agree far more closely than the
    FP64 oracle's result agrees with either: the extended result's own error
    is negligible at the FP64 scale."""
    rng = np.random.default_rng(int(w))
    a = sweep_matrix(rng, 48, w)
    t1 = expm_extended(a)
    t2 = expm_extended(a, target=1.0)
    ref, info = orc.expm(a)
    self_diff = rel1_extended(t2, t1)
    fp64 = rel1_extended(ref, t1)
    assert self_diff < 0.01 * fp64 + 1e-17, (self_diff, fp64, info)
