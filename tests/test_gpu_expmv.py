"""Expmv on the GPU against the oracle: (m, s) must match exactly, and since
the fused Taylor kernel keeps the reference's order of operations, so must the
application and early-exit counts and the result, bit for bit (1e-12
normwise is the stated bar)."""
import math

import numpy as np
import pytest

from conftest import net_matrix, random_with_one_norm, rel1

pytestmark = pytest.mark.gpu


def check(ws, orc, a, b, t, tol=1e-12):
    from csharp_linearalgebra_b200 import ExpmvDiagnostics
    d = ExpmvDiagnostics()
    y = ws.expmv(a, b, t, d)
    ref, info = orc.expmv(a, b, t)
    assert (d.degree, d.scaling) == (info["degree"], info["scaling"])
    assert rel1(y, ref) <= tol, rel1(y, ref)
    assert (d.applications, d.early_exits) == (info["applications"], info["early_exits"])
    assert np.array_equal(y, ref)
    return d


@pytest.mark.parametrize("t", [0.0, 0.5, -1.25, 3.0])
def test_real_expmv(ws, orc, t):
    a = random_with_one_norm(orc, 20, 4.0, 5)
    b = net_matrix(orc, 20, 3, 6)
    check(ws, orc, a, b, t)


@pytest.mark.parametrize("n,norm,cols", [(16, 0.5, 1), (64, 20.0, 8), (130, 200.0, 8), (300, 50.0, 16)])
def test_complex_expmv(ws, orc, n, norm, cols):
    rng = np.random.default_rng(n + cols)
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2 * n)
    a *= norm / np.abs(a).sum(axis=0).max()
    b = rng.standard_normal((n, cols)) + 0j
    check(ws, orc, a, b, 0.5)


def test_zero_operator(ws):
    from csharp_linearalgebra_b200 import ExpmvDiagnostics
    d = ExpmvDiagnostics()
    b = np.arange(1.0, 6.0).reshape(5, 1)
    y = ws.expmv(np.zeros((5, 5)), b, 1.0, d)
    assert (d.degree, d.scaling, d.applications) == (0, 1, 0)
    assert np.array_equal(y, b)


def test_diagonal(ws):
    d = np.array([-1.0, 0.0, 0.5, 2.0])
    y = ws.expmv(np.diag(d), np.ones(4), 1.5)
    assert np.allclose(y, np.exp(1.5 * d), rtol=1e-13, atol=0)


def test_early_exit_fires(ws, orc):
    a = random_with_one_norm(orc, 30, 0.5, 9)
    b = net_matrix(orc, 30, 2, 10)
    d = check(ws, orc, a, b, 1.0)
    assert d.early_exits >= 1 and d.applications < d.degree * d.scaling
