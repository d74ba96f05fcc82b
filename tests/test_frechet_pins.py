"""The oracle's way to the Frechet derivative of exp -- the upper right block
of Expm([[A, E], [0, A]]), the reference's own Expm on the block matrix
(src/Tensile/MatrixExponential.cs:181-270) -- pinned on the CPU against
closed forms:
  - diagonal A: L(A, E)_ij = E_ij (e^a_i - e^a_j) / (a_i - a_j)
    (E_ii e^a_i on the diagonal), the divided differences of exp;
  - E = A: L(A, A) = A e^A (A commutes with itself).
"""
import math

import numpy as np
import pytest


def block_frechet(orc, a, e):
    n = a.shape[0]
    blk = np.zeros((2 * n, 2 * n), dtype=np.result_type(a, e), order="F")
    blk[:n, :n] = a
    blk[:n, n:] = e
    blk[n:, n:] = a
    r, _ = orc.expm(blk)
    return r[:n, :n], r[:n, n:]


def rel(x, y):
    return np.abs(x - y).sum(axis=0).max() / np.abs(y).sum(axis=0).max()


@pytest.mark.parametrize("spread", [0.01, 1.0, 8.0])
def test_block_derivative_of_diagonal(orc, spread):
    rng = np.random.default_rng(4)
    d = rng.uniform(-spread, spread, 12)
    e = rng.standard_normal((12, 12))
    _, l = block_frechet(orc, np.diag(d), e)
    ed = np.exp(d)
    dd = np.empty((12, 12))
    for i in range(12):
        for j in range(12):
            dd[i, j] = ed[i] if d[i] == d[j] else (ed[i] - ed[j]) / (d[i] - d[j])
    assert rel(l, e * dd) <= 1e-12


def test_block_derivative_in_own_direction(orc):
    rng = np.random.default_rng(5)
    a = rng.standard_normal((15, 15)) + 1j * rng.standard_normal((15, 15))
    a *= 2.0 / np.abs(a).sum(axis=0).max()
    x, l = block_frechet(orc, a, a)
    ref, _ = orc.expm(a)
    assert rel(x, ref) <= 1e-13
    assert rel(l, a @ ref) <= 1e-12
