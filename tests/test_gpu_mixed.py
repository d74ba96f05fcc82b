"""Precision form of the solve on the GPU, through the C ABI: a low-precision LU
(trailing updates on the split-precision product) refined in FP64.

Workload: A = U diag(sigma) V^T with U, V from the QR of Gaussian matrices and
sigma log-spaced so that kappa_2 is 1e2, 1e6 or 1e10; 64 right-hand sides
N(0,1); n = 512 and the configuration's n = 4096.

Checks:
  - the backward error max_j |b_j - A x_j|_inf / (|A|_inf |x_j|_inf + |b_j|_inf)
    reaches FP64 level (<= 1e-15) for every kappa;
  - against the FP64 solve in the reference's arithmetic (Lu.Factor +
    Lu.Solve, bit-identical on the GPU, test_gpu_lu.py), the forward difference
    is within 100 kappa u: two backward-stable solutions each sit about
    kappa u from the exact one;
  - the moduli chosen from the condition estimate grow with kappa;
  - the first route (random butterfly transforms, elimination without row
    interchanges, the order padded to a multiple of 4) is the one that runs on
    these matrices, at orders that need the padding too, real and complex;
  - when that route's refinement cannot reach an FP64 backward error (no
    refinement steps allowed), the solve runs again with partial pivoting and
    reports it; an all-zero matrix ends in TNS_E_SINGULAR through the same
    fallback.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

U = 2.0 ** -53


def conditioned(n, kappa, seed, cplx=False):
    rng = np.random.default_rng(seed)

    def orth():
        g = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
        q, _ = np.linalg.qr(g)
        return q

    s = np.logspace(0.0, -math.log10(kappa), n)
    a = (orth() * s) @ orth().conj().T
    b = rng.standard_normal((n, 64)) + (1j * rng.standard_normal((n, 64)) if cplx else 0)
    return np.asfortranarray(a), np.asfortranarray(b)


def rel(x, y):
    return np.abs(x - y).sum(axis=0).max() / np.abs(y).sum(axis=0).max()


@pytest.mark.parametrize("n", [512, 4096])
@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_mixed_solve_configuration(ws, n, kappa):
    a, b = conditioned(n, kappa, seed=int(math.log10(kappa)) + n)
    x, info = ws.solve_mixed(a, b)
    x64 = ws.factor_lu(a).solve(b)
    fwd = rel(x, x64)
    print(f"n={n} kappa={kappa:.0e}: moduli {info['moduli']} factorizations {info['factorizations']} "
          f"steps {info['iterations']} backward error {info['backward_error']:.2e} "
          f"rcond {info['rcond']:.2e} vs FP64 solve {fwd:.2e}")
    assert info["backward_error"] <= 1e-15
    assert fwd <= max(1e-13, 100.0 * kappa * U)
    # 0 steps when the chosen precision already gives an FP64 backward error
    assert 0 <= info["iterations"] <= 10
    assert info["pivoting"] == 0


def test_moduli_follow_condition(ws):
    chosen = []
    for kappa in (1e2, 1e6, 1e10):
        a, b = conditioned(1024, kappa, seed=7)
        _, info = ws.solve_mixed(a, b)
        chosen.append(info["moduli"])
    assert chosen == sorted(chosen) and chosen[0] < chosen[2]


def test_fixed_moduli_and_complex(ws):
    a, b = conditioned(300, 1e4, seed=11, cplx=True)
    x, info = ws.solve_mixed(a, b, moduli=12)
    assert info["moduli"] == 12 and info["factorizations"] == 1
    assert info["backward_error"] <= 1e-15
    assert rel(x, ws.factor_lu(a).solve(b)) <= max(1e-13, 100.0 * 1e4 * U)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 63, 130, 1001])
@pytest.mark.parametrize("cplx", [False, True])
def test_butterfly_route_padded_orders(ws, n, cplx):
    a, b = conditioned(n, 1e3, seed=n, cplx=cplx)
    b = b[:, :7]
    x, info = ws.solve_mixed(a, b)
    assert info["pivoting"] == 0 and info["factorizations"] in (1, 2)
    assert info["backward_error"] <= 1e-15
    assert rel(x, np.linalg.solve(a, b)) <= max(1e-13, 100.0 * 1e3 * U)
    # the condition estimate (normest1 of A^-1 through the transformed
    # factors) is a lower bound of kappa_1, rarely far below it
    k1 = np.linalg.cond(a, 1)
    assert k1 / 30.0 <= 1.0 / info["rcond"] <= k1 * 1.01


def test_fallback_to_partial_pivoting(ws):
    # No refinement step allowed: 8 moduli (26-bit images) cannot give an
    # FP64 backward error alone, so the butterfly route declines and the
    # pivoting route answers (with the same limit).
    a, b = conditioned(1024, 1e2, seed=3)
    x, info = ws.solve_mixed(a, b, moduli=8, max_iter=0)
    assert info["pivoting"] == 1 and info["factorizations"] == 2 and info["iterations"] == 0
    assert info["backward_error"] > 8 * 2.0 ** -53
    assert rel(x, np.linalg.solve(a, b)) <= 1e-4


def test_zero_matrix_is_singular(ws):
    from csharp_linearalgebra_b200 import SingularMatrixError
    a = np.zeros((96, 96), order="F")
    b = np.ones((96, 2), order="F")
    with pytest.raises(SingularMatrixError) as e:
        ws.solve_mixed(a, b, moduli=8)
    assert "zero pivot" in str(e.value)
