"""LU with partial pivoting, solves and rcond on the GPU against the oracle.
Pivot sequences must match bit for bit."""
import numpy as np
import pytest

from conftest import net_matrix, relfro

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 2), (5, 5), (17, 17), (32, 32), (33, 33), (64, 64), (65, 65), (100, 100),
          (129, 129), (200, 73), (73, 200), (129, 64), (64, 129), (512, 512)]


@pytest.mark.parametrize("m,n", SHAPES)
@pytest.mark.parametrize("nb", [0, 32, 64])
def test_real_lu_matches_oracle(ws, orc, m, n, nb):
    a = net_matrix(orc, m, n, seed=m * 7 + n) if m * n <= 40000 else \
        np.random.default_rng(m).uniform(-0.5, 0.5, (m, n))
    lu = ws.factor_lu(a, nb)
    f, piv, info = orc.getrf(a, nb)
    assert np.array_equal(lu.pivots, piv)
    assert lu.singular_column == info["singular_column"] == -1
    assert relfro(lu.factors, f) < 1e-12
    assert np.array_equal(lu.factors, f)  # bit for bit
    assert lu.smallest_pivot == pytest.approx(info["smallest_pivot"], rel=1e-12)
    assert lu.largest_pivot == pytest.approx(info["largest_pivot"], rel=1e-12)


@pytest.mark.parametrize("m,n", [(1, 1), (3, 3), (17, 17), (64, 64), (65, 65), (100, 37), (37, 100), (300, 300)])
def test_complex_lu_matches_oracle(ws, orc, m, n):
    rng = np.random.default_rng(m * 100 + n)
    a = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    lu = ws.factor_lu(a)
    f, piv, info = orc.getrf(a)
    assert np.array_equal(lu.pivots, piv)
    assert relfro(lu.factors, f) < 1e-12
    assert np.array_equal(lu.factors, f)  # bit for bit


@pytest.mark.parametrize("m,n,cplx", [(2048, 2048, False), (3000, 200, False), (1600, 1600, True)])
def test_tall_panels_match_oracle(ws, orc, m, n, cplx):
    """Panels of 1536 rows or more run on every SM (one CTA per slab of rows,
    a grid barrier per column); factors and pivots stay bit-identical."""
    rng = np.random.default_rng(m + n)
    a = rng.uniform(-0.5, 0.5, (m, n)) + (1j * rng.uniform(-0.5, 0.5, (m, n)) if cplx else 0)
    lu = ws.factor_lu(a)
    f, piv, info = orc.getrf(a)
    assert np.array_equal(lu.pivots, piv)
    assert np.array_equal(lu.factors, f)  # bit for bit


def test_pivot_maximises_sum_of_absolute_parts(ws):
    a = np.array([[3.0, 1.0], [2.0 + 2.0j, 1.0]])
    assert ws.factor_lu(a).pivots[0] == 1


def test_pivot_ties_go_to_lowest_index(ws):
    a = np.array([[1.0 + 1.0j, 1.0], [-2.0, 2.0], [0.5 - 1.5j, 3.0]])
    assert ws.factor_lu(a).pivots[0] == 0


def test_exact_zero_pivot_is_reported(ws, orc):
    from csharp_linearalgebra_b200 import SingularMatrixError
    a = net_matrix(orc, 16, 16, 12) + 16 * np.eye(16)
    a[:, 5] = 0.0
    lu = ws.factor_lu(a, 16)
    assert lu.is_singular and lu.singular_column == 5
    with pytest.raises(SingularMatrixError):
        lu.solve(np.ones(16))
    with pytest.raises(SingularMatrixError):
        lu.solve_adjoint(np.ones(16))


@pytest.mark.parametrize("n,nrhs", [(1, 1), (17, 3), (100, 8), (129, 70), (512, 8), (300, 300)])
def test_solves_match_oracle(ws, orc, n, nrhs):
    rng = np.random.default_rng(n + nrhs)
    a = rng.uniform(-0.5, 0.5, (n, n))
    b = rng.uniform(-0.5, 0.5, (n, nrhs))
    lu = ws.factor_lu(a)
    x = lu.solve(b)
    xt = lu.solve_adjoint(b)
    f, piv, info = orc.getrf(a)
    assert relfro(x, orc.getrs(f, piv, b)) < 1e-12
    assert relfro(xt, orc.getrs(f, piv, b, adjoint=True)) < 1e-12
    # both solves keep the reference's order of operations: the same bits
    assert np.array_equal(x, orc.getrs(f, piv, b))
    assert np.array_equal(xt, orc.getrs(f, piv, b, adjoint=True))
    # backward error ||Ax - b||_inf / (||A||_inf ||x||_inf) (LuTests.cs:69-105)
    assert np.abs(a @ x - b).max() / (np.abs(a).sum(axis=1).max() * np.abs(x).max()) < 1e-12


@pytest.mark.parametrize("n,nrhs", [(5, 1), (64, 8), (200, 200)])
def test_complex_solves_match_oracle(ws, orc, n, nrhs):
    rng = np.random.default_rng(3 * n + nrhs)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal((n, nrhs)) + 1j * rng.standard_normal((n, nrhs))
    lu = ws.factor_lu(a)
    f, piv, _ = orc.getrf(a)
    assert relfro(lu.solve(b), orc.getrs(f, piv, b)) < 1e-12
    assert relfro(lu.solve_adjoint(b), orc.getrs(f, piv, b, adjoint=True)) < 1e-12
    assert np.array_equal(lu.solve(b), orc.getrs(f, piv, b))
    assert np.array_equal(lu.solve_adjoint(b), orc.getrs(f, piv, b, adjoint=True))
    x = lu.solve(b)
    # complex solve backward error (ComplexLuTests.cs:126-133)
    assert np.abs(a @ x - b).max() / (np.abs(a).sum(axis=1).max() * np.abs(x).max()) < 1e-14 * n


@pytest.mark.parametrize("n", [10, 64, 200])
@pytest.mark.parametrize("cplx", [False, True])
def test_rcond_matches_oracle(ws, orc, n, cplx):
    rng = np.random.default_rng(n)
    a = rng.uniform(-0.5, 0.5, (n, n))
    if cplx:
        a = a + 1j * rng.uniform(-0.5, 0.5, (n, n))
    lu = ws.factor_lu(a)
    f, piv, info = orc.getrf(a)
    r = lu.reciprocal_condition()
    ro = orc.gecon(f, piv, -1, orc.norm1(a))
    # every solve the estimator probes with is the reference's bit for bit
    # (adjoint ones included), so the estimate is the oracle's exactly
    assert r == ro
    exact = 1.0 / (np.linalg.norm(a, 1) * np.linalg.norm(np.linalg.inv(a), 1))
    assert exact * (1 - 1e-10) <= r <= 3 * exact


@pytest.mark.parametrize("n,cplx", [(512, False), (512, True), (1200, True), (3000, False)])
def test_rcond_and_adjoint_solves_at_larger_orders(ws, orc, n, cplx):
    """The transposed and adjoint solves stage the factor's columns through
    shared memory up to n = 3200 (real) and 1280 (complex), and complex solves
    of up to 16 right-hand sides run in one launch up to n = 1536; the
    estimate and the solves stay the oracle's bit for bit there, odd
    right-hand-side counts included."""
    rng = np.random.default_rng(n + 7)
    a = rng.uniform(-0.5, 0.5, (n, n))
    b = rng.uniform(-0.5, 0.5, (n, 3))
    if cplx:
        a = a + 1j * rng.uniform(-0.5, 0.5, (n, n))
        b = b + 1j * rng.uniform(-0.5, 0.5, (n, 3))
    lu = ws.factor_lu(a)
    f, piv, _ = orc.getrf(a)
    assert np.array_equal(lu.solve_adjoint(b), orc.getrs(f, piv, b, adjoint=True))
    assert np.array_equal(lu.solve(b), orc.getrs(f, piv, b))
    assert lu.reciprocal_condition() == orc.gecon(f, piv, -1, orc.norm1(a))


def test_determinant(ws):
    rng = np.random.default_rng(5)
    a = rng.standard_normal((12, 12))
    assert ws.factor_lu(a).determinant() == pytest.approx(np.linalg.det(a), rel=1e-12)


def test_lu_phase_timings(ws, orc):
    """LuPhaseTimings' counterpart: the four phases and the unattributed rest
    add up to the loop's total, one block step per panel; a one-panel LU
    records nothing; the factors are unchanged by the timing."""
    rng = np.random.default_rng(77)
    n = 512  # reference block size 32: 16 block steps
    a = rng.uniform(-0.5, 0.5, (n, n))
    ws.reset_stats()
    ws.set_lu_timing(True)
    try:
        lu = ws.factor_lu(a)
        t = ws.lu_timings()
        small = ws.factor_lu(rng.uniform(-0.5, 0.5, (20, 20)))  # one whole-matrix panel
        t2 = ws.lu_timings()
    finally:
        ws.set_lu_timing(False)
    f, piv, _ = orc.getrf(a)
    assert np.array_equal(lu.factors, f) and np.array_equal(lu.pivots, piv)
    assert t["factorizations"] == 1 and t["block_steps"] == 16
    phases = t["panel_ms"] + t["swaps_ms"] + t["triangular_ms"] + t["gemm_ms"]
    assert all(t[k] > 0 for k in ("panel_ms", "swaps_ms", "triangular_ms", "gemm_ms"))
    assert phases <= t["total_ms"] * 1.001 + 1e-3
    assert t["unattributed_ms"] == pytest.approx(max(0.0, t["total_ms"] - phases), abs=1e-9)
    assert t2 == t and small.rows == 20
    ws.reset_stats()
    assert ws.lu_timings()["total_ms"] == 0.0
