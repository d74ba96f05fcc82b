"""Pins the CPU oracle before it is trusted as the GPU library's checker.

The reference (managed .NET) cannot run on these machines, so the oracle is
pinned by the reference's own known-answer tests, ported here with the same
seeded inputs (System.Random restated), and by independent cross-checks with
LAPACK / scipy. Runs on CPU only.
"""
import math

import numpy as np
import pytest
import scipy.linalg as sl

from conftest import net_matrix, random_with_one_norm, rel1


# ---- Pade coefficients (MatrixExponentialTests.cs:57-115) --------------------

PADE = {
    3: [120, 60, 12, 1],
    5: [30240, 15120, 3360, 420, 30, 1],
    7: [17297280, 8648640, 1995840, 277200, 25200, 1512, 56, 1],
    9: [17643225600, 8821612800, 2075673600, 302702400, 30270240, 2162160, 110880, 3960, 90, 1],
    13: [64764752532480000, 32382376266240000, 7771770303897600, 1187353796428800, 129060195264000,
         10559470521600, 670442572800, 33522128640, 1323241920, 40840800, 960960, 16380, 182, 1],
}
BACKWARD = {3: 100800.0, 5: 10059033600.0, 7: 4487938430976000.0, 9: 5914384781877411840000.0,
            13: 113250775606021113483283660800000000.0}


def _shipped_tables():
    """The tables as the product and the oracle ship them (parsed from source)."""
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for path in ("csharp_linearalgebra_b200/csrc/pade.h", "oracle/tensile_oracle.cpp"):
        src = open(os.path.join(root, path)).read()
        tabs = {}
        for m in (3, 5, 7, 9, 13):
            mm = re.search(r"(?:k)?Pade%d\[\]\s*=\s*\{([^}]*)\}" % m, src)
            tabs[m] = [float(x.strip()) for x in mm.group(1).replace("\n", " ").split(",") if x.strip()]
        out[path] = tabs
    return out


@pytest.mark.parametrize("m", [3, 5, 7, 9, 13])
def test_pade_coefficients_match_closed_form(m):
    for tabs in _shipped_tables().values():
        shipped = tabs[m]
        assert len(shipped) == m + 1
        for j in range(m + 1):
            derived = math.factorial(2 * m - j) // (math.factorial(j) * math.factorial(m - j))
            assert float(derived) == shipped[j]
            assert int(shipped[j]) == derived  # exact in a double


@pytest.mark.parametrize("m", [3, 5, 7, 9, 13])
def test_backward_error_coefficients(m):
    derived = float(math.comb(2 * m, m) * math.factorial(2 * m + 1))
    assert abs(derived - BACKWARD[m]) <= 1e-15 * derived


# ---- closed forms (MatrixExponentialTests.cs:119-214) -----------------------

def test_exponential_of_zero_is_identity(orc):
    e, info = orc.expm(np.zeros((6, 6)))
    assert np.array_equal(e, np.eye(6))


@pytest.mark.parametrize("scale", [1e-4, 0.5, 3.0, 20.0])
def test_exponential_of_diagonal(orc, scale):
    d = np.array([0.0, 1.0, -1.0, 0.25, -2.0]) * scale
    e, _ = orc.expm(np.diag(d))
    for i in range(5):
        for j in range(5):
            exp_ = math.exp(d[i]) if i == j else 0.0
            assert abs(e[i, j] - exp_) <= 1e-11 * max(abs(exp_), 1.0)


def test_nilpotent_block(orc):
    e, _ = orc.expm(np.array([[0.0, 1.0], [0.0, 0.0]]))
    assert np.allclose(e, [[1.0, 1.0], [0.0, 1.0]], atol=1e-15, rtol=0)


@pytest.mark.parametrize("t", [0.001, 0.3, 1.0, 7.5])
def test_rotation(orc, t):
    e, _ = orc.expm(np.array([[0.0, -t], [t, 0.0]]))
    assert np.allclose(e, [[math.cos(t), -math.sin(t)], [math.sin(t), math.cos(t)]], atol=1e-12, rtol=0)


def test_jordan_block(orc):
    lam = 1.75
    e, _ = orc.expm(np.array([[lam, 1.0], [0.0, lam]]))
    ex = math.exp(lam)
    assert np.allclose(e, [[ex, ex], [0.0, ex]], atol=1e-11 * ex, rtol=0)


# ---- branch coverage on the reference's own seeded inputs --------------------

def test_every_pade_degree_is_reached(orc):
    """MatrixExponentialTests.EveryPadeDegreeIsReached: RandomWithOneNorm(8, norm,
    seed 77 + (int)(norm*10)) must select degrees {3, 5, 7, 9, 13}."""
    seen = set()
    for norm in [0.001, 0.05, 0.4, 1.2, 6.0, 40.0]:
        a = random_with_one_norm(orc, 8, norm, 77 + int(norm * 10))
        _, info = orc.expm(a)
        seen.add(info["degree"])
    assert sorted(seen) == [3, 5, 7, 9, 13]


def test_scaling_only_when_norm_demands(orc):
    small = random_with_one_norm(orc, 6, 0.05, 11)
    large = random_with_one_norm(orc, 6, 500.0, 12)
    assert orc.expm(small)[1]["squarings"] == 0
    assert orc.expm(large)[1]["squarings"] >= 6


@pytest.mark.parametrize("n,target", [(8, 0.001), (8, 0.05), (8, 0.4), (8, 1.2), (8, 6.0), (8, 40.0),
                                      (17, 0.01), (17, 0.8), (17, 12.0), (32, 2.5), (32, 30.0)])
def test_expm_agrees_with_scipy(orc, n, target):
    a = random_with_one_norm(orc, n, target, n * 1000 + int(target * 10))
    e, _ = orc.expm(a)
    assert rel1(e, sl.expm(a)) <= 1e-11


def test_complex_expm_of_real_input_takes_real_branch(orc):
    """ComplexExponentialTests: a real matrix as complex takes the real path's
    (degree, s) exactly and gives an exactly real result."""
    for norm, seed in [(0.01, 3), (0.3, 4), (2.0, 5), (50.0, 6)]:
        a = random_with_one_norm(orc, 12, norm, seed)
        er, ir = orc.expm(a)
        ez, iz = orc.expm(a.astype(np.complex128))
        assert (ir["degree"], ir["squarings"]) == (iz["degree"], iz["squarings"])
        assert np.all(ez.imag == 0.0)
        assert rel1(ez.real, er) <= 1e-14


@pytest.mark.parametrize("n,nrm", [(40, 0.01), (60, 1.0), (90, 100.0)])
def test_complex_expm_agrees_with_scipy(orc, n, nrm):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    a *= nrm / np.abs(a).sum(axis=0).max()
    e, _ = orc.expm(a)
    assert rel1(e, sl.expm(a)) <= 1e-12


# ---- LU: pivots and known answers --------------------------------------------

@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (5, 5), (17, 17), (33, 33), (65, 65), (100, 100),
                                 (129, 129), (200, 73), (73, 200)])
@pytest.mark.parametrize("nb", [8, 32, 64])
def test_real_lu_pivots_match_lapack(orc, m, n, nb):
    a = net_matrix(orc, m, n, seed=m * 31 + n)
    f, piv, info = orc.getrf(a, nb)
    lu, piv2 = sl.lu_factor(a)
    k = min(m, n)
    assert np.array_equal(piv, piv2[:k])
    p, l, u = sl.lu(a)
    # residual ||PA - LU|| / ||A|| (LuTests.cs:27-61)
    L = np.tril(f[:, :k], -1) + np.eye(m, k)
    U = np.triu(f[:k, :])
    pa = a.copy()
    for i, q in enumerate(piv):
        pa[[i, q]] = pa[[q, i]]
    assert np.linalg.norm(pa - L @ U) / np.linalg.norm(a) < 1e-12


@pytest.mark.parametrize("n", [3, 16, 64, 130])
def test_complex_lu_pivots_match_lapack(orc, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    _, piv, _ = orc.getrf(a)
    _, piv2 = sl.lu_factor(a)
    assert np.array_equal(piv, piv2)


def test_pivot_maximises_sum_of_absolute_parts(orc):
    a = np.array([[3.0, 1.0], [2.0 + 2.0j, 1.0]])
    assert orc.getrf(a)[1][0] == 1


def test_pivot_ties_go_to_lowest_index(orc):
    a = np.array([[1.0 + 1.0j, 1.0], [-2.0, 2.0], [0.5 - 1.5j, 3.0]])
    assert orc.getrf(a)[1][0] == 0


def test_exact_zero_pivot_is_reported(orc):
    a = net_matrix(orc, 16, 16, 12)
    a += 16 * np.eye(16)
    a[:, 5] = 0.0
    f, piv, info = orc.getrf(a, 4)
    assert info["singular_column"] == 5
    with pytest.raises(ZeroDivisionError):
        orc.getrs(f, piv, np.ones(16), info["singular_column"])


# ---- normest1 invariants (NormEstimateTests.cs:33-160) -----------------------

@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 16, 17, 40, 64])
def test_full_width_probe_is_exact(orc, n):
    for trial in range(5):
        a = net_matrix(orc, n, n, n * 10 + trial)
        truth = orc.norm1(a)
        est, _, _ = orc.normest_power(a, 1, t=n)
        assert abs(est - truth) <= 1e-12 * truth


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 16, 17, 40, 64])
def test_nonnegative_is_exact_and_never_exceeds(orc, n):
    for trial in range(5):
        a = np.abs(net_matrix(orc, n, n, n * 20 + trial))
        truth = orc.norm1(a)
        est, it, prods = orc.normest_power(a, 1)
        assert abs(est - truth) <= 1e-12 * truth
        r = net_matrix(orc, n, n, n * 30 + trial)
        est_r, _, _ = orc.normest_power(r, 1)
        assert est_r <= orc.norm1(r) * (1 + 1e-12)


@pytest.mark.parametrize("n,t", [(1, 1), (6, 1), (25, 1), (25, 2), (60, 2), (60, 4)])
def test_complex_estimator_equals_real_on_real_input(orc, n, t):
    """ComplexNormEstimateTests.cs:103-122: on a real matrix (RandomReal, seeds
    0..7) the complex estimator equals the real one down to the iteration and
    product counts."""
    for seed in range(8):
        a = net_matrix(orc, n, n, seed, kind="unit")
        r = orc.normest_power(a, 1, t=t)
        z = orc.normest_power(a.astype(np.complex128), 1, t=t)
        assert r == z


def test_rcond_brackets_exact(orc):
    for n, seed in [(10, 1), (40, 2), (100, 3)]:
        a = net_matrix(orc, n, n, seed)
        f, piv, info = orc.getrf(a)
        exact = 1.0 / (np.linalg.norm(a, 1) * np.linalg.norm(np.linalg.inv(a), 1))
        r = orc.gecon(f, piv, -1, orc.norm1(a))
        assert r >= exact * (1 - 1e-10) and r <= 3 * exact


# ---- expmv (MatrixExponentialActionTests.cs) ----------------------------------

def test_expmv_zero_operator(orc):
    b = np.arange(1.0, 6.0).reshape(5, 1)
    y, info = orc.expmv(np.zeros((5, 5)), b, 1.0)
    assert (info["degree"], info["scaling"], info["applications"]) == (0, 1, 0)
    assert np.array_equal(y, b)


@pytest.mark.parametrize("t", [0.0, 0.5, -1.25, 3.0])
def test_expmv_matches_expm_times_b(orc, t):
    a = random_with_one_norm(orc, 20, 4.0, 5)
    b = net_matrix(orc, 20, 3, 6)
    y, _ = orc.expmv(a, b, t)
    ref = sl.expm(t * a) @ b
    assert rel1(y, ref) <= 1e-10


def test_expmv_diagonal(orc):
    d = np.array([-1.0, 0.0, 0.5, 2.0])
    y, _ = orc.expmv(np.diag(d), np.ones((4, 1)), 1.5)
    assert np.allclose(y[:, 0], np.exp(1.5 * d), rtol=1e-13, atol=0)


def test_expmv_complex_matches_scipy(orc):
    rng = np.random.default_rng(7)
    n = 48
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / n ** 0.5 * 3.0
    b = rng.standard_normal((n, 4)) + 0j
    y, info = orc.expmv(a, b, 0.5)
    assert rel1(y, sl.expm(0.5 * a) @ b) <= 1e-10


# ---- GEMM blocking semantics -------------------------------------------------

@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (1, 1, 64), (8, 6, 4), (17, 9, 5), (65, 63, 66),
                                   (100, 37, 129), (129, 130, 2), (300, 300, 400)])
def test_gemm_matches_numpy(orc, m, n, k):
    a = net_matrix(orc, m, k, 1)
    b = net_matrix(orc, k, n, 2)
    c = orc.gemm(a, b)
    assert np.linalg.norm(c - a @ b) <= 1e-13 * max(np.linalg.norm(a @ b), 1e-300)


def test_gemm_beta_zero_overwrites_nan(orc):
    a = np.ones((4, 3))
    b = np.ones((3, 5))
    c = np.full((4, 5), np.nan)
    assert np.array_equal(orc.gemm(a, b, c, 1.0, 0.0), np.full((4, 5), 3.0))


def test_gemm_is_thread_count_invariant(orc):
    a = net_matrix(orc, 300, 300, 3)
    b = net_matrix(orc, 300, 300, 4)
    orc.set_threads(1)
    c1 = orc.gemm(a, b)
    orc.set_threads(0)
    c2 = orc.gemm(a, b)
    assert np.array_equal(c1, c2)


@pytest.mark.parametrize("norm,t", [(0.05, 1.0), (3.0, 0.5), (40.0, 1.0), (40.0, -1.0)])
def test_matrix_free_expmv_oracle(orc, norm, t):
    """The oracle's matrix-free Expmv (mu = 0, crude bound, no estimator;
    MatrixExponentialAction.cs:203-230) against scipy's expm(tA) B."""
    import scipy.linalg
    rng = np.random.default_rng(int(norm * 10))
    a = rng.standard_normal((50, 50))
    a *= norm / np.abs(a).sum(axis=0).max()
    b = rng.standard_normal((50, 4))
    r, info = orc.expmv_bound(a, b, t, np.abs(a).sum(axis=0).max())
    ref = scipy.linalg.expm(t * a) @ b
    assert np.abs(r - ref).sum(axis=0).max() / max(np.abs(ref).sum(axis=0).max(), 1.0) <= 1e-12
    assert info["degree"] > 0 and info["scaling"] >= 1
