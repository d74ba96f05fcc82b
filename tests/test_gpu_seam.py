"""The kernel seam's primitives through the C ABI (KernelEntry.cs:98-234):
the six triangular solves, the panel products and the exact norms, against
the oracle's restatements, bit for bit; the complex triangular solves and
dense operator of the generic path (BlockedLu.cs, LinearOperators.cs); and
the allocation ceiling (TensileLimits.MaxElements)."""
import numpy as np
import pytest

from conftest import net_matrix

pytestmark = pytest.mark.gpu

KINDS = ["upper", "upper_transposed", "lower", "lower_transposed", "lower_unit", "lower_unit_transposed"]


def triangle_operand(orc, n, seed):
    """A well-conditioned operand as the reference's TriangularTests build
    them: System.Random(seed) entries in [-0.5, 0.5) plus n on the diagonal."""
    return net_matrix(orc, n, n, seed) + n * np.eye(n)


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("m,n", [(1, 1), (7, 3), (33, 4), (64, 5), (130, 9), (300, 64)])
def test_real_triangular_solves(ws, orc, kind, m, n):
    a = triangle_operand(orc, m, 100 + m)
    b = net_matrix(orc, m, n, 200 + n)
    x = ws.solve_triangular(kind, a, b)
    assert np.array_equal(x, orc.trsolve(kind, a, b))


@pytest.mark.parametrize("kind", ["upper", "upper_transposed", "lower_unit", "lower_unit_transposed"])
@pytest.mark.parametrize("m,n", [(1, 1), (9, 2), (65, 3), (200, 17)])
def test_complex_triangular_solves(ws, orc, kind, m, n):
    rng = np.random.default_rng(m * 10 + n)
    a = rng.uniform(-0.5, 0.5, (m, m)) + 1j * rng.uniform(-0.5, 0.5, (m, m)) + m * np.eye(m)
    b = rng.uniform(-0.5, 0.5, (m, n)) + 1j * rng.uniform(-0.5, 0.5, (m, n))
    x = ws.solve_triangular(kind, a, b)
    assert np.array_equal(x, orc.trsolve(kind, a, b))


def test_triangular_shape_errors(ws):
    with pytest.raises(ValueError):
        ws.solve_triangular("upper", np.eye(3)[:, :2], np.ones((3, 1)))
    with pytest.raises(ValueError):
        ws.solve_triangular("upper", np.eye(3), np.ones((4, 1)))
    with pytest.raises(ValueError):
        ws.solve_triangular("lower", np.eye(3) + 0j, np.ones((3, 1)))  # no complex explicit-diagonal lower


@pytest.mark.parametrize("transposed", [False, True])
@pytest.mark.parametrize("n,t", [(1, 1), (5, 2), (64, 4), (129, 8), (300, 16), (257, 21)])
def test_panel_products(ws, orc, transposed, n, t):
    rng = np.random.default_rng(n + t)
    a = rng.uniform(-0.5, 0.5, (n, n))
    x = rng.uniform(-0.5, 0.5, (n, t))
    x[rng.uniform(size=x.shape) < 0.1] = 0.0  # zero entries are skipped, as the reference's axpy skips them
    assert np.array_equal(ws.multiply_panel(a, x, transposed), orc.panel(a, x, transposed))
    ac = a + 1j * rng.uniform(-0.5, 0.5, (n, n))
    xc = x + 1j * rng.uniform(-0.5, 0.5, (n, t))
    assert np.array_equal(ws.multiply_panel(ac, xc, transposed), orc.panel(ac, xc, transposed))


@pytest.mark.parametrize("m,n", [(1, 1), (3, 7), (64, 64), (130, 33), (500, 260)])
def test_norms_match_oracle(ws, orc, m, n):
    """Norms.One / Infinity / Frobenius (Norms.cs:11-66) and the complex
    one- and infinity-norms by Complex.Abs (ComplexKernels.cs:144-180)."""
    rng = np.random.default_rng(m * 7 + n)
    a = rng.standard_normal((m, n))
    assert ws.one_norm(a) == orc.norm1(a)
    assert ws.infinity_norm(a) == orc.norminf(a)
    assert ws.frobenius_norm(a) == pytest.approx(np.linalg.norm(a), rel=1e-14)
    z = a + 1j * rng.standard_normal((m, n))
    assert ws.one_norm(z) == orc.norm1(z)
    assert ws.infinity_norm(z) == orc.norminf(z)
    assert ws.frobenius_norm(z) == pytest.approx(np.linalg.norm(z), rel=1e-14)


def test_norms_of_empty_and_nan(ws):
    assert ws.one_norm(np.zeros((0, 3))) == 0.0
    assert ws.infinity_norm(np.zeros((4, 0))) == 0.0
    a = np.ones((5, 5))
    a[2, 3] = np.nan
    assert np.isnan(ws.one_norm(a)) and np.isnan(ws.infinity_norm(a))


def test_allocation_limit_is_enforced():
    """A request above TensileLimits.MaxElements is refused before any device
    allocation (TensileLimits.Check, TensileLimits.cs:59-65), with the
    reference's exception, and the workspace stays usable."""
    from csharp_linearalgebra_b200 import AllocationLimitError, Workspace
    with Workspace(0, max_elements=10_000) as ws:
        small = np.eye(50)
        assert np.array_equal(ws.multiply(small, small), small)  # 2500 elements each: allowed
        big = np.ones((101, 100))  # 10,100 elements
        with pytest.raises(AllocationLimitError):
            ws.multiply(big, np.ones((100, 2)))
        with pytest.raises(AllocationLimitError):
            ws.expm(np.eye(101))
        ws.set_max_elements(20_000)
        assert ws.multiply(big, np.ones((100, 2))).shape == (101, 2)
        assert np.array_equal(ws.multiply(small, small), small)
