"""normest1 over dense power operators on the GPU. The panel products keep the
reference's summation order and the bookkeeping is the reference's, so the
estimate, iteration count and product count must equal the oracle's exactly."""
import numpy as np
import pytest

from conftest import net_matrix

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 2, 5, 17, 64, 100, 257])
@pytest.mark.parametrize("power", [1, 2, 8, 10])
def test_real_power_estimate_is_bit_exact(ws, orc, n, power):
    a = net_matrix(orc, n, n, seed=n + 13 * power) if n <= 100 else \
        np.random.default_rng(n).uniform(-0.5, 0.5, (n, n))
    r = ws.estimate_power_norm(a, power)
    o = orc.normest_power(a, power)
    assert (r.value, r.iterations, r.products) == o


@pytest.mark.parametrize("n", [1, 3, 16, 60, 130])
@pytest.mark.parametrize("power", [1, 8, 10])
def test_complex_power_estimate_is_bit_exact(ws, orc, n, power):
    rng = np.random.default_rng(n * power)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    r = ws.estimate_power_norm(a, power)
    o = orc.normest_power(a, power)
    assert (r.value, r.iterations, r.products) == o


@pytest.mark.parametrize("t", [1, 2, 4, 7])
def test_probe_widths(ws, orc, t):
    a = net_matrix(orc, 40, 40, 77)
    r = ws.estimate_power_norm(a, 3, columns=t)
    assert (r.value, r.iterations, r.products) == orc.normest_power(a, 3, t=t)


def test_full_width_probe_is_exact(ws, orc):
    for n in (3, 8, 17):
        a = net_matrix(orc, n, n, n * 10)
        assert ws.estimate_power_norm(a, 1, columns=n).value == pytest.approx(orc.norm1(a), rel=1e-12)
