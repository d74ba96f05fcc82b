"""The split-precision product: the numpy model's accuracy against the FP64
product (CPU), and the tcgen05 kernel against the model, bit for bit (GPU)."""
import math

import numpy as np
import pytest

from split_model import split_product


def _mats(rng, m, k, n, cplx, scale_rows=False):
    a = rng.standard_normal((m, k))
    b = rng.standard_normal((k, n))
    if cplx:
        a = a + 1j * rng.standard_normal((m, k))
        b = b + 1j * rng.standard_normal((k, n))
    if scale_rows:
        a *= np.exp(rng.uniform(-20, 20, size=(m, 1)))
        b *= np.exp(rng.uniform(-20, 20, size=(1, n)))
    return np.asfortranarray(a), np.asfortranarray(b)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("S", [6, 7, 8])
def test_model_accuracy(cplx, S):
    """Entrywise error within (S + 2) K 2^(-7 S) of the row scale times the
    column scale (the S - 1 dropped pairs of the next weight and the slices'
    residuals), plus the FP64 product's own rounding."""
    rng = np.random.default_rng(100 + S)
    for m, k, n in [(40, 70, 30), (97, 130, 65)]:
        for scale in (False, True):
            a, b = _mats(rng, m, k, n, cplx, scale)
            ref = a @ b
            got = split_product(a, b, S)
            ra = np.abs(a).max(axis=1)[:, None]
            cb = np.abs(b).max(axis=0)[None, :]
            bound = (S + 2.0) * k * 2.0 ** (-7 * S) * ra * cb + 4 * k * 2.0 ** -53 * (np.abs(a) @ np.abs(b))
            assert np.all(np.abs(got - ref) <= bound)


def test_model_is_exact_on_small_integers():
    rng = np.random.default_rng(7)
    a = rng.integers(-50, 50, size=(9, 11)).astype(float)
    b = rng.integers(-50, 50, size=(11, 5)).astype(float)
    assert np.array_equal(split_product(a, b, 8), a @ b)


@pytest.mark.gpu
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 5, 3), (128, 128, 64), (130, 257, 65), (300, 129, 257)])
def test_kernel_matches_model(ws, cplx, shape):
    m, k, n = shape
    rng = np.random.default_rng(m * 7 + k * 3 + n)
    a, b = _mats(rng, m, k, n, cplx)
    for S in (8, 6):
        got = ws.multiply_split(a, b, S)
        assert np.array_equal(got, split_product(a, b, S)), (shape, S)


@pytest.mark.gpu
def test_kernel_scaled_rows_and_zeros(ws):
    rng = np.random.default_rng(5)
    a, b = _mats(rng, 150, 200, 140, True, scale_rows=True)
    a[3, :] = 0
    b[:, 7] = 0
    got = ws.multiply_split(a, b, 8)
    assert np.array_equal(got, split_product(a, b, 8))
    assert np.all(got[3, :] == 0) and np.all(got[:, 7] == 0)


@pytest.mark.gpu
def test_kernel_accuracy_at_sweep_orders(ws):
    """Complex products of order 1024 (the sweep's largest): normwise within 1e-14."""
    rng = np.random.default_rng(11)
    n = 1024
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(n)
    got = ws.multiply_split(np.asfortranarray(a), np.asfortranarray(a), 8)
    ref = a @ a
    assert np.abs(got - ref).sum(axis=0).max() / np.abs(ref).sum(axis=0).max() < 1e-14
