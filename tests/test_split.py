"""The split-precision product: the exact model's accuracy against the FP64
product (CPU), and the tcgen05 kernel plus its Chinese-remainder
reconstruction against the model (GPU)."""
import math

import numpy as np
import pytest

from split_model import MODULI, integer_bits, split_product


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


def test_moduli_are_pairwise_coprime_and_fit_8_bits():
    for i, p in enumerate(MODULI):
        assert 2 <= p <= 256
        for q in MODULI[:i]:
            assert math.gcd(p, q) == 1


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("nm", [14, 17, 20])
def test_model_accuracy(cplx, nm):
    """Entrywise error within K' 2^-t of the row scale times the column scale
    (the rounding of A and B to t-bit integers), plus the FP64 product's own
    rounding."""
    rng = np.random.default_rng(100 + nm)
    for m, k, n in [(40, 70, 30), (33, 130, 17)]:
        for scale in (False, True):
            a, b = _mats(rng, m, k, n, cplx, scale)
            ref = a @ b
            got, _ = split_product(a, b, nm)
            kk = 2 * k if cplx else k
            t, _ = integer_bits(nm, kk)
            ra = np.abs(a).max(axis=1)[:, None] * 2
            cb = np.abs(b).max(axis=0)[None, :] * 2
            bound = kk * 2.0 ** -t * ra * cb + 4 * k * 2.0 ** -53 * (np.abs(a) @ np.abs(b))
            assert np.all(np.abs(got - ref) <= bound)


def test_model_is_exact_on_small_integers():
    rng = np.random.default_rng(7)
    a = rng.integers(-50, 50, size=(9, 11)).astype(float)
    b = rng.integers(-50, 50, size=(11, 5)).astype(float)
    got, _ = split_product(a, b, 20)
    assert np.array_equal(got, a @ b)


def _check_kernel(ws, a, b, nm):
    got = ws.multiply_split(a, b, nm)
    ref, unit = split_product(a, b, nm)
    _, L = integer_bits(nm, 1)
    # reconstruction error below 2^(L - 95) units of the integer product, plus rounding
    tol = 4 * np.spacing(np.abs(ref)) + unit * 2.0 ** (L - 95)
    assert np.all(np.abs(got.real - ref.real) <= tol)
    if np.iscomplexobj(ref):
        assert np.all(np.abs(got.imag - ref.imag) <= tol)


@pytest.mark.gpu
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 5, 3), (128, 128, 64), (130, 257, 65), (200, 129, 150)])
def test_kernel_matches_model(ws, cplx, shape):
    m, k, n = shape
    rng = np.random.default_rng(m * 7 + k * 3 + n)
    a, b = _mats(rng, m, k, n, cplx)
    for nm in (20, 14):
        _check_kernel(ws, a, b, nm)


@pytest.mark.gpu
def test_kernel_scaled_rows_and_zeros(ws):
    rng = np.random.default_rng(5)
    a, b = _mats(rng, 150, 200, 140, True, scale_rows=True)
    a[3, :] = 0
    b[:, 7] = 0
    _check_kernel(ws, a, b, 20)
    got = ws.multiply_split(a, b, 20)
    assert np.all(got[3, :] == 0) and np.all(got[:, 7] == 0)


@pytest.mark.gpu
def test_kernel_accuracy_at_sweep_orders(ws):
    """Complex products of order 1024 (the sweep's largest): normwise within 1e-15."""
    rng = np.random.default_rng(11)
    n = 1024
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(n)
    got = ws.multiply_split(np.asfortranarray(a), np.asfortranarray(a), 20)
    ref = a @ a
    assert np.abs(got - ref).sum(axis=0).max() / np.abs(ref).sum(axis=0).max() < 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("cplx,n", [(False, 2560), (True, 1600)])
def test_cta_pair_kernel_matches_one_cta_kernel(ws, cplx, n):
    """Products whose 256-column tiles fill the GPU run on CTA pairs (two
    CTAs sharing one M = 256 MMA); with 13 row strips (complex, n = 1600) the
    last strip runs on the one-CTA kernel. Each 128-row block of A multiplied
    alone runs the one-CTA kernel on the same integer images (row scales per
    row, column scales per column, the same depth), so every row of the full
    product must equal the block's bit for bit."""
    rng = np.random.default_rng(n)
    a, b = _mats(rng, n, n, n, cplx)
    full = ws.multiply_split(a, b, 17)
    for r0 in range(0, n, 128):
        block = ws.multiply_split(np.asfortranarray(a[r0:r0 + 128]), b, 17)
        assert np.array_equal(block, full[r0:r0 + 128]), f"rows {r0}.."
    ref = a @ b
    assert np.abs(full - ref).sum(axis=0).max() / np.abs(ref).sum(axis=0).max() < 1e-14
