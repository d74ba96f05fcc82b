"""The autotuner (tns_set_autotune): launch shapes chosen by timing both on a
size class's first launch. The shapes give identical results, so every
product and every exponential must be bit-identical with it on and off, and a
size class is timed once."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def tuned(ws):
    ws.set_autotune(True)
    try:
        yield ws
    finally:
        ws.set_autotune(False)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n", [96, 700])
def test_dmma_products_unchanged(tuned, orc, cplx, n):
    rng = np.random.default_rng(n + cplx)
    a = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    b = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    tuned.reset_stats()
    first = tuned.multiply(a, b)
    trials = tuned.stats()["autotune_trials"]
    second = tuned.multiply(a, b)
    assert tuned.stats()["autotune_trials"] == trials  # the class is known now
    ref = orc.gemm(a, b) if hasattr(orc, "gemm") else None
    assert np.array_equal(first, second)
    if ref is not None:
        assert np.array_equal(first, ref)


@pytest.mark.parametrize("cplx", [False, True])
def test_split_products_unchanged(ws, cplx):
    rng = np.random.default_rng(7 + cplx)
    n = 640
    a = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    b = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    plain = ws.multiply_split(a, b, 20)
    ws.set_autotune(True)
    try:
        ws.reset_stats()
        got = ws.multiply_split(a, b, 20)
        assert ws.stats()["autotune_trials"] >= 1
        again = ws.multiply_split(a, b, 20)
    finally:
        ws.set_autotune(False)
    assert np.array_equal(got, plain) and np.array_equal(again, plain)


@pytest.mark.parametrize("moduli", [0, 20])
def test_batched_expm_unchanged(ws, moduli):
    rng = np.random.default_rng(11)
    mats = []
    for n in (70, 150, 300, 90):
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        mats.append(np.asfortranarray(a * (rng.uniform(0.5, 200.0) / np.abs(a).sum(axis=0).max())))
    ws.set_split_moduli(moduli)
    try:
        ref = ws.expm_batched(mats)
        ws.set_autotune(True)
        try:
            got = ws.expm_batched(mats)
            got2 = ws.expm_batched(mats)
        finally:
            ws.set_autotune(False)
    finally:
        ws.set_split_moduli(0)
    for r, g, g2 in zip(ref, got, got2):
        assert np.array_equal(r, g) and np.array_equal(r, g2)
