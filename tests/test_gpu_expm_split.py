"""Expm with its products in the split-precision form (8-bit residues modulo
17 or 20 moduli on the tensor cores, Chinese-remainder reconstruction).

The degree and the squaring count are the reference's exactly: their inputs
(norms, A^2, A^4, A^6, normest1) stay in plain FP64.

Tolerance. The result is compared with the oracle (the reference's FP64
rounding) in the 1-norm. The bar is 1e-12, except where the problem itself
cannot be computed that closely by any arithmetic that is not the
reference's bit for bit. That level is measured per matrix as the floor: the
change of the plain FP64 result when the input is perturbed by about one
unit in the last place. The split result must lie within SPLIT_FLOOR_FACTOR
x the floor, and within 1e-12 whenever that is below it. The floor grows with the
squarings (about 2^s u): under 1e-13 up to s = 10, above 1e-12 from s = 15.
"""
import math

import numpy as np
import pytest

from conftest import rel1

pytestmark = pytest.mark.gpu

MODULI = 20
# The bar against the oracle, in units of the matrix's FP64 floor. The split
# form is as close to exp(A) itself as the reference is (within a factor 2,
# tests/test_gpu_expm_truth.py), and the reference's own distance to exp(A)
# is a few floors, so the two results can be several floors apart.
SPLIT_FLOOR_FACTOR = 6.0


@pytest.fixture(params=[17, 20])
def split_ws(ws, request):
    """The split form at the benchmark's 17 moduli and at 20."""
    global MODULI
    MODULI = request.param
    ws.set_split_moduli(MODULI)
    try:
        yield ws
    finally:
        ws.set_split_moduli(0)
        MODULI = 20
# The bar against the oracle, in units of the matrix's FP64 floor. The split
# form is as close to exp(A) itself as the reference is (within a factor 2,
# tests/test_gpu_expm_truth.py), and the reference's own distance to exp(A)
# is a few floors, so the two results can be several floors apart.
SPLIT_FLOOR_FACTOR = 6.0


def sweep_matrix(rng, n, w):
    g = rng.standard_normal((n, n)) / math.sqrt(n)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    d = np.exp(rng.uniform(math.log(1e-3), 0.0, n))
    c = (q.T * d) @ q
    c = 0.5 * (c + c.T)
    return np.asfortranarray(-(g + 1j * w * c))


def floor_of(ws, a, ref):
    """How far the plain FP64 result moves when A moves by about one ulp."""
    rng = np.random.default_rng(12345)
    pert = a * (1.0 + 2.0 ** -52 * rng.standard_normal(a.shape))
    ws.set_split_moduli(0)
    try:
        return rel1(ws.expm(np.asfortranarray(pert)), ref)
    finally:
        ws.set_split_moduli(MODULI)


def check(ws, a, e, d, ref, info):
    assert (d.degree, d.squarings) == (info["degree"], info["squarings"])
    bar = max(1e-12, SPLIT_FLOOR_FACTOR * floor_of(ws, a, ref))
    assert rel1(e, ref) <= bar, (rel1(e, ref), bar)


def test_frequency_sweep_split(split_ws, orc):
    rng = np.random.default_rng(21)
    mats = [sweep_matrix(rng, int(rng.integers(64, 200)), w) for w in np.logspace(2.0, 6.0, 7)]
    diags = []
    outs = split_ws.expm_batched(mats, diags)
    low_s = 0
    for a, e, d in zip(mats, outs, diags):
        ref, info = orc.expm(a)
        check(split_ws, a, e, d, ref, info)
        if info["squarings"] <= 10:
            assert rel1(e, ref) <= 1e-12
            low_s += 1
    assert low_s >= 3


@pytest.mark.parametrize("n,norm", [(8, 0.4), (33, 2.0), (100, 30.0), (130, 1000.0)])
def test_dense_split(split_ws, orc, n, norm):
    from csharp_linearalgebra_b200 import ExpmDiagnostics
    rng = np.random.default_rng(n)
    for cplx in (False, True):
        a = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
        a = np.asfortranarray(a * (norm / np.abs(a).sum(axis=0).max()))
        d = ExpmDiagnostics()
        e = split_ws.expm(a, d)
        ref, info = orc.expm(a)
        check(split_ws, a, e, d, ref, info)


def test_plain_form_is_restored(ws, orc):
    """After the split form is switched off, Expm is the reference's bit for bit again."""
    rng = np.random.default_rng(3)
    a = np.asfortranarray(rng.standard_normal((60, 60)) * 0.3)
    ws.set_split_moduli(MODULI)
    ws.expm(a)
    ws.set_split_moduli(0)
    ref, _ = orc.expm(a)
    assert np.array_equal(ws.expm(a), ref)


@pytest.mark.parametrize("theta", [1.495585217958292e-2, 2.539398330063230e-1])
@pytest.mark.parametrize("cplx", [False, True])
def test_decision_on_a_threshold_takes_exact_powers(split_ws, orc, theta, cplx):
    """A scaled so that eta1 = max(||A^4||^(1/4), ||A^6||^(1/6)) lies on a
    degree threshold to within rounding: the split form cannot settle the
    comparison on its bounds, recomputes A^2, A^4, A^6 as the reference does,
    and takes the reference's degree and s."""
    from csharp_linearalgebra_b200 import ExpmDiagnostics
    rng = np.random.default_rng(int(theta * 1000) + cplx)
    n = 60
    a = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    a2 = a @ a
    a4 = a2 @ a2
    a6 = a2 @ a4
    eta1 = max(np.abs(a4).sum(axis=0).max() ** 0.25, np.abs(a6).sum(axis=0).max() ** (1 / 6))
    a = np.asfortranarray(a * (theta / eta1))
    split_ws.reset_stats()
    d = ExpmDiagnostics()
    e = split_ws.expm(a, d)
    ref, info = orc.expm(a)
    assert split_ws.stats()["exact_fallbacks"] >= 1
    assert (d.degree, d.squarings) == (info["degree"], info["squarings"])
    assert rel1(e, ref) <= 1e-12
