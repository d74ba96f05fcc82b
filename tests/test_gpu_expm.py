"""Expm on the GPU against the oracle: the Pade degree and the squaring count
must match exactly, the result to 1e-12 normwise."""
import math

import numpy as np
import pytest

from conftest import random_with_one_norm, rel1

pytestmark = pytest.mark.gpu

TOL = 1e-12


def check(ws, orc, a):
    from csharp_linearalgebra_b200 import ExpmDiagnostics
    d = ExpmDiagnostics()
    e = ws.expm(a, d)
    ref, info = orc.expm(a)
    assert (d.degree, d.squarings) == (info["degree"], info["squarings"])
    assert rel1(e, ref) <= TOL, rel1(e, ref)
    return d


def test_every_pade_degree_is_reached(ws, orc):
    seen = set()
    for norm in [0.001, 0.05, 0.4, 1.2, 6.0, 40.0]:
        a = random_with_one_norm(orc, 8, norm, 77 + int(norm * 10))
        seen.add(check(ws, orc, a).degree)
    assert sorted(seen) == [3, 5, 7, 9, 13]


@pytest.mark.parametrize("n,target", [(8, 0.001), (8, 0.4), (8, 40.0), (17, 0.01), (17, 0.8), (17, 12.0),
                                      (32, 2.5), (32, 30.0), (100, 500.0)])
def test_real_expm_matches_oracle(ws, orc, n, target):
    check(ws, orc, random_with_one_norm(orc, n, target, n * 1000 + int(target * 10)))


@pytest.mark.parametrize("n", [2, 7, 64, 65, 130])
@pytest.mark.parametrize("norm", [0.02, 1.0, 30.0, 1000.0])
def test_complex_expm_matches_oracle(ws, orc, n, norm):
    rng = np.random.default_rng(n * 7 + int(norm))
    a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2 * n)
    a *= norm / np.abs(a).sum(axis=0).max()
    check(ws, orc, a)


def test_dense_path_n512_ladder(ws, orc):
    """The n = 512 complex dense path over a log-uniform ||A||_1 ladder."""
    rng = np.random.default_rng(512)
    n = 512
    for norm in [1e-2, 1.0, 1e3]:
        a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2 * n)
        a *= norm / np.abs(a).sum(axis=0).max()
        check(ws, orc, a)


def test_closed_forms(ws):
    assert np.array_equal(ws.expm(np.zeros((6, 6))), np.eye(6))
    t = 0.3
    e = ws.expm(np.array([[0.0, -t], [t, 0.0]]))
    assert np.allclose(e, [[math.cos(t), -math.sin(t)], [math.sin(t), math.cos(t)]], atol=1e-12, rtol=0)
    lam = 1.75
    e = ws.expm(np.array([[lam, 1.0], [0.0, lam]]))
    assert np.allclose(e, [[math.exp(lam)] * 2, [0.0, math.exp(lam)]], atol=1e-11 * math.exp(lam), rtol=0)
    assert ws.expm(np.array([[-3.25]]))[0, 0] == pytest.approx(math.exp(-3.25), rel=1e-15)
    assert ws.expm(np.zeros((0, 0))).shape == (0, 0)


def test_rectangular_is_rejected(ws):
    with pytest.raises(ValueError):
        ws.expm(np.zeros((3, 4)))


def test_batched_matches_single(ws, orc):
    from csharp_linearalgebra_b200 import ExpmDiagnostics
    rng = np.random.default_rng(4)
    mats = []
    for n in [1, 2, 33, 64, 100]:
        a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * 3.0 / math.sqrt(n)
        mats.append(a)
    diags = []
    outs = ws.expm_batched(mats, diags)
    for a, e, d in zip(mats, outs, diags):
        ref, info = orc.expm(a)
        assert (d.degree, d.squarings) == (info["degree"], info["squarings"])
        assert rel1(e, ref) <= TOL


def test_frequency_sweep_matrices(ws, orc):
    """Matrices of the benchmark's frequency sweep, A = -(G + i w C), at both
    ends of the frequency range: degree and squarings equal the oracle's and
    the batched result agrees to 1e-12."""
    # orders below 200 so that the CPU oracle finishes quickly; the spectrum's
    # scale (|A| ~ w) is the sweep's
    rng = np.random.default_rng(9)
    small = []
    for k, w in enumerate(np.logspace(2.0, 6.0, 6)):
        n = int(rng.integers(64, 200))
        g = rng.standard_normal((n, n)) / math.sqrt(n)
        q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        d = np.exp(rng.uniform(math.log(1e-3), 0.0, n))
        c = (q.T * d) @ q
        c = 0.5 * (c + c.T)
        small.append(np.asfortranarray(-(g + 1j * w * c)))
    diags = []
    outs = ws.expm_batched(small, diags)
    for a, e, d in zip(small, outs, diags):
        ref, info = orc.expm(a)
        assert (d.degree, d.squarings) == (info["degree"], info["squarings"])
        assert rel1(e, ref) <= TOL, rel1(e, ref)
    assert max(d.squarings for d in diags) >= 15
