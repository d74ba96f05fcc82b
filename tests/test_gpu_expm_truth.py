"""Both GPU forms of Expm against exp(A) itself.

The truth is the extended-precision exponential of oracle/extended.py
(long double, about 2^-9 of an FP64 computation's rounding on these
matrices). The plain form is the reference's arithmetic bit for bit, so its
distance to the truth is the reference's own error; the split form's must be
no larger, within a small factor, for the split form to be as accurate as
the reference. Sweep matrices A = -(G + i w C) with w from 1e2 to 1e6 cover
s = 5 .. 20 squarings; three norm-scaled dense matrices cover s = 0 and the
low degrees.
"""
import math

import numpy as np
import pytest

from oracle.extended import expm_extended, has_extended_precision, rel1_extended

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not has_extended_precision(), reason="long double is not the 80-bit format")]

# The split form's error against the truth, at most this multiple of the
# plain form's (the reference's) error against the truth, plus 1e-15 for
# the matrices whose errors are at the unit roundoff.
FACTOR = 2.0


def sweep_matrix(rng, n, w):
    g = rng.standard_normal((n, n)) / math.sqrt(n)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    d = np.exp(rng.uniform(math.log(1e-3), 0.0, n))
    c = (q.T * d) @ q
    c = 0.5 * (c + c.T)
    return np.asfortranarray(-(g + 1j * w * c))


def matrices():
    rng = np.random.default_rng(2027)
    mats = [sweep_matrix(rng, int(rng.integers(48, 129)), w) for w in np.logspace(2.0, 6.0, 9)]
    for norm in (0.05, 1.5, 40.0):
        n = 96
        a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2 * n)
        mats.append(np.asfortranarray(a * (norm / np.abs(a).sum(axis=0).max())))
    return mats


@pytest.mark.parametrize("moduli", [17, 20])
def test_split_form_is_as_accurate_as_the_reference(ws, orc, moduli):
    mats = matrices()
    ws.set_split_moduli(0)
    pd, sd = [], []
    plain = ws.expm_batched(mats, pd)
    ws.set_split_moduli(moduli)
    try:
        split = ws.expm_batched(mats, sd)
    finally:
        ws.set_split_moduli(0)
    rows = []
    for a, p, s, dp, ds in zip(mats, plain, split, pd, sd):
        truth = expm_extended(a)
        ref, info = orc.expm(a)
        assert np.array_equal(p, ref)  # the plain form is the reference's result
        assert (dp.degree, dp.squarings) == (ds.degree, ds.squarings) == (info["degree"], info["squarings"])
        rows.append((a.shape[0], dp.degree, dp.squarings, rel1_extended(p, truth), rel1_extended(s, truth)))
    table = "\n".join(f"n={n} m={m} s={s}: reference {ep:.3e}, split {es:.3e}" for n, m, s, ep, es in rows)
    print("\n" + table)
    for n, m, s, ep, es in rows:
        assert es <= FACTOR * ep + 1e-15, table
    assert max(r[2] for r in rows) >= 18 and min(r[2] for r in rows) == 0
