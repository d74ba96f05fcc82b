"""Expm at the benchmark's own sizes: matrices of the 256-matrix frequency
sweep with orders 600..1024 and w from 1e2 to 1e6 (s up to about 20), run
through the batched entry point as the benchmark runs them.

The plain form must be the oracle's result bit for bit, with its degree and
s. The split form must take the same degree and s, and lie within the bar of
tests/test_gpu_expm_split.py: max(1e-12, SPLIT_FLOOR_FACTOR x the floor),
the floor being how far the plain result moves when the input moves by
about one unit in the last place.
"""
import math

import numpy as np
import pytest

from conftest import rel1
from test_gpu_expm_split import SPLIT_FLOOR_FACTOR, sweep_matrix

pytestmark = pytest.mark.gpu


def bench_matrices():
    rng = np.random.default_rng(1024)
    ws_ = np.logspace(2.0, 6.0, 7)
    return [sweep_matrix(rng, int(rng.integers(600, 1025)), w) for w in ws_]


def test_plain_and_split_at_bench_orders(ws, orc):
    mats = bench_matrices()
    ws.set_split_moduli(0)
    pd, sd = [], []
    plain = ws.expm_batched(mats, pd)
    rng = np.random.default_rng(12345)
    pert = [np.asfortranarray(a * (1.0 + 2.0 ** -52 * rng.standard_normal(a.shape))) for a in mats]
    moved = ws.expm_batched(pert)
    ws.set_split_moduli(17)
    try:
        split = ws.expm_batched(mats, sd)
    finally:
        ws.set_split_moduli(0)
    rows = []
    for a, p, s, q, dp, ds in zip(mats, plain, split, moved, pd, sd):
        ref, info = orc.expm(a)
        assert (dp.degree, dp.squarings) == (info["degree"], info["squarings"])
        assert (ds.degree, ds.squarings) == (info["degree"], info["squarings"])
        assert np.array_equal(p, ref), rel1(p, ref)
        floor = rel1(q, ref)
        rows.append((a.shape[0], info["squarings"], rel1(s, ref), floor))
    table = "\n".join(f"n={n} s={s}: split {e:.3e}, floor {f:.3e} ({e / f:.2f}x)" for n, s, e, f in rows)
    print("\n" + table)
    for n, s, e, f in rows:
        assert e <= max(1e-12, SPLIT_FLOOR_FACTOR * f), table
    assert max(r[1] for r in rows) >= 18
