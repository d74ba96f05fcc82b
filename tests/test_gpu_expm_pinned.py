"""Batched complex Expm from and into pinned host buffers (tns_zexpm_batched).

With page-locked outputs each matrix's result is copied to the host as soon as
it is final -- after the Pade solve when s = 0, else after its last squaring --
on a second stream, while the group's other matrices still square. The results
must be the oracle's (plain form) and the same bits as the pageable path,
which copies every result at the end, in both forms; degree and s must match.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(seed, count):
    """Complex matrices with orders 33..300 and 1-norms spread over 1e-3..1e4,
    so that the batch holds every degree and s from 0 to about 14."""
    rng = np.random.default_rng(seed)
    norms = np.exp(np.linspace(math.log(1e-3), math.log(1e4), count))
    rng.shuffle(norms)
    mats = []
    for v in norms:
        n = int(rng.integers(33, 301))
        a = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / math.sqrt(2 * n)
        mats.append(np.asfortranarray(a * (v / np.abs(a).sum(axis=0).max())))
    return mats


def _pinned_run(ws, mats):
    import torch
    host_in = [torch.from_numpy(m.T.copy()).pin_memory() for m in mats]
    host_out = [torch.zeros_like(t).pin_memory() for t in host_in]
    orders = [m.shape[0] for m in mats]
    infos = ws.expm_batched_host(len(mats), orders, [t.data_ptr() for t in host_in], orders,
                                 [t.data_ptr() for t in host_out], orders)
    return [t.numpy().T.copy() for t in host_out], infos


@pytest.mark.parametrize("moduli", [0, 17])
def test_pinned_outputs_match_pageable_and_oracle(ws, orc, moduli):
    mats = _batch(2027 + moduli, 14)
    ws.set_split_moduli(moduli)
    try:
        got, infos = _pinned_run(ws, mats)
        diags = []
        ref = ws.expm_batched(mats, diags)
    finally:
        ws.set_split_moduli(0)
    squarings = set()
    for k, m in enumerate(mats):
        assert (infos[k].degree, infos[k].squarings) == (diags[k].degree, diags[k].squarings)
        assert np.array_equal(got[k], ref[k])
        squarings.add(infos[k].squarings)
        if moduli == 0:
            want, info = orc.expm(m)
            assert (infos[k].degree, infos[k].squarings) == (info["degree"], info["squarings"])
            assert np.array_equal(got[k], want)
    assert 0 in squarings and max(squarings) >= 8  # finished in many different rounds
