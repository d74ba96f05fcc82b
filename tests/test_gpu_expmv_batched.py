"""The batched exponential action (one cooperative launch for every matrix's
Taylor recurrence) against the oracle and against the single-matrix call.

(m, s) are integer decisions and must equal the reference's; the kernel keeps
the reference's order of operations, so the application and early-exit
counts and the results must also be the oracle's, bit for bit.
"""
import math

import numpy as np
import pytest

from conftest import rel1

pytestmark = pytest.mark.gpu


def sweep_matrix(rng, n, w):
    """A = -(G + i w C), the frequency sweep's matrices."""
    g = rng.standard_normal((n, n)) / math.sqrt(n)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    d = np.exp(rng.uniform(math.log(1e-3), 0.0, n))
    c = (q.T * d) @ q
    c = 0.5 * (c + c.T)
    return np.asfortranarray(-(g + 1j * w * c))


def panel(rng, n, cols):
    return np.asfortranarray(rng.standard_normal((n, cols)) + 1j * rng.standard_normal((n, cols)))


def check_against_oracle(orc, mats, panels, t, outs, diags):
    for a, b, y, d in zip(mats, panels, outs, diags):
        ref, info = orc.expmv(a, b, t)
        assert (d.degree, d.scaling) == (info["degree"], info["scaling"])
        assert (d.applications, d.early_exits) == (info["applications"], info["early_exits"])
        assert rel1(y, ref) <= 1e-12, rel1(y, ref)
        assert np.array_equal(y, ref)


def test_sweep_matrices_eight_columns(ws, orc):
    """Configuration 4's shape (t = 0.5, B n x 8) on sweep matrices of mixed
    orders, the low end of the frequency range (what the CPU oracle finishes
    in seconds)."""
    rng = np.random.default_rng(44)
    mats, panels = [], []
    for w in np.logspace(2.0, 2.6, 6):
        n = int(rng.integers(64, 260))
        mats.append(sweep_matrix(rng, n, w))
        panels.append(panel(rng, n, 8))
    diags = []
    outs = ws.expmv_batched(mats, panels, 0.5, diags)
    check_against_oracle(orc, mats, panels, 0.5, outs, diags)
    assert all(d.applications > 100 for d in diags)


def test_batched_equals_single_calls(ws):
    rng = np.random.default_rng(45)
    mats = [sweep_matrix(rng, n, 150.0) for n in (70, 129, 200)]
    panels = [panel(rng, a.shape[0], 8) for a in mats]
    outs = ws.expmv_batched(mats, panels, 0.5)
    for a, b, y in zip(mats, panels, outs):
        assert np.array_equal(ws.expmv(a, b, 0.5), y)


@pytest.mark.parametrize("cols", [1, 5, 16, 20, 40])
def test_panel_widths(ws, orc, cols):
    """One, a partial slot, two and four columns per thread, and a panel wider
    than the kernel holds (the host-driven loop)."""
    rng = np.random.default_rng(cols)
    mats = [sweep_matrix(rng, n, 120.0) for n in (33, 96)]
    panels = [panel(rng, a.shape[0], cols) for a in mats]
    diags = []
    outs = ws.expmv_batched(mats, panels, 0.5, diags)
    check_against_oracle(orc, mats, panels, 0.5, outs, diags)


def test_real_batch_and_edge_orders(ws, orc):
    rng = np.random.default_rng(46)
    mats = [rng.standard_normal((n, n)) * (3.0 / math.sqrt(max(n, 1))) for n in (1, 2, 17, 130)]
    panels = [rng.standard_normal((a.shape[0], 3)) for a in mats]
    diags = []
    outs = ws.expmv_batched(mats, panels, -1.25, diags)
    check_against_oracle(orc, mats, panels, -1.25, outs, diags)


def test_zero_order_and_zero_time(ws, orc):
    rng = np.random.default_rng(47)
    mats = [np.zeros((0, 0), dtype=complex), sweep_matrix(rng, 40, 200.0)]
    panels = [np.zeros((0, 4), dtype=complex), panel(rng, 40, 4)]
    outs = ws.expmv_batched(mats, panels, 0.0)
    assert outs[0].shape == (0, 4)
    assert np.array_equal(outs[1], orc.expmv(mats[1], panels[1], 0.0)[0])


def test_one_large_matrix_uses_the_whole_gpu(ws, orc):
    """A single matrix of the sweep's largest order: its rows spread over
    many CTAs that meet at a barrier in global memory every application."""
    rng = np.random.default_rng(48)
    a = sweep_matrix(rng, 1000, 100.0)
    b = panel(rng, 1000, 8)
    diags = []
    outs = ws.expmv_batched([a], [b], 0.5, diags)
    check_against_oracle(orc, [a], [b], 0.5, outs, diags)


def test_parameter_selection_over_the_whole_frequency_range(ws, orc):
    """(m, s) for sweep matrices up to w = 1e6, where the recurrence itself
    (about 1.4 w applications) is out of reach for a test, from the
    selection-only entry point: equal to the reference's choice."""
    rng = np.random.default_rng(49)
    mats = [sweep_matrix(rng, int(rng.integers(40, 120)), w) for w in np.logspace(2.0, 6.0, 9)]
    got = ws.expmv_select_batched(mats, 8, 0.5)
    for a, ms in zip(mats, got):
        assert ms == orc.expmv_params(a, 8, 0.5)
    assert max(s for _, s in got) > 1000


def test_zero_entries_in_the_panel(ws, orc):
    """The reference skips a term whose x is zero; the kernel forms it, which
    adds +-0 to a sum that is never -0: the same bits."""
    rng = np.random.default_rng(50)
    mats = [sweep_matrix(rng, n, 150.0) for n in (40, 97)]
    panels = []
    for a in mats:
        b = panel(rng, a.shape[0], 6)
        b[rng.uniform(size=b.shape) < 0.5] = 0.0
        b[:, 2] = 0.0  # a whole zero column
        panels.append(np.asfortranarray(b))
    diags = []
    outs = ws.expmv_batched(mats, panels, 0.5, diags)
    check_against_oracle(orc, mats, panels, 0.5, outs, diags)


def test_non_finite_operator_follows_the_reference(ws, orc):
    """A non-finite entry: the shifted operator here is nilpotent, so the
    sharp bounds are 0 and the parameters finite (m = 1, s = 1), and the
    recurrence runs. The reference skips every term whose x is zero (no 0 x
    inf); the kernel's explicit-skip form, taken for such launches, gives the
    reference's infinities and NaNs in the same places."""
    a = np.eye(5, dtype=complex)
    a[1, 3] = np.inf
    b = np.ones((5, 2), dtype=complex)
    b[3, 0] = 0.0
    diags = []
    out = ws.expmv_batched([a], [b], 0.5, diags)[0]
    ref, info = orc.expmv(a, b, 0.5)
    assert (diags[0].degree, diags[0].scaling) == (info["degree"], info["scaling"])
    for part in (np.real, np.imag):
        assert np.array_equal(part(out), part(ref), equal_nan=True)
