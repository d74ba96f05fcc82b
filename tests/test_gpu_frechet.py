"""Differentiation form on the GPU, through the C ABI: the Frechet derivative
L(A, E) of exp and the gradient of ||exp(tA) B - Y||_F^2.

Oracles:
  - the reference's way to L(A, E): the upper right block of its Expm of
    [[A, E], [0, A]]. At small orders that is the oracle's Expm (pinned in
    test_frechet_pins.py); at the differentiation configuration's n = 1024 it
    is the library's plain Expm of the 2048-order block, itself checked equal
    to the oracle's Expm of that block bit for bit;
  - central finite differences, fourth order,
        dF ~ (-F(2h) + 8 F(h) - 8 F(-h) + F(-2h)) / (12 h),
    in unit-1-norm directions with h = 1e-3 to 3e-3, each F from the exact
    Expm. For the loss the difference is taken of F and contracted with
    G = 2 (F - Y), which is the loss's exact first-order change (the loss is
    quadratic in F), so no two large losses are subtracted.

Tolerances: L(A, E) and exp(A) within 1e-11 (1-norm, relative) of the block
Expm: two backward-stable FP64 evaluations with different degree and
scaling. Gradients within 1e-8 of the finite differences, the stated target
for the differentiation form, at operator norms where finite differences
can resolve it (|A|_1 ~ 40: their own error is about 5e-11). At the
configuration's operator (w = 1e4, |A|_1 ~ 7e4, 14 squarings) every FP64 Expm
carries rounding of about 4e-10 of its norm, which a difference quotient
divides by h: the finite differences of the reference's own block Expm miss
it by 2e-7 at h = 3e-3 and 7e-7 at h = 1e-3, falling as 1/h, while L agrees
with that block Expm to 5e-14. There the block Expm is the check.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_BLOCK = 1e-11
TOL_FD = 1e-8


def rel(x, y):
    return np.abs(x - y).sum(axis=0).max() / np.abs(y).sum(axis=0).max()


def block_frechet(orc, a, e):
    n = a.shape[0]
    blk = np.zeros((2 * n, 2 * n), dtype=np.result_type(a, e), order="F")
    blk[:n, :n] = a
    blk[:n, n:] = e
    blk[n:, n:] = a
    r, _ = orc.expm(blk)
    return r[:n, :n], r[:n, n:]


def sweep_operator(rng, n, w):
    """A as in the batching configuration: -(G + i w C)."""
    g = rng.standard_normal((n, n)) / math.sqrt(n)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    d = np.exp(rng.uniform(math.log(1e-3), 0.0, n))
    c = (q.T * d) @ q
    c = 0.5 * (c + c.T)
    return np.asfortranarray(-(g + 1j * w * c))


def unit(rng, shape, cplx):
    x = rng.standard_normal(shape) + (1j * rng.standard_normal(shape) if cplx else 0)
    return np.asfortranarray(x / np.abs(x).sum(axis=0).max())


def stencil(fn, h):
    return (-fn(2 * h) + 8 * fn(h) - 8 * fn(-h) + fn(-2 * h)) / (12 * h)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n,norm,degree", [(8, 5e-3, 3), (20, 0.15, 5), (33, 0.6, 7), (40, 1.5, 9),
                                           (64, 4.0, 13), (100, 30.0, 13), (130, 400.0, 13)])
def test_frechet_matches_block_expm(ws, orc, cplx, n, norm, degree):
    from csharp_linearalgebra_b200 import ExpmDiagnostics
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    a = np.asfortranarray(a * (norm / np.abs(a).sum(axis=0).max()))
    e = unit(rng, (n, n), cplx)
    d = ExpmDiagnostics()
    x, l = ws.expm_frechet(a, e, d)
    assert d.degree == degree
    xr, lr = block_frechet(orc, a, e)
    print(f"n={n} norm={norm} cplx={cplx} degree={d.degree} s={d.squarings} "
          f"L {rel(l, lr):.2e} exp {rel(x, xr):.2e}")
    assert rel(l, lr) <= TOL_BLOCK
    assert rel(x, xr) <= TOL_BLOCK


def test_frechet_is_linear_in_direction(ws):
    rng = np.random.default_rng(9)
    a = sweep_operator(rng, 96, 30.0)
    e1, e2 = unit(rng, a.shape, True), unit(rng, a.shape, True)
    _, l1 = ws.expm_frechet(a, e1)
    _, l2 = ws.expm_frechet(a, e2)
    _, l12 = ws.expm_frechet(a, 2.0 * e1 - 3.0 * e2)
    assert rel(l12, 2.0 * l1 - 3.0 * l2) <= 1e-13


def test_checkpoints_recomputed_give_same_bits(ws):
    """Keeping every squaring or squaring again from X_0 runs the same products
    on the same operands: the derivative is bit-identical."""
    rng = np.random.default_rng(10)
    a = sweep_operator(rng, 150, 300.0)
    e = unit(rng, a.shape, True)
    from csharp_linearalgebra_b200 import ExpmDiagnostics
    d = ExpmDiagnostics()
    x1, l1 = ws.expm_frechet(a, e, d)
    assert d.squarings >= 3
    ws.set_checkpoint_bytes(0)
    try:
        x2, l2 = ws.expm_frechet(a, e)
    finally:
        ws.set_checkpoint_bytes(-1)
    assert np.array_equal(l1, l2)
    assert np.array_equal(x1, x2)


def gpu_block_frechet(ws, a, e):
    """Upper right block of the plain (reference-arithmetic) Expm of
    [[A, E], [0, A]], E scaled to unit 1-norm and the block scaled back."""
    n = a.shape[0]
    scale = np.abs(e).sum(axis=0).max()
    blk = np.zeros((2 * n, 2 * n), dtype=np.complex128, order="F")
    blk[:n, :n] = a
    blk[:n, n:] = e / scale
    blk[n:, n:] = a
    return ws.expm(blk)[:n, n:] * scale


def test_frechet_finite_differences(ws):
    rng = np.random.default_rng(512)
    a = sweep_operator(rng, 512, 10.0)
    e = unit(rng, a.shape, True)
    _, l = ws.expm_frechet(a, e)
    fd = stencil(lambda h: ws.expm(np.asfortranarray(a + h * e)), 3e-3)
    print(f"Frechet n=512 vs finite differences: {rel(l, fd):.2e}")
    assert rel(l, fd) <= TOL_FD


def test_frechet_block_n1024(ws, orc):
    """L(A, E) at n = 1024 (the differentiation configuration's Frechet case),
    A as in the batching sweep at w = 1e4, E random. The block Expm it is
    checked against is first checked against the oracle's Expm of the same
    2048-order block, bit for bit (the reference's own route to L)."""
    from csharp_linearalgebra_b200 import ExpmDiagnostics
    rng = np.random.default_rng(1024)
    a = sweep_operator(rng, 1024, 1e4)
    e = unit(rng, a.shape, True)
    d = ExpmDiagnostics()
    x, l = ws.expm_frechet(a, e, d)
    lb = gpu_block_frechet(ws, a, e)
    n = a.shape[0]
    scale = np.abs(e).sum(axis=0).max()
    blk = np.zeros((2 * n, 2 * n), dtype=np.complex128, order="F")
    blk[:n, :n] = a
    blk[:n, n:] = e / scale
    blk[n:, n:] = a
    ref, _ = orc.expm(blk)
    assert np.array_equal(ref[:n, n:] * scale, lb)
    print(f"Frechet n=1024 (s={d.squarings}) vs block Expm: {rel(l, lb):.2e}; exp vs Expm {rel(x, ws.expm(a)):.2e}")
    assert rel(l, lb) <= TOL_BLOCK
    assert rel(x, ws.expm(a)) <= TOL_BLOCK


def gradient_checks(ws, a, b, y, t):
    rng = np.random.default_rng(77)
    cplx = np.iscomplexobj(a)
    r = ws.expmv_gradient(a, b, y, t)

    def f_of(a_, b_, t_):
        return ws.expm(np.asfortranarray(t_ * a_)) @ b_

    f0 = f_of(a, b, t)
    g = 2.0 * (f0 - y)
    assert rel(r["f"], f0) <= 1e-11
    assert abs(r["loss"] - np.linalg.norm(f0 - y) ** 2) <= 1e-11 * r["loss"]

    def inner(x, z):
        return float(np.real(np.vdot(x, z)))

    da = unit(rng, a.shape, cplx)
    db = unit(rng, b.shape, cplx)
    ha = 1e-3
    ht = 1e-3 / np.abs(a).sum(axis=0).max()
    fd_a = inner(g, stencil(lambda h: f_of(a + h * da, b, t), ha))
    fd_b = inner(g, stencil(lambda h: f_of(a, b + h * db, t), ha))
    fd_t = inner(g, stencil(lambda h: f_of(a, b, t + h), ht))
    ad_a, ad_b, ad_t = inner(r["grad_a"], da), inner(r["grad_b"], db), r["grad_t"]
    errs = (abs(ad_a - fd_a) / abs(fd_a), abs(ad_b - fd_b) / abs(fd_b), abs(ad_t - fd_t) / abs(fd_t))
    print(f"gradient vs finite differences (A, B, t): {errs[0]:.2e} {errs[1]:.2e} {errs[2]:.2e}")
    for err in errs:
        assert err <= TOL_FD
    return r


@pytest.mark.parametrize("cplx", [False, True])
def test_gradient_small(ws, orc, cplx):
    rng = np.random.default_rng(31)
    n, c, t = 60, 4, 0.7
    a = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    a = np.asfortranarray(a * (6.0 / np.abs(a).sum(axis=0).max()))
    b = np.asfortranarray(rng.standard_normal((n, c)) + (1j * rng.standard_normal((n, c)) if cplx else 0))
    y = np.asfortranarray(rng.standard_normal((n, c)) + (1j * rng.standard_normal((n, c)) if cplx else 0))
    r = gradient_checks(ws, a, b, y, t)
    # dloss/dA against the block Expm: t L(t A^H, G B^H).
    f0 = orc.expm(t * a)[0] @ b
    g = 2.0 * (f0 - y)
    _, lr = block_frechet(orc, np.asfortranarray(t * a.conj().T), np.asfortranarray(g @ b.conj().T))
    assert rel(r["grad_a"], t * lr) <= TOL_BLOCK


def test_gradient_finite_differences(ws):
    """The configuration's shapes (B n x 16, t = 1) at an operator norm where
    finite differences resolve 1e-8 (w = 10, n = 512)."""
    rng = np.random.default_rng(2049)
    n, c = 512, 16
    a = sweep_operator(rng, n, 10.0)
    b = np.asfortranarray(rng.standard_normal((n, c)) + 1j * rng.standard_normal((n, c)))
    y = np.asfortranarray(rng.standard_normal((n, c)) + 1j * rng.standard_normal((n, c)))
    gradient_checks(ws, a, b, y, 1.0)


def test_gradient_differentiation_configuration(ws):
    """n = 2048, B 2048 x 16 (N(0,1)), Y random, t = 1, A as in the sweep at
    w = 1e4: each gradient against its definition, evaluated with the plain
    Expm (dloss/dA through the block Expm of t A^H in the direction G B^H)."""
    rng = np.random.default_rng(2048)
    n, c, t = 2048, 16, 1.0
    a = sweep_operator(rng, n, 1e4)
    b = np.asfortranarray(rng.standard_normal((n, c)) + 1j * rng.standard_normal((n, c)))
    y = np.asfortranarray(rng.standard_normal((n, c)) + 1j * rng.standard_normal((n, c)))
    r = ws.expmv_gradient(a, b, y, t)
    x = ws.expm(np.asfortranarray(t * a))
    f0 = x @ b
    g = 2.0 * (f0 - y)
    assert rel(r["f"], f0) <= TOL_BLOCK
    assert abs(r["loss"] - np.linalg.norm(f0 - y) ** 2) <= 1e-11 * r["loss"]
    # A product's error scale is the product of its factors' norms: at w = 1e4
    # exp(tA) oscillates and X^H G is far smaller than |X^H| |G|, so the two
    # exponentials' 4e-14 difference is measured against |X^H| |G|.
    xh = x.conj().T
    n1 = lambda m: np.abs(m).sum(axis=0).max()
    assert n1(r["grad_b"] - xh @ g) <= TOL_BLOCK * n1(xh) * n1(g)
    gt = float(np.real(np.vdot(g, a @ f0)))
    assert abs(r["grad_t"] - gt) <= 1e-11 * abs(gt)
    # L(X, D) = int_0^1 e^{sX} D e^{(1-s)X} ds: both evaluations round on the
    # scale |e^X| |D|, and the rank-16 direction D = G B^H gives an L far
    # below it, so the difference is measured against t |e^{tA^H}| |D|.
    dr = np.asfortranarray(g @ b.conj().T)
    la = gpu_block_frechet(ws, np.asfortranarray(t * a.conj().T), dr)
    err = n1(r["grad_a"] - t * la)
    scale = t * n1(xh) * n1(dr)
    print(f"gradient n=2048 (s={r['squarings']}): dA vs block Expm {rel(r['grad_a'], t * la):.2e} of |dA|, "
          f"{err / scale:.2e} of t |e^(tA^H)| |G B^H|")
    assert err <= TOL_BLOCK * scale
