"""DMMA GEMM (real and fused 4M complex) against the oracle, through the C ABI."""
import numpy as np
import pytest

from conftest import net_matrix, relfro

pytestmark = pytest.mark.gpu

# GemmTests.cs:31-44 plus the 1024^3 benchmark shape.
SHAPES = [(1, 1, 1), (1, 1, 64), (8, 6, 4), (16, 8, 16), (17, 9, 5), (31, 33, 7), (48, 48, 48),
          (64, 64, 64), (65, 63, 66), (100, 37, 129), (129, 130, 2), (300, 257, 511), (1024, 1024, 1024)]


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_dgemm_matches_oracle(ws, orc, m, n, k):
    a = net_matrix(orc, m, k, 11) if m * k <= 40000 else np.random.default_rng(1).uniform(-1, 1, (m, k))
    b = net_matrix(orc, k, n, 12) if k * n <= 40000 else np.random.default_rng(2).uniform(-1, 1, (k, n))
    c = ws.multiply(a, b)
    ref = orc.gemm(a, b)
    assert relfro(c, ref) < 1e-13
    # DMMA accumulates as the reference's FMA chain and the fold points match its KC slabs
    assert np.array_equal(c, ref)


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (1.0, 1.0), (-1.0, 1.0), (0.0, 1.0), (2.5, -0.5)])
def test_dgemm_alpha_beta(ws, orc, alpha, beta):
    a = net_matrix(orc, 65, 66, 1)
    b = net_matrix(orc, 66, 63, 2)
    c0 = net_matrix(orc, 65, 63, 3)
    c = ws.multiply(a, b, c0, alpha, beta)
    ref = orc.gemm(a, b, c0, alpha, beta)
    assert relfro(c, ref) < 1e-13
    # DMMA accumulates as the reference's FMA chain and the fold points match its KC slabs
    assert np.array_equal(c, ref)


def test_beta_zero_overwrites_nan(ws):
    a = np.ones((17, 9))
    b = np.ones((9, 5))
    c = np.full((17, 5), np.nan)
    out = ws.multiply(a, b, c, 1.0, 0.0)
    assert np.array_equal(out, np.full((17, 5), 9.0))


def test_padding_is_never_written(ws):
    """Only the m x n block of a strided C changes (GemmTests.cs:107-129)."""
    from csharp_linearalgebra_b200 import _native as N
    import ctypes as C
    m, n, k, ldc = 10, 7, 5, 13
    a = np.asfortranarray(np.random.default_rng(3).standard_normal((m, k)))
    b = np.asfortranarray(np.random.default_rng(4).standard_normal((k, n)))
    cbuf = np.full((ldc, n), 7.25, order="F")
    rc = N.load().tns_dgemm(ws.handle, m, n, k, 1.0, a.ctypes.data, m, b.ctypes.data, k, 0.0,
                            cbuf.ctypes.data, ldc)
    assert rc == 0
    assert np.all(cbuf[m:, :] == 7.25)
    assert relfro(cbuf[:m, :], a @ b) < 1e-14


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (17, 9, 5), (65, 63, 66), (100, 37, 129), (256, 256, 256), (512, 512, 512)])
def test_zgemm_matches_oracle(ws, orc, m, n, k):
    rng = np.random.default_rng(m + n + k)
    a = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    c = ws.multiply(a, b)
    ref = orc.gemm(a, b)
    assert relfro(c, ref) < 1e-13
    # DMMA accumulates as the reference's FMA chain and the fold points match its KC slabs
    assert np.array_equal(c, ref)


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (1.0, 1.0), (-1.0, 1.0), (2.0 - 1.0j, 0.5 + 0.25j)])
def test_zgemm_alpha_beta(ws, orc, alpha, beta):
    rng = np.random.default_rng(9)
    a = rng.standard_normal((33, 31)) + 1j * rng.standard_normal((33, 31))
    b = rng.standard_normal((31, 29)) + 1j * rng.standard_normal((31, 29))
    c0 = rng.standard_normal((33, 29)) + 1j * rng.standard_normal((33, 29))
    c = ws.multiply(a, b, c0, complex(alpha), complex(beta))
    ref = orc.gemm(a, b, c0, complex(alpha), complex(beta))
    assert relfro(c, ref) < 1e-13
    # DMMA accumulates as the reference's FMA chain and the fold points match its KC slabs
    assert np.array_equal(c, ref)


def test_4m_keeps_small_imaginary_parts(ws, orc):
    """ComplexMultiplyTests.cs:185-212: with tiny imaginary parts the 4M product
    keeps Im(AB) to relative accuracy (3M would lose it)."""
    rng = np.random.default_rng(21)
    n = 64
    ar, br = rng.standard_normal((n, n)), rng.standard_normal((n, n))
    ai, bi = 1e-9 * rng.standard_normal((n, n)), 1e-9 * rng.standard_normal((n, n))
    c = ws.multiply(ar + 1j * ai, br + 1j * bi)
    im_exact = ar @ bi + ai @ br
    assert np.linalg.norm(c.imag - im_exact) / np.linalg.norm(im_exact) < 1e-13


# A single product whose tiles leave SMs idle and whose K spans several KC
# slabs runs slab-split: one unit per (tile, slab, pass), each slab's raw
# product to its own plane, then a fold into C in slab order. These shapes take
# that route with both tile sizes and ragged last slabs (K = 704: 256 + 256 +
# 192; K = 528: 256 + 256 + 16; K = 4096: sixteen slabs of one tile).
SLAB_SPLIT_REAL = [((520, 390, 700), 1.0, 0.0), ((520, 390, 700), 2.5, -0.5), ((520, 390, 700), -1.0, 1.0),
                   ((64, 64, 4096), 1.0, 0.0), ((1030, 900, 520), 0.75, 1.0)]


@pytest.mark.parametrize("shape,alpha,beta", SLAB_SPLIT_REAL)
def test_dgemm_slab_split_matches_oracle(ws, orc, shape, alpha, beta):
    m, n, k = shape
    rng = np.random.default_rng(m + n + k)
    a = rng.uniform(-1, 1, (m, k))
    b = rng.uniform(-1, 1, (k, n))
    c0 = rng.uniform(-1, 1, (m, n))
    c = ws.multiply(a, b, c0, alpha, beta)
    assert np.array_equal(c, orc.gemm(a, b, c0, alpha, beta))


def test_dgemm_slab_split_beta_zero_overwrites_nan(ws, orc):
    rng = np.random.default_rng(5)
    a = rng.uniform(-1, 1, (300, 600))
    b = rng.uniform(-1, 1, (600, 250))
    c0 = np.full((300, 250), np.nan)
    c = ws.multiply(a, b, c0, 1.5, 0.0)
    assert not np.isnan(c).any()
    assert np.array_equal(c, orc.gemm(a, b, c0, 1.5, 0.0))


SLAB_SPLIT_COMPLEX = [((300, 200, 600), 1.0, 0.0), ((300, 200, 600), 2.0 - 1.0j, 0.5 + 0.25j),
                      ((300, 200, 600), 1.0, 1.0), ((300, 200, 600), -0.5, 0.0),
                      ((768, 640, 520), 2.0 - 1.0j, 0.5 + 0.25j), ((1024, 1024, 1024), 1.0, 0.0)]


@pytest.mark.parametrize("shape,alpha,beta", SLAB_SPLIT_COMPLEX)
def test_zgemm_slab_split_matches_oracle(ws, orc, shape, alpha, beta):
    m, n, k = shape
    rng = np.random.default_rng(m * n + k)
    a = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    c0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    c = ws.multiply(a, b, c0, complex(alpha), complex(beta))
    assert np.array_equal(c, orc.gemm(a, b, c0, complex(alpha), complex(beta)))
