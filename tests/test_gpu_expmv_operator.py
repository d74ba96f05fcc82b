"""Matrix-free Expmv on the GPU (MatrixExponentialAction.Expmv over
ILinearOperator<T>, src/Tensile/MatrixExponentialAction.cs:203-230): the
operator is a caller's function applied to device panels on the library's
stream, here written with torch. (m, s) equal the oracle's exactly (they
follow from |t| times the caller's norm bound); results within 1e-12."""
import numpy as np
import pytest
import torch

from conftest import rel1

pytestmark = pytest.mark.gpu


class Panel:
    """A device panel seen by torch: n x ncols column-major with leading
    dimension ld, exposed as the row-major (ncols, ld) array it is."""

    def __init__(self, ptr, ncols, ld, cplx):
        self.__cuda_array_interface__ = {"shape": (ncols, ld), "typestr": "<c16" if cplx else "<f8",
                                         "data": (ptr, False), "version": 3, "strides": None}


def dense_operator(a):
    cplx = np.iscomplexobj(a)
    at = torch.from_numpy(np.ascontiguousarray(a)).to("cuda")  # row-major A
    n = a.shape[0]

    def apply(x, y, ncols, ld, stream):
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            xv = torch.as_tensor(Panel(x, ncols, ld, cplx), device="cuda")
            yv = torch.as_tensor(Panel(y, ncols, ld, cplx), device="cuda")
            yv[:, :n] = xv[:, :n] @ at.T  # (A X)^T = X^T A^T
    return apply


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("norm,t", [(0.05, 1.0), (3.0, 0.5), (40.0, 1.0), (40.0, -0.7)])
def test_operator_matches_oracle(ws, orc, cplx, norm, t):
    from csharp_linearalgebra_b200 import ExpmvDiagnostics
    rng = np.random.default_rng(int(norm * 100) + cplx)
    n = 120
    a = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if cplx else 0)
    a = np.asfortranarray(a * (norm / np.abs(a).sum(axis=0).max()))
    b = np.asfortranarray(rng.standard_normal((n, 6)) + (1j * rng.standard_normal((n, 6)) if cplx else 0))
    bound = np.abs(a).sum(axis=0).max()
    d = ExpmvDiagnostics()
    out = ws.expmv_operator(dense_operator(a), n, b, t, bound, complex_=cplx, diagnostics=d)
    ref, info = orc.expmv_bound(a, b, t, bound)
    assert (d.degree, d.scaling) == (info["degree"], info["scaling"])
    assert rel1(out, ref) <= 1e-12


def test_stencil_operator(ws):
    """A second-difference stencil never formed as a matrix: y_i = x_{i-1} - 2 x_i + x_{i+1}."""
    import scipy.linalg
    n = 400

    def apply(x, y, ncols, ld, stream):
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            xv = torch.as_tensor(Panel(x, ncols, ld, False), device="cuda")[:, :n]
            yv = torch.as_tensor(Panel(y, ncols, ld, False), device="cuda")
            r = -2.0 * xv
            r[:, 1:] += xv[:, :-1]
            r[:, :-1] += xv[:, 1:]
            yv[:, :n] = r

    b = np.random.default_rng(3).standard_normal((n, 3))
    out = ws.expmv_operator(apply, n, b, 2.0, 4.0)
    a = -2.0 * np.eye(n) + np.eye(n, k=1) + np.eye(n, k=-1)
    assert rel1(out, scipy.linalg.expm(2.0 * a) @ b) <= 1e-12


def test_operator_failure_and_bad_bound(ws):
    def broken(x, y, ncols, ld, stream):
        raise KeyError("operator failed")

    b = np.ones((10, 2))
    with pytest.raises(KeyError):
        ws.expmv_operator(broken, 10, b, 1.0, 1.0)
    with pytest.raises(OverflowError):
        ws.expmv_operator(broken, 10, b, 1.0, -1.0)
    # the workspace stays usable
    assert rel1(ws.expmv_operator(dense_operator(np.zeros((10, 10))), 10, b, 1.0, 0.0), b) == 0.0


def adjoint_pair(a):
    """apply and adjoint callbacks of a dense A (torch on the library's stream)."""
    cplx = np.iscomplexobj(a)
    n = a.shape[0]
    at = torch.from_numpy(np.ascontiguousarray(a)).to("cuda")

    def make(mat):
        def fn(x, y, ncols, ld, stream):
            with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                xv = torch.as_tensor(Panel(x, ncols, ld, cplx), device="cuda")
                yv = torch.as_tensor(Panel(y, ncols, ld, cplx), device="cuda")
                yv[:, :n] = xv[:, :n] @ mat.T
        return fn
    return make(at), make(at.conj().T.contiguous())


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n", [64, 128])
def test_operator_normest_matches_oracle(ws, orc, cplx, n):
    """Small-integer entries and the estimator's probes (1/n, +-1, unit
    vectors) make every product exact in any summation order, so the estimate,
    iterations and products equal the oracle's exactly."""
    rng = np.random.default_rng(n + 5 * cplx)
    a = rng.integers(-5, 6, (n, n)).astype(float)
    if cplx:
        a = a + 1j * rng.integers(-5, 6, (n, n))
    a = np.asfortranarray(a)
    apply, adjoint = adjoint_pair(a)
    got = ws.estimate_operator_norm(apply, adjoint, n, complex_=cplx)
    ref = orc.normest_power(a, 1)
    exact = np.abs(a).sum(axis=0).max()
    assert got.value <= exact * (1 + 1e-15)
    assert (got.value, got.iterations, got.products) == ref
