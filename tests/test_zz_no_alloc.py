"""tns_zgemm_device_noalloc: the complex product for callers that may not
allocate device memory (an application whose allocator has reserved the GPU's
memory, a loop that must stay off the driver's allocation path). It must give
the existing entry point's result, call after call, although every call reuses
the same fixed working array. Collected last, so that a run stopping at its
first failure has run everything else before it."""
import ctypes as C

import numpy as np
import pytest

from conftest import relfro

pytestmark = pytest.mark.gpu


def _device(x):
    """A column-major complex128 device copy of x (a torch tensor holding x^T)."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(x, dtype=np.complex128).T)).to("cuda")


def _noalloc(lib, m, n, k, alpha, a, b, beta, c0):
    import torch
    da, db, dc = _device(a), _device(b), _device(c0)
    al = np.array([complex(alpha).real, complex(alpha).imag])
    be = np.array([complex(beta).real, complex(beta).imag])
    torch.cuda.synchronize()
    rc = lib.tns_zgemm_device_noalloc(None, m, n, k, al.ctypes.data_as(C.c_void_p), da.data_ptr(), max(m, 1),
                                      db.data_ptr(), max(k, 1), be.ctypes.data_as(C.c_void_p), dc.data_ptr(),
                                      max(m, 1))
    assert rc == 0, lib.tns_last_error(None)
    return dc.cpu().numpy().T


def _allocating(lib, ws, m, n, k, alpha, a, b, beta, c0):
    """The same product through tns_zgemm_device (device operands, the
    library's own allocations)."""
    import torch
    da, db, dc = _device(a), _device(b), _device(c0)
    al = np.array([complex(alpha).real, complex(alpha).imag])
    be = np.array([complex(beta).real, complex(beta).imag])
    torch.cuda.synchronize()
    rc = lib.tns_zgemm_device(ws._h, m, n, k, al.ctypes.data_as(C.c_void_p), da.data_ptr(), max(m, 1),
                              db.data_ptr(), max(k, 1), be.ctypes.data_as(C.c_void_p), dc.data_ptr(), max(m, 1))
    assert rc == 0, lib.tns_last_error(ws._h)
    return dc.cpu().numpy().T


def test_noalloc_matches_the_allocating_entry_point_on_consecutive_calls(ws):
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    rng = np.random.default_rng(77)
    # Calls in a row with different shapes and scalars: each finds the
    # previous one's data in the working array. Odd m and n exercise the
    # padding to even extents; the two paths run the same kernel with the
    # same summation order, so the results are the same bits.
    for m, n, k, alpha, beta in [(300, 257, 129, 1.0, 0.0), (130, 63, 200, 2.0 - 1.0j, 0.5 + 0.25j),
                                 (301, 77, 33, 1.0, 1.0), (1, 1, 1, -1.0j, 0.0)]:
        a = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
        b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
        c0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
        expected = _allocating(lib, ws, m, n, k, alpha, a, b, beta, c0)
        got = _noalloc(lib, m, n, k, alpha, a, b, beta, c0)
        assert np.array_equal(got, expected), relfro(got, expected)
        # and the product itself, against the host-buffer entry point
        assert relfro(got, ws.multiply(a, b, c0, complex(alpha), complex(beta))) < 1e-13


def test_noalloc_empty_depth_scales_c_by_beta_only(ws):
    """k == 0: C := beta*C, alpha unread (a NaN alpha must not reach C)."""
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    rng = np.random.default_rng(5)
    m, n = 37, 12
    c0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    a = np.zeros((m, 0), dtype=np.complex128)
    b = np.zeros((0, n), dtype=np.complex128)
    for beta in (0.5 + 0.25j, 0.0):
        got = _noalloc(lib, m, n, 0, complex(np.nan, 0.0), a, b, beta, c0)
        expected = _allocating(lib, ws, m, n, 0, complex(np.nan, 0.0), a, b, beta, c0)
        assert np.array_equal(got, expected)
        assert np.all(np.isfinite(got))


def test_noalloc_refuses_products_beyond_its_fixed_storage():
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    al = np.array([1.0, 0.0])
    rc = lib.tns_zgemm_device_noalloc(None, 2048, 2048, 2048, al.ctypes.data_as(C.c_void_p), 16, 2048, 16, 2048,
                                      al.ctypes.data_as(C.c_void_p), 16, 2048)
    assert rc == _native.TNS_E_OUT_OF_RANGE
    assert b"tns_zgemm_device" in lib.tns_last_error(None)
