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
    rc = lib.tns_zgemm_device_noalloc(None, m, n, k, al.ctypes.data_as(C.c_void_p), da.data_ptr(), m,
                                      db.data_ptr(), k, be.ctypes.data_as(C.c_void_p), dc.data_ptr(), m)
    assert rc == 0, lib.tns_last_error(None)
    return dc.cpu().numpy().T


def test_noalloc_matches_the_allocating_entry_point_on_consecutive_calls(ws):
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    rng = np.random.default_rng(77)
    # Two calls in a row with different shapes and scalars: the second finds
    # the first one's data in the working array.
    for m, n, k, alpha, beta in [(300, 257, 129, 1.0, 0.0), (130, 63, 200, 2.0 - 1.0j, 0.5 + 0.25j)]:
        a = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
        b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
        c0 = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
        expected = ws.multiply(a, b, c0, complex(alpha), complex(beta))
        got = _noalloc(lib, m, n, k, alpha, a, b, beta, c0)
        assert relfro(got, expected) < 1e-13


def test_noalloc_refuses_products_beyond_its_fixed_storage():
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    al = np.array([1.0, 0.0])
    rc = lib.tns_zgemm_device_noalloc(None, 2048, 2048, 2048, al.ctypes.data_as(C.c_void_p), 16, 2048, 16, 2048,
                                      al.ctypes.data_as(C.c_void_p), 16, 2048)
    assert rc == _native.TNS_E_OUT_OF_RANGE
    assert b"tns_zgemm_device" in lib.tns_last_error(None)
