"""Failure paths without a GPU fault: an allocation refused on the host side
of the library (an injected out-of-memory at the k-th device allocation), and
a device-side wait that runs out on a barrier nothing arrives on. Each call
must report its status, leave its destination untouched, and leave the
context usable for the next call."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _zexpm_raw(ws, a, out):
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    info = _native.ExpmInfo()
    n = a.shape[0]
    return lib.tns_zexpm(ws.handle, n, a.ctypes.data_as(C.c_void_p), n, out.ctypes.data_as(C.c_void_p), n,
                         C.byref(info))


@pytest.mark.parametrize("k", [1, 2, 3, 5, 8])
def test_injected_allocation_failure(ws, orc, k):
    from csharp_linearalgebra_b200 import _native
    rng = np.random.default_rng(k)
    n = 70
    a = np.asfortranarray((rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / 4.0)
    out = np.full((n, n), 7.0 + 7.0j, dtype=np.complex128, order="F")
    lib = _native.load()
    assert lib.tns_inject_allocation_failure(ws.handle, k) == 0
    rc = _zexpm_raw(ws, a, out)
    assert rc == _native.TNS_E_OUT_OF_MEMORY, lib.tns_last_error(ws.handle)
    assert b"injected" in lib.tns_last_error(ws.handle)
    assert np.all(out == 7.0 + 7.0j)  # the destination is untouched
    # the next call allocates normally and gives the reference's result
    assert _zexpm_raw(ws, a, out) == 0
    assert np.array_equal(out, orc.expm(a)[0])


def test_injection_can_be_disarmed(ws):
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    assert lib.tns_inject_allocation_failure(ws.handle, 1) == 0
    assert lib.tns_inject_allocation_failure(ws.handle, 0) == 0
    x = np.eye(8)
    assert np.array_equal(ws.multiply(x, x), x)
    assert lib.tns_inject_allocation_failure(ws.handle, -1) == _native.TNS_E_OUT_OF_RANGE


def test_device_wait_gives_up_and_the_context_survives(ws):
    from csharp_linearalgebra_b200 import DeviceTimeoutError, _native
    lib = _native.load()
    with pytest.raises(DeviceTimeoutError):
        ws._call("tns_selftest_wait", 1_000_000)  # 1 ms
    assert b"device-side wait gave up" in lib.tns_last_error(ws.handle)
    # the flag was cleared: the same context computes again
    x = np.arange(16.0).reshape(4, 4)
    assert np.array_equal(ws.multiply(x, np.eye(4)), x)
    assert lib.tns_selftest_wait(ws.handle, 3_000_000_000) == _native.TNS_E_OUT_OF_RANGE
