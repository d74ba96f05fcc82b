"""The C ABI library: it loads, exports every entry point include/tensile_b200.h
declares, and rejects a null context before touching a GPU. CPU only."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "tensile_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tns_\w+)\s*\(", src)))


def test_library_builds_and_loads():
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    assert os.path.exists(_native.LIB_PATH)
    assert lib is not None


def test_every_declared_symbol_is_exported():
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each of them
    assert set(names) <= set(_native.SIGNATURES), set(names) - set(_native.SIGNATURES)


@pytest.mark.parametrize("name", ["tns_dgemm", "tns_zgemm", "tns_dgetrf", "tns_zexpm", "tns_dexpmv",
                                  "tns_dnormest1_power", "tns_zgecon", "tns_dnorm"])
def test_null_context_is_disposed_error(name):
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    argtypes = _native.SIGNATURES[name][1]
    def zero(t):
        if t is C.c_char:
            return b"1"  # the norm kind
        if isinstance(t, type) and issubclass(t, C._Pointer):
            return None
        return 0
    args = [None] + [zero(t) for t in argtypes[1:]]
    assert getattr(lib, name)(*args) == _native.TNS_E_DISPOSED
    assert b"null" in lib.tns_last_error(None) or b"destroyed" in lib.tns_last_error(None)


def test_create_without_device_fails_cleanly():
    """On a machine without a GPU, tns_create returns an error code rather than
    crashing; with a GPU it succeeds."""
    from csharp_linearalgebra_b200 import _native
    lib = _native.load()
    h = C.c_void_p()
    rc = lib.tns_create(0, 0, C.byref(h))
    if rc == _native.TNS_OK:
        assert lib.tns_destroy(h) == _native.TNS_OK
    else:
        assert rc in (_native.TNS_E_DEVICE, _native.TNS_E_ARGUMENT)
        assert h.value is None


def test_package_has_no_cpu_fallback():
    """The product package never imports the oracle."""
    pkg = os.path.join(ROOT, "csharp_linearalgebra_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".h", ".cuh", ".cpp")):
                text = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in text.lower(), f
