"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

The oracle (tensile_oracle.cpp) restates the reference library's CPU
algorithms. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg import this module; the product package never does.

Arrays are numpy, column-major (Fortran order). Complex arrays are complex128,
whose memory layout is the interleaved (re, im) layout of
System.Numerics.Complex.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")


class LuInfo(C.Structure):
    _fields_ = [("singular_column", C.c_int), ("smallest_pivot", C.c_double),
                ("largest_pivot", C.c_double)]


class NormestResult(C.Structure):
    _fields_ = [("value", C.c_double), ("iterations", C.c_int), ("products", C.c_int)]


class ExpmInfo(C.Structure):
    _fields_ = [("degree", C.c_int), ("squarings", C.c_int), ("eta1", C.c_double),
                ("eta3", C.c_double), ("eta5", C.c_double), ("d4", C.c_double),
                ("d6", C.c_double), ("d8", C.c_double), ("d10", C.c_double)]


class ExpmvInfo(C.Structure):
    _fields_ = [("degree", C.c_int), ("scaling", C.c_int), ("applications", C.c_int),
                ("early_exits", C.c_int)]


def build() -> str:
    """Compile the oracle with its Makefile (g++, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        i, d = C.c_int, C.c_double
        L.orc_random_new.restype = P
        L.orc_random_new.argtypes = [i]
        L.orc_random_free.argtypes = [P]
        L.orc_random_next.argtypes = [P, i]
        L.orc_random_next_double.argtypes = [P]
        L.orc_random_next_double.restype = d
        L.orc_sort_keys_items.argtypes = [i, P, P]
        L.orc_set_threads.argtypes = [i]
        L.orc_get_threads.restype = i
        L.orc_dgemm.argtypes = [i, i, i, d, P, i, P, i, d, P, i, i]
        L.orc_zgemm.argtypes = [i, i, i, P, P, i, P, i, P, P, i, i]
        for name in ("orc_dnorm1", "orc_dnorminf", "orc_dnormfro", "orc_znorm1", "orc_znorminf"):
            getattr(L, name).argtypes = [i, i, P, i]
            getattr(L, name).restype = d
        L.orc_zabs.argtypes = [d, d]
        L.orc_zabs.restype = d
        for name in ("orc_dgetrf", "orc_zgetrf"):
            getattr(L, name).argtypes = [i, i, P, i, i, P, C.POINTER(LuInfo)]
        for name in ("orc_dgetrs", "orc_zgetrs"):
            getattr(L, name).argtypes = [i, i, P, i, P, i, P, i, i]
        for name in ("orc_dnormest_power", "orc_znormest_power"):
            getattr(L, name).argtypes = [i, P, i, i, i, i, i, C.POINTER(NormestResult)]
        for name in ("orc_dgecon", "orc_zgecon"):
            getattr(L, name).argtypes = [i, P, i, P, i, d, C.POINTER(d)]
        for name in ("orc_dexpm", "orc_zexpm"):
            getattr(L, name).argtypes = [i, P, i, P, i, C.POINTER(ExpmInfo)]
        for name in ("orc_dexpmv", "orc_zexpmv"):
            getattr(L, name).argtypes = [i, P, i, i, P, i, d, P, i, C.POINTER(ExpmvInfo)]
        for name in ("orc_dexpmv_bound", "orc_zexpmv_bound"):
            getattr(L, name).argtypes = [i, P, i, i, P, i, d, d, P, i, C.POINTER(ExpmvInfo)]
        for name in ("orc_dexpmv_params", "orc_zexpmv_params"):
            getattr(L, name).argtypes = [i, P, i, i, d, C.POINTER(ExpmvInfo)]
        for name in ("orc_dtrsolve", "orc_ztrsolve"):
            getattr(L, name).argtypes = [i, i, i, P, i, P, i]
        for name in ("orc_dpanel", "orc_zpanel"):
            getattr(L, name).argtypes = [i, i, i, P, i, P, i, P, i]
        _lib = L
    return _lib


def _f(a, dtype):
    return np.asfortranarray(a, dtype=dtype)


def _ld(a):
    return max(1, a.shape[0])


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return lib().orc_get_threads()


class NetRandom:
    """.NET System.Random(seed): Next(max) and NextDouble()."""

    def __init__(self, seed: int):
        self._h = C.c_void_p(lib().orc_random_new(int(seed)))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_random_free(self._h)
            self._h = None

    def next(self, max_value: int) -> int:
        return lib().orc_random_next(self._h, int(max_value))

    def next_double(self) -> float:
        return lib().orc_random_next_double(self._h)


def net_sort(keys, items):
    k = np.ascontiguousarray(keys, dtype=np.float64).copy()
    v = np.ascontiguousarray(items, dtype=np.int32).copy()
    lib().orc_sort_keys_items(len(k), _p(k), _p(v))
    return k, v


def gemm(a, b, c=None, alpha=1.0, beta=0.0, multithreaded=True):
    """C := beta*C + alpha*A*B with the reference's blocking semantics."""
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b) or (c is not None and np.iscomplexobj(c)) \
        or isinstance(alpha, complex) or isinstance(beta, complex)
    dt = np.complex128 if cplx else np.float64
    a, b = _f(a, dt), _f(b, dt)
    m, k = a.shape
    k2, n = b.shape
    assert k == k2
    c = np.zeros((m, n), dtype=dt, order="F") if c is None else _f(c, dt).copy(order="F")
    if cplx:
        al = np.array([complex(alpha).real, complex(alpha).imag])
        be = np.array([complex(beta).real, complex(beta).imag])
        rc = lib().orc_zgemm(m, n, k, _p(al), _p(a), _ld(a), _p(b), _ld(b), _p(be), _p(c), _ld(c),
                             int(multithreaded))
    else:
        rc = lib().orc_dgemm(m, n, k, float(alpha), _p(a), _ld(a), _p(b), _ld(b), float(beta),
                             _p(c), _ld(c), int(multithreaded))
    assert rc == 0
    return c


def norm1(a):
    a = np.asfortranarray(a)
    m, n = a.shape
    if np.iscomplexobj(a):
        a = _f(a, np.complex128)
        return lib().orc_znorm1(m, n, _p(a), _ld(a))
    a = _f(a, np.float64)
    return lib().orc_dnorm1(m, n, _p(a), _ld(a))


def norminf(a):
    a = np.asfortranarray(a)
    m, n = a.shape
    if np.iscomplexobj(a):
        a = _f(a, np.complex128)
        return lib().orc_znorminf(m, n, _p(a), _ld(a))
    a = _f(a, np.float64)
    return lib().orc_dnorminf(m, n, _p(a), _ld(a))


def zabs(z: complex) -> float:
    return lib().orc_zabs(z.real, z.imag)


def getrf(a, nb=0):
    """LU with partial pivoting. Returns (factors, pivots, info dict)."""
    cplx = np.iscomplexobj(a)
    f = _f(a, np.complex128 if cplx else np.float64).copy(order="F")
    m, n = f.shape
    piv = np.zeros(min(m, n), dtype=np.int32)
    info = LuInfo()
    fn = lib().orc_zgetrf if cplx else lib().orc_dgetrf
    assert fn(m, n, _p(f), _ld(f), int(nb), _p(piv), C.byref(info)) == 0
    return f, piv, {"singular_column": info.singular_column, "smallest_pivot": info.smallest_pivot,
                    "largest_pivot": info.largest_pivot}


def getrs(factors, piv, b, singular_column=-1, adjoint=False):
    cplx = np.iscomplexobj(factors)
    dt = np.complex128 if cplx else np.float64
    f = _f(factors, dt)
    x = _f(b, dt).copy(order="F")
    squeeze = x.ndim == 1
    if squeeze:
        x = x.reshape(-1, 1, order="F")
    n = f.shape[0]
    piv = np.ascontiguousarray(piv, dtype=np.int32)
    fn = lib().orc_zgetrs if cplx else lib().orc_dgetrs
    rc = fn(n, x.shape[1], _p(f), _ld(f), _p(piv), int(singular_column), _p(x), _ld(x), int(adjoint))
    if rc == 2:
        raise ZeroDivisionError("singular factorization")
    return x[:, 0] if squeeze else x


def normest_power(a, power=1, t=2, itmax=5, seed=20260915):
    cplx = np.iscomplexobj(a)
    a = _f(a, np.complex128 if cplx else np.float64)
    out = NormestResult()
    fn = lib().orc_znormest_power if cplx else lib().orc_dnormest_power
    assert fn(a.shape[0], _p(a), _ld(a), int(power), int(t), int(itmax), int(seed), C.byref(out)) == 0
    return out.value, out.iterations, out.products


def gecon(factors, piv, singular_column, anorm):
    cplx = np.iscomplexobj(factors)
    f = _f(factors, np.complex128 if cplx else np.float64)
    piv = np.ascontiguousarray(piv, dtype=np.int32)
    r = C.c_double()
    fn = lib().orc_zgecon if cplx else lib().orc_dgecon
    assert fn(f.shape[0], _p(f), _ld(f), _p(piv), int(singular_column), float(anorm), C.byref(r)) == 0
    return r.value


def expm(a):
    """exp(A). Returns (result, info dict)."""
    cplx = np.iscomplexobj(a)
    dt = np.complex128 if cplx else np.float64
    a = _f(a, dt)
    n = a.shape[0]
    out = np.zeros((n, n), dtype=dt, order="F")
    info = ExpmInfo()
    fn = lib().orc_zexpm if cplx else lib().orc_dexpm
    rc = fn(n, _p(a), _ld(a), _p(out), _ld(out), C.byref(info))
    if rc == 2:
        raise ZeroDivisionError("singular Pade denominator")
    assert rc == 0
    return out, {k: getattr(info, k) for k, _ in ExpmInfo._fields_}


def expmv_bound(a, b, t, bound):
    """exp(tA)B by the matrix-free Expmv (mu = 0, the caller's bound on
    ||A||_1, no estimator), A applied as a dense operator. Returns (result, info dict)."""
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    dt = np.complex128 if cplx else np.float64
    a, b = _f(a, dt), _f(b, dt)
    n, c = b.shape
    out = np.zeros((n, c), dtype=dt, order="F")
    info = ExpmvInfo()
    fn = lib().orc_zexpmv_bound if cplx else lib().orc_dexpmv_bound
    rc = fn(n, _p(a), _ld(a), c, _p(b), _ld(b), float(t), float(bound), _p(out), _ld(out), C.byref(info))
    if rc == 8:
        raise OverflowError("||tA|| too large for the exponential action")
    assert rc == 0
    return out, {k: getattr(info, k) for k, _ in ExpmvInfo._fields_}


def expmv(a, b, t=1.0):
    """exp(tA)B. Returns (result, info dict)."""
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    dt = np.complex128 if cplx else np.float64
    a, b = _f(a, dt), _f(b, dt)
    squeeze = b.ndim == 1
    if squeeze:
        b = b.reshape(-1, 1, order="F")
    n, c = b.shape
    out = np.zeros((n, c), dtype=dt, order="F")
    info = ExpmvInfo()
    fn = lib().orc_zexpmv if cplx else lib().orc_dexpmv
    rc = fn(n, _p(a), _ld(a), c, _p(b), _ld(b), float(t), _p(out), _ld(out), C.byref(info))
    if rc == 8:
        raise OverflowError("||tA|| too large for the exponential action")
    assert rc == 0
    res = out[:, 0] if squeeze else out
    return res, {k: getattr(info, k) for k, _ in ExpmvInfo._fields_}


# Triangular solve kinds, in the kernel seam's order (KernelEntry.cs:98-173).
TRI_KINDS = {"upper": 0, "upper_transposed": 1, "lower": 2, "lower_transposed": 3, "lower_unit": 4,
             "lower_unit_transposed": 5}


def trsolve(kind, a, b):
    """B := T^-1 B (or T^-T B; complex: T^-H B) for the triangle of A named
    by kind. Returns the solution (a new array)."""
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    dt = np.complex128 if cplx else np.float64
    a = _f(a, dt)
    x = _f(b, dt).copy(order="F")
    m, n = x.shape
    fn = lib().orc_ztrsolve if cplx else lib().orc_dtrsolve
    rc = fn(TRI_KINDS[kind], m, n, _p(a), _ld(a), _p(x), _ld(x))
    assert rc == 0, f"no {'complex ' if cplx else ''}{kind} solve"
    return x


def panel(a, x, transposed=False):
    """Y := A X, or A^T X (real) / A^H X (complex) for a panel X."""
    cplx = np.iscomplexobj(a) or np.iscomplexobj(x)
    dt = np.complex128 if cplx else np.float64
    a, x = _f(a, dt), _f(x, dt)
    n, t = x.shape
    y = np.zeros((n, t), dtype=dt, order="F")
    fn = lib().orc_zpanel if cplx else lib().orc_dpanel
    fn(int(transposed), n, t, _p(a), _ld(a), _p(x), _ld(x), _p(y), _ld(y))
    return y


def expmv_params(a, ncols, t=1.0):
    """(m, s) that Expmv selects for A, an ncols-column panel and t, without
    running the recurrence."""
    cplx = np.iscomplexobj(a)
    a = _f(a, np.complex128 if cplx else np.float64)
    info = ExpmvInfo()
    fn = lib().orc_zexpmv_params if cplx else lib().orc_dexpmv_params
    rc = fn(a.shape[0], _p(a), _ld(a), int(ncols), float(t), C.byref(info))
    if rc == 8:
        raise OverflowError("||tA|| too large for the exponential action")
    assert rc == 0
    return info.degree, info.scaling
