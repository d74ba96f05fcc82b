"""tensile_b200: the Tensile dense hot path on B200 (sm_100a).

A host-side mirror of the reference library's public surface for the hot path
(src/Tensile: Workspace.Multiply, FactorLu / LuDecomposition<T>.Solve /
SolveAdjoint / Determinant / ReciprocalCondition, NormEstimate.Of over dense
power operators, MatrixExponential.Expm, MatrixExponentialAction.Expmv),
calling the CUDA library through its C ABI. Matrices are numpy arrays
(float64 or complex128); they are read in column-major order, as Matrix<T>
stores them.

Errors map to the reference's exceptions:
  ArgumentException            -> ValueError
  ArgumentNullException        -> ValueError
  ArgumentOutOfRangeException  -> OverflowError / ValueError
  InvalidOperationException    -> SingularMatrixError (singular factorization)
  AllocationLimitException     -> AllocationLimitError
  ObjectDisposedException      -> ObjectDisposedError
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N

__all__ = [
    "Workspace", "LuDecomposition", "NormEstimateResult", "ExpmDiagnostics", "ExpmvDiagnostics",
    "SingularMatrixError", "AllocationLimitError", "ObjectDisposedError", "DeviceTimeoutError",
    "DEFAULT_SEED", "DEFAULT_COLUMNS", "DEFAULT_MAX_ITERATIONS",
]

DEFAULT_COLUMNS = 2          # NormEstimate.DefaultColumns
DEFAULT_MAX_ITERATIONS = 5   # NormEstimate.DefaultMaxIterations
DEFAULT_SEED = 20260915      # NormEstimate.DefaultSeed


class SingularMatrixError(ArithmeticError):
    """InvalidOperationException for an exactly singular factorization."""


class AllocationLimitError(MemoryError):
    """AllocationLimitException: a request exceeds TensileLimits.MaxElements."""


class ObjectDisposedError(RuntimeError):
    """ObjectDisposedException: the workspace has been disposed."""


class DeviceTimeoutError(RuntimeError):
    """A bounded device-side wait gave up; the context stays usable."""


def _raise(code: int, msg: str):
    if code == N.TNS_E_ARGUMENT or code == N.TNS_E_NULL:
        raise ValueError(msg)
    if code == N.TNS_E_SINGULAR:
        raise SingularMatrixError(msg)
    if code == N.TNS_E_ALLOCATION_LIMIT:
        raise AllocationLimitError(msg)
    if code == N.TNS_E_OUT_OF_RANGE:
        raise OverflowError(msg)
    if code == N.TNS_E_DISPOSED:
        raise ObjectDisposedError(msg)
    if code == N.TNS_E_TIMEOUT:
        raise DeviceTimeoutError(msg)
    if code == N.TNS_E_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise RuntimeError(f"tensile_b200 error {code}: {msg}")


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _fortran(a, complex_: bool):
    return np.asfortranarray(a, dtype=np.complex128 if complex_ else np.float64)


def _ld(a: np.ndarray) -> int:
    return max(1, a.shape[0])


@dataclass(frozen=True)
class NormEstimateResult:
    """NormEstimateResult(Value, Iterations, Products)."""
    value: float
    iterations: int
    products: int


@dataclass
class ExpmDiagnostics:
    degree: int = 0
    squarings: int = 0


@dataclass
class ExpmvDiagnostics:
    degree: int = 0
    scaling: int = 0
    applications: int = 0
    early_exits: int = 0


class Workspace:
    """One CUDA stream plus the device buffers of one workspace
    (src/Tensile/Workspace.cs). Operations on one workspace are serialised."""

    def __init__(self, device: int = 0, max_elements: int | None = None):
        self._lib = N.load()
        h = C.c_void_p()
        rc = self._lib.tns_create(int(device), int(max_elements or 0), C.byref(h))
        if rc != N.TNS_OK:
            _raise(rc, self._lib.tns_last_error(None).decode())
        self._h = h

    # -- plumbing -----------------------------------------------------------
    def _call(self, name, *args):
        if self._h is None:
            raise ObjectDisposedError("The workspace has been disposed.")
        rc = getattr(self._lib, name)(self._h, *args)
        if rc != N.TNS_OK:
            _raise(rc, self._lib.tns_last_error(self._h).decode())

    def dispose(self):
        if getattr(self, "_h", None) is not None:
            self._lib.tns_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.dispose()

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_max_elements(self, value: int):
        self._call("tns_set_max_elements", int(value))

    # -- diagnostics --------------------------------------------------------
    def stats(self) -> dict:
        s = N.Stats()
        self._call("tns_get_stats", C.byref(s))
        return {k: getattr(s, k) for k, _ in N.Stats._fields_}

    def set_lu_timing(self, enabled: bool):
        """Collect the blocked LU's per-phase device times (LuPhaseTimings)."""
        self._call("tns_set_lu_timing", int(bool(enabled)))

    def lu_timings(self) -> dict:
        """Summed per-phase times (ms) of the LUs timed since the last reset:
        panel, swaps, triangular, gemm, total, unattributed; block steps and
        factorizations."""
        t = N.LuTimings()
        self._call("tns_get_lu_timings", C.byref(t))
        return {k: getattr(t, k) for k, _ in N.LuTimings._fields_}

    def reset_stats(self):
        self._call("tns_reset_stats")

    def set_workers(self, workers: int):
        """How many matrices of a batch run concurrently (streams)."""
        self._call("tns_set_workers", int(workers))

    def set_timing(self, enabled: bool):
        self._call("tns_set_timing", int(bool(enabled)))

    @property
    def stream(self) -> int:
        """The cudaStream_t this workspace issues its work on."""
        s = C.c_void_p()
        self._call("tns_get_stream", C.byref(s))
        return s.value or 0

    def expm_batched_device(self, count, orders, a_ptrs, lds, out_ptrs, ldos):
        """Batched complex exp over device-resident matrices (raw device
        pointers, e.g. from torch tensors). Returns the diagnostics."""
        orders_c = (C.c_int * count)(*orders)
        lda_c = (C.c_int * count)(*lds)
        ldo_c = (C.c_int * count)(*ldos)
        ap = (C.c_void_p * count)(*a_ptrs)
        op = (C.c_void_p * count)(*out_ptrs)
        infos = (N.ExpmInfo * count)()
        self._call("tns_zexpm_batched_device", count, orders_c, ap, lda_c, op, ldo_c, infos)
        return [ExpmDiagnostics(i.degree, i.squarings) for i in infos]

    def expm_batched_host(self, count, orders, a_ptrs, lds, out_ptrs, ldos):
        """Batched complex exp over host buffers given by address (pinned or
        pageable); the copies to and from the device happen inside the call."""
        orders_c = (C.c_int * count)(*orders)
        lda_c = (C.c_int * count)(*lds)
        ldo_c = (C.c_int * count)(*ldos)
        ap = (C.c_void_p * count)(*a_ptrs)
        op = (C.c_void_p * count)(*out_ptrs)
        infos = (N.ExpmInfo * count)()
        self._call("tns_zexpm_batched", count, orders_c, ap, lda_c, op, ldo_c, infos)
        return [ExpmDiagnostics(i.degree, i.squarings) for i in infos]

    # -- products -----------------------------------------------------------
    def multiply(self, a, b, c=None, alpha=1.0, beta=0.0):
        """C := beta*C + alpha*A*B (Workspace.Multiply). Returns C."""
        cplx = any(np.iscomplexobj(x) for x in (a, b, c) if x is not None) or \
            isinstance(alpha, complex) or isinstance(beta, complex)
        a, b = _fortran(a, cplx), _fortran(b, cplx)
        if a.ndim != 2 or b.ndim != 2:
            raise ValueError("operands must be matrices")
        m, k = a.shape
        k2, n = b.shape
        if k != k2:
            raise ValueError(f"Inner dimensions disagree: A is {m}x{k}, B is {k2}x{n}.")
        if c is None:
            c = np.zeros((m, n), dtype=a.dtype, order="F")
        else:
            c = _fortran(c, cplx).copy(order="F")
            if c.shape != (m, n):
                raise ValueError(f"Destination is {c.shape[0]}x{c.shape[1]}, expected {m}x{n}.")
        if cplx:
            al = np.array([complex(alpha).real, complex(alpha).imag])
            be = np.array([complex(beta).real, complex(beta).imag])
            self._call("tns_zgemm", m, n, k, _p(al), _p(a), _ld(a), _p(b), _ld(b), _p(be), _p(c), _ld(c))
        else:
            self._call("tns_dgemm", m, n, k, float(alpha), _p(a), _ld(a), _p(b), _ld(b), float(beta),
                       _p(c), _ld(c))
        return c

    def multiply_split(self, a, b, moduli: int = 20):
        """A*B in the split-precision form: t-bit integer images of the
        operands (power-of-two row and column scales), their residues modulo
        `moduli` coprime moduli multiplied on the 8-bit tensor cores, the
        product rebuilt by the Chinese remainder theorem. Returns a new matrix."""
        cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
        a, b = _fortran(a, cplx), _fortran(b, cplx)
        if a.ndim != 2 or b.ndim != 2:
            raise ValueError("operands must be matrices")
        m, k = a.shape
        k2, n = b.shape
        if k != k2:
            raise ValueError(f"Inner dimensions disagree: A is {m}x{k}, B is {k2}x{n}.")
        c = np.zeros((m, n), dtype=a.dtype, order="F")
        name = "tns_zgemm_split" if cplx else "tns_dgemm_split"
        self._call(name, m, n, k, _p(a), _ld(a), _p(b), _ld(b), _p(c), _ld(c), int(moduli))
        return c

    def set_split_moduli(self, moduli: int):
        """0: Expm entirely in plain FP64 (the reference's rounding); 8..22: its
        Pade-evaluation and squaring products in the split-precision form."""
        self._call("tns_set_split_moduli", int(moduli))

    # -- norms --------------------------------------------------------------
    def _norm(self, a, kind: bytes) -> float:
        cplx = np.iscomplexobj(a)
        a = _fortran(a, cplx)
        out = C.c_double()
        self._call("tns_znorm" if cplx else "tns_dnorm", kind, a.shape[0], a.shape[1], _p(a), _ld(a),
                   C.byref(out))
        return out.value

    def one_norm(self, a) -> float:
        return self._norm(a, b"1")

    def infinity_norm(self, a) -> float:
        return self._norm(a, b"I")

    def frobenius_norm(self, a) -> float:
        return self._norm(a, b"F")

    # -- the kernel seam's primitives ------------------------------------------
    _SOLVES = {
        (False, "upper"): "tns_dsolve_upper", (False, "upper_transposed"): "tns_dsolve_upper_transposed",
        (False, "lower"): "tns_dsolve_lower", (False, "lower_transposed"): "tns_dsolve_lower_transposed",
        (False, "lower_unit"): "tns_dsolve_lower_unit",
        (False, "lower_unit_transposed"): "tns_dsolve_lower_unit_transposed",
        (True, "upper"): "tns_zsolve_upper", (True, "upper_transposed"): "tns_zsolve_upper_adjoint",
        (True, "lower_unit"): "tns_zsolve_lower_unit", (True, "lower_unit_transposed"): "tns_zsolve_lower_unit_adjoint",
    }

    def solve_triangular(self, kind: str, a, b):
        """X := T^-1 B (kind "upper", "lower", "lower_unit") or T^-T B
        ("..._transposed"; complex: T^-H B) for the triangle T of square A
        (KernelEntry.Solve* / Structures.cs's triangular structures). Returns X."""
        cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
        name = self._SOLVES.get((cplx, kind))
        if name is None:
            raise ValueError(f"no {'complex ' if cplx else ''}{kind} triangular solve")
        a = _fortran(a, cplx)
        x = _fortran(b, cplx).copy(order="F")
        vec = x.ndim == 1
        if vec:
            x = x.reshape(-1, 1, order="F")
        if a.ndim != 2 or a.shape[0] != a.shape[1]:
            raise ValueError(f"The triangle must be square, got {a.shape}.")
        if x.shape[0] != a.shape[0]:
            raise ValueError(f"B has {x.shape[0]} rows, expected {a.shape[0]}.")
        self._call(name, a.shape[0], x.shape[1], _p(a), _ld(a), _p(x), _ld(x))
        return x[:, 0] if vec else x

    def multiply_panel(self, a, x, transposed: bool = False):
        """Y := A X, or A^T X (A^H X for complex) for a panel X
        (KernelEntry.MultiplyPanel / MultiplyPanelTransposed; the complex dense
        operator's Apply / ApplyAdjoint)."""
        cplx = np.iscomplexobj(a) or np.iscomplexobj(x)
        a, x = _fortran(a, cplx), _fortran(x, cplx)
        if a.ndim != 2 or a.shape[0] != a.shape[1] or x.ndim != 2 or x.shape[0] != a.shape[0]:
            raise ValueError("A must be square and X must have A's number of rows")
        n, t = x.shape
        y = np.zeros((n, t), dtype=x.dtype, order="F")
        name = ("tns_zmultiply_panel_adjoint" if transposed else "tns_zmultiply_panel") if cplx else \
            ("tns_dmultiply_panel_transposed" if transposed else "tns_dmultiply_panel")
        self._call(name, n, t, _p(a), _ld(a), _p(x), _ld(x), _p(y), _ld(y))
        return y

    # -- LU -----------------------------------------------------------------
    def factor_lu(self, a, block_size: int = 0) -> "LuDecomposition":
        """P*A = L*U with partial pivoting (Workspace.FactorLu)."""
        cplx = np.iscomplexobj(a)
        f = _fortran(a, cplx).copy(order="F")
        if f.ndim != 2:
            raise ValueError("a matrix is required")
        m, n = f.shape
        piv = np.zeros(min(m, n), dtype=np.int32)
        info = N.LuInfo()
        self._call("tns_zgetrf" if cplx else "tns_dgetrf", m, n, _p(f), _ld(f), int(block_size), _p(piv),
                   C.byref(info))
        return LuDecomposition(self, f, piv, info)

    # -- estimation ---------------------------------------------------------
    def estimate_power_norm(self, a, power: int = 1, columns: int = DEFAULT_COLUMNS,
                            max_iterations: int = DEFAULT_MAX_ITERATIONS,
                            seed: int = DEFAULT_SEED) -> NormEstimateResult:
        """NormEstimate.Of(new DenseMatrixOperator(a, power), ...): a lower
        bound on ||A^power||_1 without forming the power."""
        cplx = np.iscomplexobj(a)
        a = _fortran(a, cplx)
        if a.shape[0] != a.shape[1]:
            raise ValueError(f"A linear operator must be square, got {a.shape[0]}x{a.shape[1]}.")
        out = N.NormestResult()
        self._call("tns_znormest1_power" if cplx else "tns_dnormest1_power", a.shape[0], _p(a), _ld(a),
                   int(power), int(columns), int(max_iterations), int(seed), C.byref(out))
        return NormEstimateResult(out.value, out.iterations, out.products)

    def estimate_operator_norm(self, apply, adjoint, n: int, complex_: bool = False,
                               columns: int = DEFAULT_COLUMNS, max_iterations: int = DEFAULT_MAX_ITERATIONS,
                               seed: int = DEFAULT_SEED) -> NormEstimateResult:
        """NormEstimate.Of(IAdjointOperator<T>, ...) for a matrix-free operator:
        apply(x_ptr, y_ptr, ncols, ld, stream) writes y := A x and
        adjoint(...) writes y := A^H x on device panels."""
        failure = []

        def wrap(fn):
            def trampoline(user, ncols, x, y, ld, stream):
                try:
                    fn(x, y, ncols, ld, stream)
                    return 0
                except BaseException as e:  # reported as TNS_E_OPERATOR, then re-raised below
                    failure.append(e)
                    return 1
            return N.APPLY_FN(trampoline)

        ap, ad = wrap(apply), wrap(adjoint)
        out = N.NormestResult()
        try:
            self._call("tns_znormest1_operator" if complex_ else "tns_dnormest1_operator", int(n), ap, ad, None,
                       int(columns), int(max_iterations), int(seed), C.byref(out))
        except Exception:
            if failure:
                raise failure[0]
            raise
        return NormEstimateResult(out.value, out.iterations, out.products)

    # -- exponentials -------------------------------------------------------
    def expm(self, a, diagnostics: ExpmDiagnostics | None = None):
        """exp(A) (MatrixExponential.Expm)."""
        cplx = np.iscomplexobj(a)
        a = _fortran(a, cplx)
        if a.ndim != 2 or a.shape[0] != a.shape[1]:
            raise ValueError(f"The matrix exponential requires a square matrix, got {a.shape}.")
        n = a.shape[0]
        out = np.zeros((n, n), dtype=a.dtype, order="F")
        info = N.ExpmInfo()
        self._call("tns_zexpm" if cplx else "tns_dexpm", n, _p(a), _ld(a), _p(out), _ld(out), C.byref(info))
        if diagnostics is not None:
            diagnostics.degree, diagnostics.squarings = info.degree, info.squarings
        return out

    def expm_batched(self, mats, diagnostics: list | None = None):
        """exp of every complex matrix in `mats` (the frequency-sweep form)."""
        arrs = [_fortran(m, True) for m in mats]
        for m in arrs:
            if m.ndim != 2 or m.shape[0] != m.shape[1]:
                raise ValueError("every matrix must be square")
        outs = [np.zeros_like(m, order="F") for m in arrs]
        cnt = len(arrs)
        orders = (C.c_int * cnt)(*[m.shape[0] for m in arrs])
        lds = (C.c_int * cnt)(*[_ld(m) for m in arrs])
        ldo = (C.c_int * cnt)(*[_ld(m) for m in outs])
        ap = (C.c_void_p * cnt)(*[m.ctypes.data for m in arrs])
        op = (C.c_void_p * cnt)(*[m.ctypes.data for m in outs])
        infos = (N.ExpmInfo * cnt)()
        self._call("tns_zexpm_batched", cnt, orders, ap, lds, op, ldo, infos)
        if diagnostics is not None:
            diagnostics.clear()
            diagnostics.extend(ExpmDiagnostics(i.degree, i.squarings) for i in infos)
        return outs

    def expmv(self, a, b, t: float = 1.0, diagnostics: ExpmvDiagnostics | None = None):
        """exp(tA)B (MatrixExponentialAction.Expmv)."""
        cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
        a, b = _fortran(a, cplx), _fortran(b, cplx)
        vec = b.ndim == 1
        if vec:
            b = b.reshape(-1, 1, order="F")
        if a.shape[0] != a.shape[1]:
            raise ValueError(f"The exponential action requires a square matrix, got {a.shape}.")
        if b.shape[0] != a.shape[0]:
            raise ValueError(f"B has {b.shape[0]} rows, expected the operator's order {a.shape[0]}.")
        n, c = b.shape
        out = np.zeros((n, c), dtype=a.dtype, order="F")
        info = N.ExpmvInfo()
        self._call("tns_zexpmv" if cplx else "tns_dexpmv", n, _p(a), _ld(a), c, _p(b), _ld(b), float(t),
                   _p(out), _ld(out), C.byref(info))
        if diagnostics is not None:
            diagnostics.degree, diagnostics.scaling = info.degree, info.scaling
            diagnostics.applications, diagnostics.early_exits = info.applications, info.early_exits
        return out[:, 0] if vec else out

    def expmv_batched(self, mats, panels, t: float = 1.0, diagnostics: list | None = None):
        """exp(t A_k) B_k for every pair (the frequency-sweep form of Expmv):
        every B_k with the same number of columns; the Taylor recurrences of
        all matrices run in one device launch. Returns the results."""
        cplx = any(np.iscomplexobj(m) for m in mats) or any(np.iscomplexobj(b) for b in panels)
        arrs = [_fortran(m, cplx) for m in mats]
        bs = [_fortran(b, cplx) for b in panels]
        if len(arrs) != len(bs):
            raise ValueError("one panel per matrix")
        for m, b in zip(arrs, bs):
            if m.ndim != 2 or m.shape[0] != m.shape[1]:
                raise ValueError("every matrix must be square")
            if b.ndim != 2 or b.shape[0] != m.shape[0]:
                raise ValueError("every panel needs its operator's order of rows")
        ncols = bs[0].shape[1] if bs else 0
        if any(b.shape[1] != ncols for b in bs):
            raise ValueError("every panel must have the same number of columns")
        outs = [np.zeros_like(b, order="F") for b in bs]
        cnt = len(arrs)
        orders = (C.c_int * cnt)(*[m.shape[0] for m in arrs])
        lda = (C.c_int * cnt)(*[_ld(m) for m in arrs])
        ldb = (C.c_int * cnt)(*[_ld(b) for b in bs])
        ldo = (C.c_int * cnt)(*[_ld(o) for o in outs])
        ap = (C.c_void_p * cnt)(*[m.ctypes.data for m in arrs])
        bp = (C.c_void_p * cnt)(*[b.ctypes.data for b in bs])
        op = (C.c_void_p * cnt)(*[o.ctypes.data for o in outs])
        infos = (N.ExpmvInfo * cnt)()
        self._call("tns_zexpmv_batched" if cplx else "tns_dexpmv_batched", cnt, orders, ap, lda, ncols, bp, ldb,
                   float(t), op, ldo, infos)
        if diagnostics is not None:
            diagnostics.clear()
            diagnostics.extend(ExpmvDiagnostics(i.degree, i.scaling, i.applications, i.early_exits) for i in infos)
        return outs

    def expmv_select_batched(self, mats, ncols: int, t: float = 1.0, device: bool = False, orders=None, lds=None):
        """(m, s) that the batched Expmv chooses for every complex matrix, for
        panels of ncols columns, without running the recurrences. mats are
        numpy arrays, or raw device pointers with device=True (orders and lds
        given)."""
        if device:
            count = len(mats)
            ptrs = (C.c_void_p * count)(*mats)
        else:
            arrs = [_fortran(m, True) for m in mats]
            count = len(arrs)
            orders = [m.shape[0] for m in arrs]
            lds = [_ld(m) for m in arrs]
            ptrs = (C.c_void_p * count)(*[m.ctypes.data for m in arrs])
        infos = (N.ExpmvInfo * count)()
        self._call("tns_zexpmv_select_batched_device" if device else "tns_zexpmv_select_batched", count,
                   (C.c_int * count)(*orders), ptrs, (C.c_int * count)(*lds), int(ncols), float(t), infos)
        return [(i.degree, i.scaling) for i in infos]

    def expmv_batched_device(self, count, orders, a_ptrs, lds, ncols, b_ptrs, ldbs, t, out_ptrs, ldos):
        """The batched complex Expmv over device-resident operands (raw device
        pointers). Returns the diagnostics."""
        ic = lambda v: (C.c_int * count)(*v)  # noqa: E731
        pc = lambda v: (C.c_void_p * count)(*v)  # noqa: E731
        infos = (N.ExpmvInfo * count)()
        self._call("tns_zexpmv_batched_device", count, ic(orders), pc(a_ptrs), ic(lds), int(ncols), pc(b_ptrs),
                   ic(ldbs), float(t), pc(out_ptrs), ic(ldos), infos)
        return [ExpmvDiagnostics(i.degree, i.scaling, i.applications, i.early_exits) for i in infos]

    def expmv_operator(self, apply, n: int, b, t: float, one_norm_bound: float, complex_: bool = False,
                       diagnostics: ExpmvDiagnostics | None = None):
        """exp(tA)B for a matrix-free operator (MatrixExponentialAction.Expmv over
        ILinearOperator<T>): apply(x_ptr, y_ptr, ncols, ld, stream) must write
        y := A x for device panels (column-major, leading dimension ld
        elements, complex interleaved) on the given CUDA stream. No trace
        shift; one_norm_bound bounds ||A||_1."""
        cplx = complex_ or np.iscomplexobj(b)
        b = _fortran(b, cplx)
        vec = b.ndim == 1
        if vec:
            b = b.reshape(-1, 1, order="F")
        if b.shape[0] != n:
            raise ValueError(f"B has {b.shape[0]} rows, expected the operator's order {n}.")
        c = b.shape[1]
        out = np.zeros((n, c), dtype=b.dtype, order="F")
        info = N.ExpmvInfo()
        failure = []

        def trampoline(user, ncols, x, y, ld, stream):
            try:
                apply(x, y, ncols, ld, stream)
                return 0
            except BaseException as e:  # reported as TNS_E_OPERATOR, then re-raised below
                failure.append(e)
                return 1

        cb = N.APPLY_FN(trampoline)
        try:
            self._call("tns_zexpmv_operator" if cplx else "tns_dexpmv_operator", n, cb, None, c, _p(b), _ld(b),
                       float(t), float(one_norm_bound), _p(out), _ld(out), C.byref(info))
        except Exception:
            if failure:
                raise failure[0]
            raise
        if diagnostics is not None:
            diagnostics.degree, diagnostics.scaling = info.degree, info.scaling
            diagnostics.applications, diagnostics.early_exits = info.applications, info.early_exits
        return out[:, 0] if vec else out

    # -- differentiation ------------------------------------------------------
    def expm_frechet(self, a, e, diagnostics: ExpmDiagnostics | None = None):
        """(exp(A), L(A, E)): the exponential and its Frechet derivative in the
        direction E (Al-Mohy and Higham's algorithm; no reference counterpart,
        which obtains L(A, E) from Expm of [[A, E], [0, A]])."""
        cplx = np.iscomplexobj(a) or np.iscomplexobj(e)
        a, e = _fortran(a, cplx), _fortran(e, cplx)
        if a.ndim != 2 or a.shape[0] != a.shape[1] or e.shape != a.shape:
            raise ValueError(f"A and E must be square and of one shape, got {a.shape} and {e.shape}.")
        n = a.shape[0]
        x = np.zeros((n, n), dtype=a.dtype, order="F")
        l = np.zeros((n, n), dtype=a.dtype, order="F")
        info = N.ExpmInfo()
        self._call("tns_zexpm_frechet" if cplx else "tns_dexpm_frechet", n, _p(a), _ld(a), _p(e), _ld(e),
                   _p(x), _ld(x), _p(l), _ld(l), C.byref(info))
        if diagnostics is not None:
            diagnostics.degree, diagnostics.squarings = info.degree, info.squarings
        return x, l

    def expmv_gradient(self, a, b, y, t: float = 1.0):
        """loss = ||exp(tA) B - Y||_F^2 and its gradients with respect to A, B
        and t (complex gradients hold d/dRe + i d/dIm). Returns a dict with
        loss, f = exp(tA) B, grad_a, grad_b, grad_t, degree, squarings."""
        cplx = any(np.iscomplexobj(v) for v in (a, b, y))
        a, b, y = _fortran(a, cplx), _fortran(b, cplx), _fortran(y, cplx)
        if a.ndim != 2 or a.shape[0] != a.shape[1]:
            raise ValueError(f"A must be square, got {a.shape}.")
        if b.ndim != 2 or b.shape[0] != a.shape[0] or y.shape != b.shape:
            raise ValueError(f"B and Y must be {a.shape[0]} x c and of one shape, got {b.shape} and {y.shape}.")
        n, c = b.shape
        ga = np.zeros((n, n), dtype=a.dtype, order="F")
        gb = np.zeros((n, c), dtype=a.dtype, order="F")
        f = np.zeros((n, c), dtype=a.dtype, order="F")
        loss, gt = C.c_double(), C.c_double()
        info = N.ExpmInfo()
        self._call("tns_zexpmv_gradient" if cplx else "tns_dexpmv_gradient", n, c, float(t), _p(a), _ld(a),
                   _p(b), _ld(b), _p(y), _ld(y), C.byref(loss), _p(ga), _ld(ga), _p(gb), _ld(gb), C.byref(gt),
                   _p(f), _ld(f), C.byref(info))
        return {"loss": loss.value, "f": f, "grad_a": ga, "grad_b": gb, "grad_t": gt.value,
                "degree": info.degree, "squarings": info.squarings}

    # -- precision form of the solve --------------------------------------------
    def solve_mixed(self, a, b, moduli: int = 0, max_iter: int = 20):
        """A^-1 B by a low-precision LU (trailing updates on the split-precision
        product) and FP64 iterative refinement. Returns (X, info dict)."""
        cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
        a, b = _fortran(a, cplx), _fortran(b, cplx)
        vec = b.ndim == 1
        if vec:
            b = b.reshape(-1, 1, order="F")
        if a.ndim != 2 or a.shape[0] != a.shape[1] or b.shape[0] != a.shape[0]:
            raise ValueError(f"A must be square and B have its order of rows, got {a.shape} and {b.shape}.")
        n, c = b.shape
        x = np.zeros((n, c), dtype=a.dtype, order="F")
        info = N.MixedInfo()
        self._call("tns_zgesv_mixed" if cplx else "tns_dgesv_mixed", n, c, _p(a), _ld(a), _p(b), _ld(b), _p(x),
                   _ld(x), int(moduli), int(max_iter), C.byref(info))
        d = {k: getattr(info, k) for k, _ in N.MixedInfo._fields_}
        return (x[:, 0] if vec else x), d

    def set_autotune(self, enabled: bool):
        """Choose the GEMMs' launch shapes by timing them on each size class's
        first launch (identical results either way)."""
        self._call("tns_set_autotune", int(bool(enabled)))

    def set_checkpoint_bytes(self, nbytes: int):
        """Device bytes the Frechet derivative may hold for its squarings (-1: automatic)."""
        self._call("tns_set_checkpoint_bytes", int(nbytes))


class LuDecomposition:
    """LuDecomposition<T> (src/Tensile/LuDecomposition.cs): packed factors,
    0-based pivots, solves, determinant and reciprocal condition."""

    def __init__(self, ws: Workspace, factors, pivots, info):
        self._ws = ws
        self.factors = factors
        self.pivots = pivots
        self.singular_column = info.singular_column
        self.smallest_pivot = info.smallest_pivot
        self.largest_pivot = info.largest_pivot
        self.one_norm_of_a = info.one_norm

    @property
    def rows(self):
        return self.factors.shape[0]

    @property
    def columns(self):
        return self.factors.shape[1]

    @property
    def is_square(self):
        return self.rows == self.columns

    @property
    def is_singular(self):
        return self.singular_column >= 0

    @property
    def pivot_ratio(self):
        return 0.0 if self.largest_pivot == 0.0 else self.smallest_pivot / self.largest_pivot

    def _solve(self, b, adjoint: bool):
        if not self.is_square:
            raise SingularMatrixError("Solve requires a square factorization.")
        cplx = np.iscomplexobj(self.factors)
        x = _fortran(b, cplx).copy(order="F")
        vec = x.ndim == 1
        if vec:
            x = x.reshape(-1, 1, order="F")
        if x.shape[0] != self.rows:
            raise ValueError(f"Right-hand side has {x.shape[0]} rows, expected {self.rows}.")
        self._ws._call("tns_zgetrs" if cplx else "tns_dgetrs", self.rows, x.shape[1], _p(self.factors),
                       _ld(self.factors), _p(self.pivots), int(self.singular_column), _p(x), _ld(x),
                       int(adjoint))
        return x[:, 0] if vec else x

    def solve(self, b):
        return self._solve(b, False)

    def solve_adjoint(self, b):
        return self._solve(b, True)

    def determinant(self):
        if not self.is_square:
            raise SingularMatrixError("Determinant requires a square factorization.")
        d = np.prod(np.diagonal(self.factors)) if self.rows else (1.0 + 0j if np.iscomplexobj(self.factors) else 1.0)
        swaps = int(np.sum(self.pivots != np.arange(len(self.pivots))))
        return -d if swaps % 2 else d

    def reciprocal_condition(self) -> float:
        """1/(||A||_1 * est ||A^-1||_1), 0 when singular (ReciprocalCondition)."""
        cplx = np.iscomplexobj(self.factors)
        out = C.c_double()
        self._ws._call("tns_zgecon" if cplx else "tns_dgecon", self.rows, _p(self.factors), _ld(self.factors),
                       _p(self.pivots), int(self.singular_column), float(self.one_norm_of_a), C.byref(out))
        return out.value
