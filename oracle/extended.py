"""exp(A) in extended precision: the truth both GPU forms are measured against.

numpy's long double on x86-64 is the 80-bit format, a 64-bit significand
(unit roundoff 2^-64, 2^11 below FP64's). The exponential is computed by
scaling and squaring with a Taylor polynomial: A / 2^s with ||A/2^s||_1 <= 2,
the Taylor series to degree 40 in Horner form (truncation below 2^41/41!,
under 1e-36), then s squarings. A rounding error made before the squarings
grows about twofold per squaring on these matrices, so the scaling is kept
close to the one Al-Mohy and Higham's algorithm takes (||A/2^s|| near 5.4):
at most two squarings more. Every step is in long double, so the result
carries about 2^-11 x 4 = 2^-9 of the rounding error of an FP64 computation
of the same matrix. This is test infrastructure, run on the host only: the
tests and the benchmark's accuracy check measure the GPU forms against it.
"""
from __future__ import annotations

import math

import numpy as np

DEGREE = 40


def has_extended_precision() -> bool:
    """True when numpy's long double has a 64-bit significand."""
    return np.finfo(np.longdouble).nmant >= 63


def expm_extended(a: np.ndarray, target: float = 2.0) -> np.ndarray:
    """exp(a) computed in long double; returned in long double (complex or
    real, as a). `target` bounds ||A/2^s||_1 (a smaller one adds squarings;
    the tests use it to check the result's own accuracy)."""
    dt = np.clongdouble if np.iscomplexobj(a) else np.longdouble
    x = np.asarray(a).astype(dt)
    n = x.shape[0]
    if n == 0:
        return x.copy()
    norm = float(np.abs(x).sum(axis=0).max())
    s = 0 if norm <= target else int(math.ceil(math.log2(norm / target)))
    x = x * dt(np.ldexp(np.longdouble(1), -s))  # a power of two: exact
    eye = np.eye(n, dtype=dt)
    # Horner: T = I + X (I + X/2 (I + X/3 (... (I + X/DEGREE))))
    t = eye.copy()
    for k in range(DEGREE, 0, -1):
        t = eye + (x @ t) / dt(k)
    for _ in range(s):
        t = t @ t
    return t


def rel1_extended(x: np.ndarray, truth: np.ndarray) -> float:
    """||x - truth||_1 / ||truth||_1, the difference taken in long double."""
    dt = np.clongdouble if np.iscomplexobj(truth) or np.iscomplexobj(x) else np.longdouble
    d = np.asarray(x).astype(dt) - truth.astype(dt)
    num = np.abs(d).sum(axis=0).max()
    den = np.abs(truth).sum(axis=0).max()
    return float(num / den)
