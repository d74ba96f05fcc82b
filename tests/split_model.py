"""A numpy model of the split-precision product (csrc/ozaki.cu): the same
exponents, 8-bit slices, exact integer sums per weight 2^(-7 d), FP64
summation from the smallest weight to the largest, and power-of-two scaling.
The GPU kernel must reproduce it bit for bit; its accuracy against the FP64
product is checked separately."""
import numpy as np


def _exponents(mags):
    # least e with every |x| < 2^e: frexp gives m = f 2^e with f in [0.5, 1)
    return np.where(mags > 0, np.frexp(mags)[1], 0).astype(np.int64)


def _slices(x, e, S):
    x = np.ldexp(x, -e)
    out = []
    for _ in range(S):
        x = x * 128.0
        t = np.trunc(x)
        x = x - t
        out.append(t.astype(np.int64))
    return out


def split_product(a, b, S):
    a = np.asarray(a)
    b = np.asarray(b)
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    m, k = a.shape
    n = b.shape[1]
    if cplx:
        a = a.astype(np.complex128)
        b = b.astype(np.complex128)
        left = np.concatenate([a.real, a.imag], axis=1)                       # m x 2k
        right = np.empty((2 * n, 2 * k))
        right[0::2, :k], right[0::2, k:] = b.real.T, -b.imag.T
        right[1::2, :k], right[1::2, k:] = b.imag.T, b.real.T
        ea = _exponents(np.maximum(np.abs(a.real), np.abs(a.imag)).max(axis=1, initial=0.0))
        eb = _exponents(np.maximum(np.abs(b.real), np.abs(b.imag)).max(axis=0, initial=0.0))
        eb_rows = np.repeat(eb, 2)
    else:
        left = a.astype(np.float64)
        right = b.astype(np.float64).T
        ea = _exponents(np.abs(left).max(axis=1, initial=0.0))
        eb = _exponents(np.abs(right).max(axis=1, initial=0.0))
        eb_rows = eb
    sa = _slices(left, ea[:, None], S)
    sb = _slices(right, eb_rows[:, None], S)
    acc = None
    for d in range(S + 1, 1, -1):
        p = np.zeros((m, right.shape[0]), dtype=np.int64)
        for s in range(max(1, d - S), min(S, d - 1) + 1):
            p += sa[s - 1] @ sb[d - s - 1].T
        x = p.astype(np.float64) * 2.0 ** (-7 * d)
        acc = x if acc is None else acc + x
    out = np.ldexp(acc, ea[:, None] + eb_rows[None, :])
    if cplx:
        return out[:, 0::2] + 1j * out[:, 1::2]
    return out
