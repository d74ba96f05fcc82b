"""An exact model of the split-precision product (csrc/ozaki.cu): the same
power-of-two scales and t-bit integer images A' = rint(A 2^(t-e)),
B' = rint(B 2^(t-f)), their exact integer product (Python integers, no
residues needed), correctly rounded to FP64 and scaled back. The GPU result
rebuilds the same integer product from its residues, so it must agree with
this model to within a few units in the last place; the model's own accuracy
against the FP64 product is checked separately."""
import numpy as np

MODULI = [256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223,
          217, 211, 199, 197, 193, 191, 181, 179, 173, 167, 163]


def integer_bits(nm, kmax):
    """t, the largest with 2 K' 2^(2t) < P (as the library computes it)."""
    P = 1
    for p in MODULI[:nm]:
        P *= p
    L = P.bit_length() - 1
    c = 0
    while (1 << c) < max(1, kmax):
        c += 1
    return min(96, (L - 2 - c) // 2), L


def _exponents(mags):
    # least e with every |x| < 2^e: frexp gives m = f 2^e with f in [0.5, 1)
    return np.where(mags > 0, np.frexp(mags)[1], 0).astype(np.int64)


def _limbs(x):
    """Integer-valued doubles (|x| <= 2^96) as four signed 24-bit limbs."""
    out = []
    for _ in range(4):
        r = np.fmod(x, 2.0 ** 24)
        out.append(r.astype(np.int64))
        x = (x - r) / 2.0 ** 24
    return out


def exact_int_product(left, right):
    """left (m x K) times right^T (n x K), integer-valued doubles, as Python ints."""
    la, lb = _limbs(left), _limbs(right)
    out = np.zeros((left.shape[0], right.shape[0]), dtype=object)
    for i, a in enumerate(la):
        for j, b in enumerate(lb):
            part = (a @ b.T).astype(object)   # |limb products| < 2^48, K' <= 2^11: exact in int64
            out = out + part * (1 << (24 * (i + j)))
    return out


def operands(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    k = a.shape[1]
    n = b.shape[1]
    if cplx:
        a = a.astype(np.complex128)
        b = b.astype(np.complex128)
        left = np.concatenate([a.real, a.imag], axis=1)
        right = np.empty((2 * n, 2 * k))
        right[0::2, :k], right[0::2, k:] = b.real.T, -b.imag.T
        right[1::2, :k], right[1::2, k:] = b.imag.T, b.real.T
        ea = _exponents(np.maximum(np.abs(a.real), np.abs(a.imag)).max(axis=1, initial=0.0))
        eb = np.repeat(_exponents(np.maximum(np.abs(b.real), np.abs(b.imag)).max(axis=0, initial=0.0)), 2)
    else:
        left = a.astype(np.float64)
        right = b.astype(np.float64).T
        ea = _exponents(np.abs(left).max(axis=1, initial=0.0))
        eb = _exponents(np.abs(right).max(axis=1, initial=0.0))
    return cplx, left, right, ea, eb


def split_product(a, b, nm):
    """The model's result and, per entry, the scale 2^(e_i + f_j - 2t) of one
    unit of the integer product."""
    cplx, left, right, ea, eb = operands(a, b)
    t, _ = integer_bits(nm, left.shape[1])
    ai = np.rint(np.ldexp(left, (t - ea)[:, None]))
    bi = np.rint(np.ldexp(right, (t - eb)[:, None]))
    prod = exact_int_product(ai, bi)
    sc = ea[:, None] + eb[None, :] - 2 * t
    out = np.empty(prod.shape)
    for i in range(prod.shape[0]):
        for j in range(prod.shape[1]):
            out[i, j] = np.ldexp(float(prod[i, j]), int(sc[i, j]))
    unit = np.ldexp(1.0, sc)
    if cplx:
        return out[:, 0::2] + 1j * out[:, 1::2], unit[:, 0::2]
    return out, unit
