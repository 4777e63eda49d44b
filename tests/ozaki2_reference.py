"""Exact restatement of the Ozaki II (CRT) GEMM arithmetic for the tests.

Test infrastructure only: the CRT constants with Python integers, and a numpy
emulation of the device path that must agree with it bit for bit (scaled
integer operands, symmetric residues, exact int products, the FP64 CRT
evaluation on the two binary grids, the final scaling)."""

import math

import numpy as np

MODULI = (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199)


def modulus_product(n):
    return math.prod(MODULI[:n])


def crt_constants(n):
    """Exact CRT constants for the first n moduli."""
    P = modulus_product(n)
    e1 = max(0, (256 * n * P).bit_length() - 53)
    e2 = max(0, e1 + (256 * n).bit_length() - 53)
    w1, w2, frac, y = [], [], [], []
    for p in MODULI[:n]:
        Q = P // p
        yy = pow(Q % p, -1, p)
        W = Q * yy
        W1 = (W >> e1) << e1
        W2 = ((W - W1) >> e2) << e2
        w1.append(float(W1))
        w2.append(float(W2))
        frac.append(np.float32(yy / p))
        y.append(yy)
    P1 = (P >> e1) << e1
    P2 = ((P - P1) >> e2) << e2
    return {"P": P, "e1": e1, "e2": e2, "w1": np.array(w1), "w2": np.array(w2),
            "P1": float(P1), "P2": float(P2), "frac": np.array(frac, dtype=np.float32),
            "y": y}


def operand_bits(n, K):
    L = (modulus_product(n).bit_length() - 1) - 2 - (int(K - 1).bit_length() if K > 1 else 0)
    return min(50, L // 2), min(50, L - L // 2)


def row_exponents(X):
    m = np.abs(X).max(axis=1) if X.shape[1] else np.zeros(X.shape[0])
    e = np.frexp(m)[1].astype(np.int64)
    e[m == 0] = 0
    return e


def sym_residue(Xi, p):
    """Symmetric residue of an int64 array: [-128, 127] for 256, else
    [-(p-1)/2, (p-1)/2]."""
    h = p // 2 if p == 256 else (p - 1) // 2
    return ((Xi + h) % p) - h


def scaled_integers(A, B, n):
    K = A.shape[1]
    a, b = operand_bits(n, K)
    ea = row_exponents(A)
    eb = row_exponents(B.T)
    Ai = np.rint(np.ldexp(A, (a - ea)[:, None])).astype(np.int64)
    Bi = np.rint(np.ldexp(B.T, (b - eb)[:, None])).astype(np.int64)
    return Ai, Bi, ea, eb, a, b


def emulate(A, B, n, alpha=1.0):
    """C = alpha A B through the Ozaki II arithmetic of the device path."""
    Ai, Bi, ea, eb, a, b = scaled_integers(A, B, n)
    c = crt_constants(n)
    res = []
    for p in MODULI[:n]:
        ra = sym_residue(Ai, p).astype(np.float64)
        rb = sym_residue(Bi, p).astype(np.float64)
        acc = np.rint(ra @ rb.T).astype(np.int64)     # exact: |acc| < 2^31
        res.append(sym_residue(acc, p).astype(np.float64))
    kf = sum(r * (y / p) for r, y, p in zip(res, c["y"], MODULI[:n], strict=False))
    k = np.rint(kf)
    d1 = -k * c["P1"]
    d2 = -k * c["P2"]
    for m, r in enumerate(res):
        d1 = d1 + r * c["w1"][m]     # every product and partial sum is exact
        d2 = d2 + r * c["w2"][m]
    x = d1 + d2
    return alpha * np.ldexp(x, ea[:, None] + eb[None, :] - a - b)


def rounding_error_bound(A, B, n):
    """Bound on |C - A B| per entry from rounding A and B to a and b bits."""
    K = A.shape[1]
    a, b = operand_bits(n, K)
    ra = np.abs(A).max(axis=1)[:, None]
    cb = np.abs(B).max(axis=0)[None, :]
    return K * ra * cb * (2.0 ** -(a - 1) + 2.0 ** -(b - 1))
