"""Pure-Python big-integer reference for tiny cases (TEST INFRASTRUCTURE ONLY).

An implementation independent of the C oracle (no Montgomery arithmetic, no
shared code) used to cross-check it: the O(n^2) DFT definition of the NTT and
affine double-and-add on y^2 = x^3 + 3.  Values are canonical Python ints;
helpers convert to / from the 4 x u64 Montgomery limb layout
(cuda/bn256.h:10-13, src/lib.rs:22-35).
"""
from __future__ import annotations

R_MOD = 21888242871839275222246405745257275088548364400416034343698204186575808495617
Q_MOD = 21888242871839275222246405745257275088696311157297823662689037894645226208583
MONT_R = 1 << 256
GEN = 7  # multiplicative generator of Fr*


def limbs_to_int(limbs) -> int:
    return sum(int(v) << (64 * i) for i, v in enumerate(list(limbs)))


def int_to_limbs(x: int, words: int = 4):
    return [(x >> (64 * i)) & (2**64 - 1) for i in range(words)]


def mont_to_int(limbs, p=R_MOD) -> int:
    return limbs_to_int(limbs) * pow(MONT_R, -1, p) % p


def int_to_mont(x: int, p=R_MOD):
    return int_to_limbs(x * MONT_R % p)


def root_of_unity(log_n: int) -> int:
    """primitive 2^log_n-th root: 7^((r-1)/2^28) squared (28 - log_n) times"""
    w = pow(GEN, (R_MOD - 1) >> 28, R_MOD)
    for _ in range(28 - log_n):
        w = w * w % R_MOD
    return w


def dft(a: list[int], w: int) -> list[int]:
    n = len(a)
    return [sum(a[i] * pow(w, i * k, R_MOD) for i in range(n)) % R_MOD for k in range(n)]


# ---- affine G1 over Fq, identity None ---------------------------------------
def g1_add(P, Q):
    if P is None:
        return Q
    if Q is None:
        return P
    (x1, y1), (x2, y2) = P, Q
    if x1 == x2:
        if (y1 + y2) % Q_MOD == 0:
            return None
        lam = 3 * x1 * x1 * pow(2 * y1, -1, Q_MOD) % Q_MOD
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, Q_MOD) % Q_MOD
    x3 = (lam * lam - x1 - x2) % Q_MOD
    return (x3, (lam * (x1 - x3) - y1) % Q_MOD)


def g1_mul(P, k: int):
    acc = None
    for bit in bin(k % R_MOD)[2:] if k % R_MOD else "":
        acc = g1_add(acc, acc)
        if bit == "1":
            acc = g1_add(acc, P)
    return acc


def msm(scalars: list[int], points: list) -> object:
    acc = None
    for s, P in zip(scalars, points):
        acc = g1_add(acc, g1_mul(P, s))
    return acc


def point_to_limbs(P):
    """affine point -> 8 Montgomery limbs, identity as (0, 0)"""
    if P is None:
        return [0] * 8
    return int_to_mont(P[0], Q_MOD) + int_to_mont(P[1], Q_MOD)


def limbs_to_point(limbs):
    limbs = [int(v) for v in limbs]
    if all(v == 0 for v in limbs):
        return None
    return (mont_to_int(limbs[:4], Q_MOD), mont_to_int(limbs[4:8], Q_MOD))
