"""Small numpy reference integrals for tests (test infrastructure).

Overlap integrals between contracted spherical shells by McMurchie-Davidson
E coefficients, used to pin the basis normalization, ordering and phase
conventions against the ORCA overlap matrix of the golden fixture.
"""

from math import factorial

import numpy as np


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def _binom(n, k):
    if k < 0 or k > n:
        return 0
    return factorial(n) // (factorial(k) * factorial(n - k))


def cart_list(l):
    return [(i, j, l - i - j) for i in range(l, -1, -1) for j in range(l - i, -1, -1)]


def solid_harmonics(l):
    """Real solid harmonics (m = -l..l) over cart_list(l), unit-normalized for
    contraction coefficients normalized like common/normalization.f90."""
    carts = cart_list(l)
    T = np.zeros((2 * l + 1, len(carts)))
    for m in range(-l, l + 1):
        am = abs(m)
        N = 1.0 / (2**am * factorial(l)) * np.sqrt(2 * factorial(l + am) * factorial(l - am) / (2 if m == 0 else 1))
        vm2 = 1 if m < 0 else 0
        v2max = 2 * int(np.floor(am / 2 - vm2 / 2)) + vm2
        for t in range((l - am) // 2 + 1):
            for u in range(t + 1):
                for v2 in range(vm2, v2max + 1, 2):
                    c = (-1) ** (t + (v2 - vm2) // 2) * 0.25**t * _binom(l, t) * _binom(l - t, am + t) * _binom(t, u) * _binom(am, v2)
                    key = (2 * t + am - 2 * u - v2, 2 * u + v2, l - 2 * t - am)
                    T[m + l, carts.index(key)] += N * c
        s = 0.0
        for a, ea in enumerate(carts):
            for b, eb in enumerate(carts):
                f = T[m + l, a] * T[m + l, b]
                for d in range(3):
                    n = ea[d] + eb[d]
                    f = 0.0 if n % 2 else f * _dfact(n - 1)
                s += f
        T[m + l] /= np.sqrt(s)
    return T


def norm_coeffs(coeffs, exps, L):
    c = np.array(coeffs, float)
    e = np.array(exps, float)
    lp = L + 1.5
    N = np.sum(np.outer(c, c) / np.add.outer(e, e) ** lp * np.sqrt(np.outer(e, e)) ** lp)
    return c * np.sqrt(e**lp / (np.pi**1.5 / 2**L * N))


def _E(i, j, t, a, b, XAB):
    p = a + b
    q = a * b / p
    if t < 0 or t > i + j:
        return 0.0
    if i == j == t == 0:
        return np.exp(-q * XAB**2)
    if j == 0:
        return (_E(i - 1, j, t - 1, a, b, XAB) / (2 * p) - q * XAB / a * _E(i - 1, j, t, a, b, XAB)
                + (t + 1) * _E(i - 1, j, t + 1, a, b, XAB))
    return (_E(i, j - 1, t - 1, a, b, XAB) / (2 * p) + q * XAB / b * _E(i, j - 1, t, a, b, XAB)
            + (t + 1) * _E(i, j - 1, t + 1, a, b, XAB))


def overlap_block(sa, sb):
    Ta, Tb = solid_harmonics(sa.L), solid_harmonics(sb.L)
    ca, cb = norm_coeffs(sa.coeffs, sa.exps, sa.L), norm_coeffs(sb.coeffs, sb.exps, sb.L)
    A, B = np.asarray(sa.center), np.asarray(sb.center)
    carts_a, carts_b = cart_list(sa.L), cart_list(sb.L)
    S = np.zeros((len(carts_a), len(carts_b)))
    for ka, a in zip(ca, sa.exps):
        for kb, b in zip(cb, sb.exps):
            p = a + b
            for ia, ea in enumerate(carts_a):
                for ib, eb in enumerate(carts_b):
                    v = ka * kb * (np.pi / p) ** 1.5
                    for d in range(3):
                        v *= _E(ea[d], eb[d], 0, a, b, A[d] - B[d])
                    S[ia, ib] += v
    return Ta @ S @ Tb.T


def overlap_matrix(shells):
    offs = shells.sph_offsets()
    n = shells.sph_size
    S = np.zeros((n, n))
    for i, sa in enumerate(shells):
        for j, sb in enumerate(shells):
            S[offs[i]:offs[i] + sa.sph_size, offs[j]:offs[j] + sb.sph_size] = overlap_block(sa, sb)
    return S
