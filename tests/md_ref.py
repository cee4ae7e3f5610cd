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


def schwarz_pair_mp(sa, sb, dps=40):
    """sqrt(||(ab|ab)||_F) of two single-primitive shells in mpmath arithmetic
    (McMurchie-Davidson with mpmath Boys values) -- a high-precision check."""
    import mpmath as mp

    mp.mp.dps = dps
    assert sa.nprims == 1 and sb.nprims == 1

    def E(i, j, t, Qx, a, b):
        p = a + b
        q = a * b / p
        if t < 0 or t > i + j:
            return mp.mpf(0)
        if i == j == t == 0:
            return mp.exp(-q * Qx * Qx)
        if j == 0:
            return E(i - 1, j, t - 1, Qx, a, b) / (2 * p) - (q * Qx / a) * E(i - 1, j, t, Qx, a, b) + (t + 1) * E(i - 1, j, t + 1, Qx, a, b)
        return E(i, j - 1, t - 1, Qx, a, b) / (2 * p) + (q * Qx / b) * E(i, j - 1, t, Qx, a, b) + (t + 1) * E(i, j - 1, t + 1, Qx, a, b)

    al, be = mp.mpf(float(sa.exps[0])), mp.mpf(float(sb.exps[0]))
    ca = mp.mpf(float(norm_coeffs(sa.coeffs, sa.exps, sa.L)[0]))
    cb = mp.mpf(float(norm_coeffs(sb.coeffs, sb.exps, sb.L)[0]))
    A = [mp.mpf(float(x)) for x in sa.center]
    B = [mp.mpf(float(x)) for x in sb.center]
    p = al + be
    Ta, Tb = solid_harmonics(sa.L), solid_harmonics(sb.L)
    cla, clb = cart_list(sa.L), cart_list(sb.L)
    herm = []
    for ma in range(2 * sa.L + 1):
        for mb in range(2 * sb.L + 1):
            d = {}
            for i1, e1 in enumerate(cla):
                for i2, e2 in enumerate(clb):
                    c = mp.mpf(float(Ta[ma, i1])) * mp.mpf(float(Tb[mb, i2]))
                    if c == 0:
                        continue
                    for t in range(e1[0] + e2[0] + 1):
                        for u in range(e1[1] + e2[1] + 1):
                            for v in range(e1[2] + e2[2] + 1):
                                val = c * ca * cb * E(e1[0], e2[0], t, A[0] - B[0], al, be) * E(e1[1], e2[1], u, A[1] - B[1], al, be) * E(e1[2], e2[2], v, A[2] - B[2], al, be)
                                d[(t, u, v)] = d.get((t, u, v), 0) + val
            herm.append(d)
    alpha = p / 2
    # R_tuv(alpha, 0): nonzero for even t, u, v only
    boys = {}

    def F(n):
        if n not in boys:
            boys[n] = mp.mpf(1) / (2 * n + 1)
        return boys[n]

    def R0(t, u, v):
        if t % 2 or u % 2 or v % 2:
            return mp.mpf(0)
        val = mp.mpf(1)
        for k in (t, u, v):
            val *= mp.mpf((-1) ** (k // 2) * _dfact(k - 1))
        n = (t + u + v) // 2
        return val * (2 * alpha) ** n * F(n) * (-1) ** 0

    pref = 2 * mp.pi ** mp.mpf(2.5) / (p * p * mp.sqrt(2 * p))
    tot = mp.mpf(0)
    for dr in herm:
        for ds in herm:
            val = mp.mpf(0)
            for (t, u, v), x in dr.items():
                for (t2, u2, v2), y in ds.items():
                    val += x * y * (-1) ** (t2 + u2 + v2) * R0(t + t2, u + u2, v + v2)
            tot += (pref * val) ** 2
    return float(mp.sqrt(mp.sqrt(tot)))
