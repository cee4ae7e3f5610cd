"""Algorithmic work model of the three-center contraction (for roofline reports).

A unit of work is one surviving (bra primitive pair, auxiliary primitive)
combination of a shell triplet that passes the Schwarz test. With
L = lab + lc, NH = (lab+1)(lab+2)(lab+3)/6 Hermite components of the bra and
NC = 2 lc + 1 auxiliary functions, its floating-point operations are counted as

  boys  = 20 (L + 1)                       Boys values F_0..F_L
  R     = 3 sum_(n<L) (ncum(L - n) - 1)    Hermite Coulomb recurrence
  X     = 2 NH NC nnz(lc)                  solid-harmonic contraction of R
  G     = 2 nd NH NC                       density-folded bra times X

with nnz(lc) the average number of Cartesian terms of a real solid harmonic of
degree lc. The same counts are used by bench.py's roofline line; the spherical
integral count of the metric is (2la+1)(2lb+1)(2lc+1) per surviving shell
triplet.
"""

import numpy as np

from .common.shells import Shells


def ncum(l):
    return (l + 1) * (l + 2) * (l + 3) // 6 if l >= 0 else 0


# average nonzeros per row of the real solid harmonics (m = -l..l) of degree l
NNZ = {0: 1.0, 1: 1.0, 2: 1.6, 3: 16 / 7, 4: 28 / 9, 5: 46 / 11, 6: 70 / 13}


def triple_flops(lab, lc, nd):
    L = lab + lc
    NH, NC = ncum(lab), 2 * lc + 1
    boys = 20 * (L + 1)
    R = 3 * sum(ncum(L - n) - 1 for n in range(L))
    X = 2 * NH * NC * NNZ[lc]
    G = 2 * nd * NH * NC
    return boys + R + X + G


def model(shells: Shells, shells_aux: Shells, q_bra, q_aux, nd, thresh=float(np.float32(1e-10)),
          chunk=20000):
    """(flops of the 3c contraction, surviving shell triplets, spherical integrals).

    Shell pairs are processed in chunks so that the pair x aux-shell test
    arrays stay small at large systems."""
    n = len(shells)
    La = np.array([s.L for s in shells])
    Pa = np.array([s.nprims for s in shells])
    Lc = np.array([s.L for s in shells_aux])
    Pc = np.array([s.nprims for s in shells_aux])
    ia, ib = np.tril_indices(n)
    qb_all = np.asarray(q_bra)  # packed a(a+1)/2 + b, which is tril order (row-major)
    qa = np.asarray(q_aux)
    flops = 0.0
    ntrip = 0
    nints = 0
    for p0 in range(0, len(ia), chunk):
        sl = slice(p0, p0 + chunk)
        a_, b_ = ia[sl], ib[sl]
        qb = qb_all[sl]
        lab = La[a_] + La[b_]
        units = Pa[a_] * Pa[b_]
        nab = (2 * La[a_] + 1) * (2 * La[b_] + 1)
        for lc in np.unique(Lc):
            sel = Lc == lc
            qc = qa[sel]
            pc = Pc[sel]
            surv = (qb[:, None] * qc[None, :]) >= thresh
            per_pair_trip = surv.sum(axis=1)
            per_pair_prim = (surv * pc[None, :]).sum(axis=1)
            ntrip += int(per_pair_trip.sum())
            nints += int((nab * per_pair_trip).sum() * (2 * lc + 1))
            for l in np.unique(lab):
                m = lab == l
                flops += triple_flops(int(l), int(lc), nd) * float((units[m] * per_pair_prim[m]).sum())
    return flops, ntrip, nints
