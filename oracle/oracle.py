"""ctypes front end of the oracle -- test infrastructure, not product code.

Loads ``oracle/liboracle.so`` (a C++ FP64 CPU restatement of the reference's
density-fitting path, see ``oracle.h``) and exposes the reference's Python
entry points over it with the same argument meaning, so parity tests read like
the reference's own tests. Only tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this module.

BLAS/LAPACK: the reference calls dpotrf/dtrtri/dtrmm/dgemm. The oracle gets the
same routines from scipy's bundled OpenBLAS (through ``scipy.linalg.cython_*``
function pointers) when scipy is importable, and falls back to plain loops.
"""

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

_lib = None

_i = ctypes.c_int
_d = ctypes.c_double
_pi = ctypes.POINTER(ctypes.c_int)
_pd = ctypes.POINTER(ctypes.c_double)


class OracleStats(ctypes.Structure):
    _fields_ = [
        ("ntriplets", ctypes.c_longlong),
        ("nskipped", ctypes.c_longlong),
        ("nints", ctypes.c_longlong),
        ("t_screener", ctypes.c_double),
        ("t_metric", ctypes.c_double),
        ("t_chol", ctypes.c_double),
        ("t_3c", ctypes.c_double),
        ("t_trmm", ctypes.c_double),
        ("t_total", ctypes.c_double),
    ]


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _capsule_ptr(capsule):
    get_name = ctypes.pythonapi.PyCapsule_GetName
    get_name.restype = ctypes.c_char_p
    get_name.argtypes = [ctypes.py_object]
    get_ptr = ctypes.pythonapi.PyCapsule_GetPointer
    get_ptr.restype = ctypes.c_void_p
    get_ptr.argtypes = [ctypes.py_object, ctypes.c_char_p]
    return get_ptr(capsule, get_name(capsule))


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    L = ctypes.CDLL(str(LIB_PATH))
    basis = [_i, _i, _pi, _pi, _pd]
    L.oracle_boys.argtypes = [_i, _d, _pd]
    L.oracle_erfinv.argtypes = [_d]
    L.oracle_erfinv.restype = _d
    L.oracle_contracted_center.argtypes = [_i, _pd, _pd, _pd, _i, _pd, _pd, _pd, _pd]
    L.oracle_eri_block.argtypes = [_i, _i, _pd, _pd, _pd] * 4 + [_pd]
    L.oracle_eri_block.restype = _i
    L.oracle_int_schwarz_aux.argtypes = basis + [_pd]
    L.oracle_int_schwarz_bra.argtypes = basis + [_pd]
    L.oracle_int2c2e_metric.argtypes = basis + [_i, _pd]
    L.oracle_contract_coulomb_densities_2d.argtypes = basis + basis + [_i, _i, _pd, _i, _pd]
    L.oracle_contract_coulomb_densities_4d.argtypes = basis + basis + [_i, _i, _pd, _i, _pd]
    L.oracle_intor_eri2c.argtypes = basis + basis + [_i, _pd]
    L.oracle_intor_df1c.argtypes = basis + basis + [_i, _i, _pd]
    L.oracle_intor_df2c_mo.argtypes = basis + basis + [_i, _i, _pd, _i, _pd]
    L.oracle_set_boys_mode.argtypes = [_i]
    L.oracle_get_boys_mode.restype = _i
    L.oracle_set_threads.argtypes = [_i]
    L.oracle_set_skip_metric.argtypes = [_i]
    L.oracle_set_metric_shift.argtypes = [_d]
    L.oracle_set_screening.argtypes = [_i]
    L.oracle_set_reuse_screening.argtypes = [_i]
    L.oracle_get_threads.restype = _i
    L.oracle_register_lapack.argtypes = [ctypes.c_void_p] * 4
    L.oracle_last_stats.argtypes = [ctypes.POINTER(OracleStats)]
    L.oracle_chol_solve_ld.argtypes = [_i, _pd, _i, _pd, _pd, _pd]
    L.oracle_chol_solve_ld.restype = _i
    L.oracle_chol_backward_error_ld.argtypes = [_i, _pd, _pd]
    L.oracle_chol_backward_error_ld.restype = _d
    L.oracle_int3c2e_estimates.argtypes = basis + basis + [ctypes.c_longlong, _pd,
                                                           ctypes.POINTER(ctypes.c_longlong)]
    L.oracle_int3c2e_estimates.restype = ctypes.c_longlong
    L.oracle_eval_densities.argtypes = basis + [_i, _pd, _i, _i, _pd, _pd, _i, _d]
    L.oracle_eval_prim_density.argtypes = [_i, _i, _i, _pi, _pd, _pd, _pd, _d, _pd]
    if os.environ.get("PA_ORACLE_NO_LAPACK", "0") != "1":
        try:
            from scipy.linalg import cython_blas, cython_lapack

            L.oracle_register_lapack(
                _capsule_ptr(cython_lapack.__pyx_capi__["dpotrf"]),
                _capsule_ptr(cython_lapack.__pyx_capi__["dtrtri"]),
                _capsule_ptr(cython_blas.__pyx_capi__["dtrmm"]),
                _capsule_ptr(cython_blas.__pyx_capi__["dgemm"]),
            )
        except ImportError:  # plain loops inside the oracle
            pass
    L.oracle_init()
    _lib = L
    return L


def _p(arr, ctype):
    return arr.ctypes.data_as(ctypes.POINTER(ctype))


def _basis_args(shells):
    bc, bs, bd = shells.as_arrays(fortran=True)
    bc = np.asfortranarray(bc, dtype=np.int32)
    bs = np.asfortranarray(bs, dtype=np.int32)
    bd = np.ascontiguousarray(bd, dtype=np.float64)
    keep = (bc, bs, bd)
    return keep, [len(bc), len(bd), _p(bc, ctypes.c_int), _p(bs, ctypes.c_int), _p(bd, ctypes.c_double)]


def set_boys_mode(mode):
    lib().oracle_set_boys_mode({"exact": 0, "reference": 1}.get(mode, mode))


def get_boys_mode():
    return lib().oracle_get_boys_mode()


def set_skip_metric(skip):
    lib().oracle_set_skip_metric(int(bool(skip)))


def set_metric_shift(shift):
    lib().oracle_set_metric_shift(float(shift))


def set_screening(mode):
    """'schwarz' (default) or 'qvl': the triplet estimate of the Coulomb
    contraction (diabatization/intor.f90:137-138)."""
    lib().oracle_set_screening({"schwarz": 0, "qvl": 1}[mode])


def set_reuse_screening(reuse):
    """Keep the bra Schwarz vector of the last orbital basis for later calls
    with the same basis (timing aid for sampled baselines)."""
    lib().oracle_set_reuse_screening(int(bool(reuse)))


def set_threads(n):
    lib().oracle_set_threads(int(n))


def get_threads():
    return lib().oracle_get_threads()


def last_stats():
    st = OracleStats()
    lib().oracle_last_stats(ctypes.byref(st))
    return {name: getattr(st, name) for name, _ in OracleStats._fields_}


def boys(nmax, x):
    out = np.zeros(nmax + 1)
    lib().oracle_boys(nmax, float(x), _p(out, ctypes.c_double))
    return out


def erfinv(x):
    return lib().oracle_erfinv(float(x))


def contracted_center(axs, das, A, bxs, dbs, B):
    arrs = [np.ascontiguousarray(v, dtype=float) for v in (axs, das, A, bxs, dbs, B)]
    R = np.zeros(3)
    lib().oracle_contracted_center(
        len(arrs[0]), *[_p(a, ctypes.c_double) for a in arrs[:3]],
        len(arrs[3]), *[_p(a, ctypes.c_double) for a in arrs[3:]],
        _p(R, ctypes.c_double),
    )
    return R


def eri_block(a, b=None, c=None, d=None):
    """Contracted spherical block (ab|cd) of Shell objects; None = unit s function."""
    shells = [a, b, c, d]
    args, keep = [], []
    dims = []
    for s, partner in zip(shells, [a, a, c if c is not None else a, c if c is not None else a]):
        if s is None:
            e = np.zeros(1)
            co = np.ones(1)
            X = np.ascontiguousarray(partner.center, dtype=float)
            args += [-1, 1, _p(e, ctypes.c_double), _p(co, ctypes.c_double), _p(X, ctypes.c_double)]
            keep += [e, co, X]
            dims.append(1)
        else:
            e = np.ascontiguousarray(s.exps, dtype=float)
            co = np.ascontiguousarray(s.coeffs, dtype=float)
            X = np.ascontiguousarray(s.center, dtype=float)
            args += [s.L, len(e), _p(e, ctypes.c_double), _p(co, ctypes.c_double), _p(X, ctypes.c_double)]
            keep += [e, co, X]
            dims.append(2 * s.L + 1)
    out = np.zeros(int(np.prod(dims)))
    rc = lib().oracle_eri_block(*args, _p(out, ctypes.c_double))
    if rc != 0:
        raise ValueError("angular momentum above the oracle's maximum")
    return out.reshape(dims)


def int_schwarz_aux(shells):
    keep, b = _basis_args(shells)
    out = np.zeros(len(shells))
    lib().oracle_int_schwarz_aux(*b, _p(out, ctypes.c_double))
    return out


def int_schwarz_bra(shells):
    keep, b = _basis_args(shells)
    n = len(shells)
    out = np.zeros(n * (n + 1) // 2)
    lib().oracle_int_schwarz_bra(*b, _p(out, ctypes.c_double))
    return out


def int2c2e(shells):
    keep, b = _basis_args(shells)
    n = shells.sph_size
    out = np.zeros((n, n), order="F")
    lib().oracle_int2c2e_metric(*b, n, _p(out, ctypes.c_double))
    return out


def contract_coulomb_densities_2d(shells, shells_aux, densities):
    k1, b1 = _basis_args(shells)
    k2, b2 = _basis_args(shells_aux)
    D = np.asfortranarray(densities, dtype=np.float64)
    ndens, nbf, _ = D.shape
    naux = shells_aux.sph_size
    out = np.zeros((naux, ndens), order="F")
    lib().oracle_contract_coulomb_densities_2d(*b1, *b2, ndens, nbf, _p(D, ctypes.c_double), naux,
                                               _p(out, ctypes.c_double))
    return out


def contract_coulomb_densities_4d(shells, shells_aux, densities):
    k1, b1 = _basis_args(shells)
    k2, b2 = _basis_args(shells_aux)
    D = np.asfortranarray(densities, dtype=np.float64)
    ndens, nbf, _ = D.shape
    nstates = int(round((np.sqrt(8 * ndens + 1) - 1) / 2))
    assert nstates * (nstates + 1) // 2 == ndens
    out = np.zeros((nstates,) * 4, order="F")
    lib().oracle_contract_coulomb_densities_4d(*b1, *b2, ndens, nbf, _p(D, ctypes.c_double),
                                               nstates, _p(out, ctypes.c_double))
    return out


def int_eri2c(shells, shells_aux):
    k1, b1 = _basis_args(shells)
    k2, b2 = _basis_args(shells_aux)
    nbf = shells.sph_size
    out = np.zeros((nbf, nbf), order="F")
    lib().oracle_intor_eri2c(*b1, *b2, nbf, _p(out, ctypes.c_double))
    return out


def int_df1c(shells, shells_aux):
    k1, b1 = _basis_args(shells)
    k2, b2 = _basis_args(shells_aux)
    nbf, naux = shells.sph_size, shells_aux.sph_size
    out = np.zeros((nbf, naux), order="F")
    lib().oracle_intor_df1c(*b1, *b2, nbf, naux, _p(out, ctypes.c_double))
    return out


def int_df2c_mo(shells, shells_aux, mo_tensor):
    k1, b1 = _basis_args(shells)
    k2, b2 = _basis_args(shells_aux)
    C = np.asfortranarray(mo_tensor, dtype=np.float64)
    nbf, nmos = C.shape
    naux = shells_aux.sph_size
    out = np.zeros((nmos * (nmos + 1) // 2, naux), order="F")
    lib().oracle_intor_df2c_mo(*b1, *b2, nbf, nmos, _p(C, ctypes.c_double), naux,
                               _p(out, ctypes.c_double))
    return out


def chol_solve_ld(M, B, want_L=False):
    """Y = L^-1 B with L = chol(M), factor and solve in long double (64-bit
    significand), rounded to double. Checker for FP64 solves of
    ill-conditioned metrics; returns Y (and L with want_L)."""
    M = np.asfortranarray(M, dtype=np.float64)
    n = M.shape[0]
    B2 = np.asfortranarray(np.asarray(B, dtype=np.float64).reshape(n, -1))
    Y = np.zeros_like(B2, order="F")
    L = np.zeros((n, n), order="F") if want_L else None
    rc = lib().oracle_chol_solve_ld(n, _p(M, ctypes.c_double), B2.shape[1], _p(B2, ctypes.c_double),
                                    _p(Y, ctypes.c_double), _p(L, ctypes.c_double) if want_L else None)
    if rc:
        raise np.linalg.LinAlgError(f"long-double Cholesky: non-positive pivot in column {rc}")
    Y = Y.reshape(np.shape(B))
    return (Y, L) if want_L else Y


def chol_backward_error_ld(M, L):
    """||L L^T - M||_F / ||M||_F in long double (lower triangle of L)."""
    M = np.asfortranarray(M, dtype=np.float64)
    L = np.asfortranarray(L, dtype=np.float64)
    return lib().oracle_chol_backward_error_ld(M.shape[0], _p(M, ctypes.c_double), _p(L, ctypes.c_double))


def coulomb_from_df(df, nstates):
    """The Coulomb tensor R[i,j,k,l] = sum_m B[m,(ij)] B[m,(kl)] of a df matrix
    (naux x ndens, pairs i >= j in the order of diabatization/intor.f90:241-269)."""
    df = np.asarray(df)
    G = df.T @ df
    R = np.zeros((nstates,) * 4)
    pairs = [(i, j) for i in range(nstates) for j in range(i + 1)]
    for p, (i, j) in enumerate(pairs):
        for q, (k, l) in enumerate(pairs):
            v = G[p, q]
            for a, b in ((i, j), (j, i)):
                for c, d in ((k, l), (l, k)):
                    R[a, b, c, d] = v
    return R


def eval_densities(shells, grid3d, densities, blk_size=100, thresh=1e-8):
    """Densities on grid points, (ndens, npoints) F-ordered, like
    pysisyphus_addons.grid.grid.eval_densities (grid/_grid.pyx:35-75):
    grid3d (npoints, 3), Cartesian AO densities (ndens, nbfs, nbfs)."""
    k1, b1 = _basis_args(shells)
    G = np.asfortranarray(np.asarray(grid3d, dtype=np.float64).T)
    D = np.asfortranarray(densities, dtype=np.float64)
    ndens, nbfs = D.shape[0], D.shape[1]
    npoints = G.shape[1]
    out = np.zeros((ndens, npoints), order="F")
    lib().oracle_eval_densities(*b1, npoints, _p(G, ctypes.c_double), ndens, nbfs, _p(D, ctypes.c_double),
                                _p(out, ctypes.c_double), int(blk_size), float(thresh))
    return out


def eval_prim_density(Ls_inds, prim_data, coords3d, P_tot_cart, switch, rho_pseudo):
    """In-place like pysisyphus_addons.gdma.prim_dens.eval_prim_density
    (gdma/prim_dens.pyx:26-50): Ls_inds (nprims, 2), prim_data (nprims, 5),
    coords3d (npoints, 3), P_tot_cart (nbfs, nbfs)."""
    Li = np.asfortranarray(np.asarray(Ls_inds, dtype=np.int32).T)
    Pd = np.asfortranarray(np.asarray(prim_data, dtype=np.float64).T)
    C = np.asfortranarray(np.asarray(coords3d, dtype=np.float64).T)
    P = np.asfortranarray(P_tot_cart, dtype=np.float64)
    rho = np.zeros(C.shape[1])
    lib().oracle_eval_prim_density(Li.shape[1], C.shape[1], P.shape[0], _p(Li, ctypes.c_int), _p(Pd, ctypes.c_double),
                                   _p(C, ctypes.c_double), _p(P, ctypes.c_double), float(switch),
                                   _p(rho, ctypes.c_double))
    rho_pseudo[:] = rho
    return rho_pseudo


def int3c2e_estimates(shells, shells_aux):
    """(records (n, 4), nskipped) of the estimator study
    (intor/benchmark.f90:15-132): schwarz_estimate, qvl_estimate, ||(ab|c)||_2
    and the pair-center distance per record."""
    k1, b1 = _basis_args(shells)
    k2, b2 = _basis_args(shells_aux)
    sk = ctypes.c_longlong()
    n = lib().oracle_int3c2e_estimates(*b1, *b2, 0, None, ctypes.byref(sk))
    rec = np.zeros((max(n, 1), 4))
    lib().oracle_int3c2e_estimates(*b1, *b2, n, _p(rec, ctypes.c_double), ctypes.byref(sk))
    return rec[:n], sk.value
