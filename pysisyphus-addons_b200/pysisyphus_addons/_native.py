"""ctypes binding of libpa_b200.so (the C-ABI declared in include/pa_b200.h).

This replaces the Cython modules (``*/_intor.pyx``) of the reference: the
argument lists are the ones of the reference's ``bind(c)`` wrappers, arrays are
column-major, basis pointers 1-based. There is no CPU fallback -- if the CUDA
library has not been built, importing this module raises.
"""

import ctypes
import os
import threading
from collections import OrderedDict
from pathlib import Path

import numpy as np

LIB_PATH = Path(os.environ.get("PA_B200_LIB", Path(__file__).resolve().parent / "_lib" / "libpa_b200.so"))

PA_OK = 0
PA_ERR_ARG = 1
PA_ERR_LMAX = 2
PA_ERR_NOT_SPD = 3
PA_ERR_CUDA = 4
PA_ERR_TIMEOUT = 5
PA_ERR_NO_DEVICE = 6
PA_ERR_SCRATCH = 7

PA_BOYS_EXACT = 0
PA_BOYS_REFERENCE = 1
PA_PRECISION_FP64 = 0
PA_PRECISION_MIXED = 1
PA_SCREEN_SCHWARZ = 0
PA_SCREEN_QVL = 1
PA_LAYOUT_FORTRAN = 0
PA_LAYOUT_C = 1
LMAX, LAUXMAX = 4, 5  # PA_LMAX_ORBITAL, PA_LMAX_AUX of pa_b200.h
PA_LMAX_ORBITAL = 4
PA_LMAX_AUX = 5
PA_NOALLOC_SCRATCH_DOUBLES = 1 << 20

_ERRNAMES = {
    PA_ERR_ARG: "invalid argument",
    PA_ERR_LMAX: "angular momentum above the compiled maximum",
    PA_ERR_NOT_SPD: "metric not positive definite",
    PA_ERR_CUDA: "CUDA error",
    PA_ERR_TIMEOUT: "device timeout",
    PA_ERR_NO_DEVICE: "no CUDA device",
    PA_ERR_SCRATCH: "scratch capacity exceeded",
}


class PaError(RuntimeError):
    def __init__(self, code, message):
        self.code = code
        super().__init__(f"{_ERRNAMES.get(code, 'error')} ({code}): {message}")


class PaStats(ctypes.Structure):
    _fields_ = [
        ("ntriplets", ctypes.c_longlong),
        ("nskipped", ctypes.c_longlong),
        ("nints", ctypes.c_longlong),
        ("ms_total", ctypes.c_double),
        ("ms_screen", ctypes.c_double),
        ("ms_bra", ctypes.c_double),
        ("ms_metric", ctypes.c_double),
        ("ms_3c", ctypes.c_double),
        ("ms_solve", ctypes.c_double),
        ("kernel_launches", ctypes.c_int),
        ("launches_3c", ctypes.c_int),
    ]


_i = ctypes.c_int
_d = ctypes.c_double
_pi = ctypes.POINTER(ctypes.c_int)
_pd = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_BASIS = [_i, _i, _pi, _pi, _pd]

# Symbols declared in include/pa_b200.h with their argument types.
SIGNATURES = {
    "f_init": [],
    "f_int_schwarz_aux": _BASIS + [_pd],
    "f_int_schwarz_bra": _BASIS + [_pd],
    "f_contract_coulomb_densities_2d": _BASIS + _BASIS + [_i, _i, _pd, _i, _pd],
    "f_contract_coulomb_densities_4d": _BASIS + _BASIS + [_i, _i, _pd, _i, _pd],
    "f_intor_eri2c": _BASIS + _BASIS + [_i, _pd],
    "f_intor_df1c": _BASIS + _BASIS + [_i, _i, _pd],
    "f_intor_df2c_mo": _BASIS + _BASIS + [_i, _i, _pd, _i, _pd],
    "pa_last_error": [],
    "pa_set_boys_mode": [_i],
    "pa_get_boys_mode": [],
    "pa_set_screen_threshold": [_d],
    "pa_set_skip_metric": [_i],
    "pa_set_metric_shift": [_d],
    "pa_set_precision": [_i, _d],
    "pa_set_items_per_sm": [_i],
    "pa_get_precision": [],
    "pa_set_mixed_kernels": [_i],
    "pa_set_class_grid": [_i],
    "pa_basis_cache_clear": [],
    "pa_get_device": [_pi],
    "pa_get_mixed_kernels": [],
    "pa_set_screening": [_i],
    "pa_get_screening": [],
    "pa_get_stats": [ctypes.POINTER(PaStats)],
    "pa_basis_create": [_i, _i, _pi, _pi, _pd, _i, ctypes.POINTER(_vp)],
    "pa_basis_destroy": [_vp],
    "pa_basis_info": [_vp, _pi, _pi, _pi],
    "pa_df_2d": [_vp, _vp, _i, _i, _vp, _i, _vp, _vp],
    "pa_df_4d": [_vp, _vp, _i, _i, _vp, _i, _i, _vp, _vp],
    "pa_df_4d_batch": [_i, ctypes.POINTER(_vp), ctypes.POINTER(_vp), _pi, ctypes.POINTER(_vp), _i, _pi,
                       ctypes.POINTER(_vp), _i, _vp],
    "pa_contract_coulomb_densities_2d": [_vp, _vp, _i, _i, _pd, _i, _pd],
    "pa_contract_coulomb_densities_4d": [_vp, _vp, _i, _i, _pd, _i, _i, _pd],
    "pa_count_triplets": [_vp, _vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                          ctypes.POINTER(ctypes.c_longlong)],
    "pa_boys_eval": [_i, _i, _i, _pd, _pd],
    "pa_metric": [_vp, _pd],
    "pa_cholesky_solve": [_i, _pd, _i, _pd],
    "pa_std_df1c": [_vp, _vp, _vp, _vp],
    "pa_std_eri2c": [_vp, _vp, _vp, _vp],
    "pa_std_df2c_mo": [_vp, _vp, _i, _vp, _vp, _vp],
    "pa_cholesky_solve_noalloc": [_i, _vp, _i, _vp, _vp, _vp],
    "pa_df_solve": [_vp, _i, _vp, _vp, _i, _vp, _vp],
    "pa_set_class_timing": [_i],
    "pa_get_class_times": [_i, _pi, _pi, _pd],
    "pa_set_tile_variant": [_i, _i, _i],
    "pa_get_tile_variant": [_i, _i, _pi],
    "pa_tile_shape": [_i, _i, _i, _pi],
    "pa_load_tile_table": [ctypes.c_char_p, _pi],
    "f_benchmark_int3c2e": _BASIS + _BASIS,
    "pa_int3c2e_estimates": [_vp, _vp, ctypes.c_longlong, _pd, ctypes.POINTER(ctypes.c_longlong),
                             ctypes.POINTER(ctypes.c_longlong)],
    "f_eval_densities": _BASIS + [_i, _pd, _i, _i, _pd, _pd, _i, _d],
    "f_eval_prim_density": [_i, _i, _i, _pi, _pd, _pd, _pd, _d, _pd],
    "pa_split_product_check": [_i, _i, _i, _pd, _pd, _pd],
}

_lib = None


def load():
    """Load libpa_b200.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} not found: build the CUDA library first "
            "(make -C pysisyphus-addons_b200, or __graft_entry__.build())"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_char_p if name == "pa_last_error" else ctypes.c_int
    _lib = lib
    return lib


def check(rc):
    if rc != PA_OK:
        msg = load().pa_last_error().decode(errors="replace")
        raise PaError(rc, msg)


def ptr(arr, ctype=ctypes.c_double):
    return arr.ctypes.data_as(ctypes.POINTER(ctype))


def basis_args(shells):
    """(keep-alive arrays, ctypes argument list) of a shells object."""
    bc, bs, bd = shells.as_arrays(fortran=True)
    bc = np.asfortranarray(bc, dtype=np.int32)
    bs = np.asfortranarray(bs, dtype=np.int32)
    bd = np.ascontiguousarray(bd, dtype=np.float64)
    return (bc, bs, bd), [len(bc), len(bd), ptr(bc, ctypes.c_int), ptr(bs, ctypes.c_int), ptr(bd)]


def nsph(shells):
    _, bs, _ = shells.as_arrays(fortran=True)
    return int(np.sum(2 * np.asarray(bs)[:, 1] + 1))


def set_boys_mode(mode):
    """'reference' (default; the reference's interpolation) or 'exact'."""
    code = {"exact": PA_BOYS_EXACT, "reference": PA_BOYS_REFERENCE}.get(mode, mode)
    check(load().pa_set_boys_mode(int(code)))


def get_boys_mode():
    return {PA_BOYS_EXACT: "exact", PA_BOYS_REFERENCE: "reference"}[load().pa_get_boys_mode()]


def set_screen_threshold(thresh):
    check(load().pa_set_screen_threshold(float(thresh)))


def set_precision(mode="fp64", fp32_thresh=1e-6):
    """'fp64' (default) or 'mixed': FP32 recurrences for shell triplets whose
    Schwarz bound is below fp32_thresh."""
    code = {"fp64": PA_PRECISION_FP64, "mixed": PA_PRECISION_MIXED}.get(mode, mode)
    check(load().pa_set_precision(int(code), float(fp32_thresh)))


def set_mixed_kernels(mode):
    """Kernels of the mixed form: 0 (default) keeps the weak triplets in the
    FP64 class kernels with FP32 recurrences, 1 runs them on their own kernels
    with the split-BF16 tensor-core product."""
    check(load().pa_set_mixed_kernels(int(mode)))


def get_mixed_kernels():
    return int(load().pa_get_mixed_kernels())


def set_items_per_sm(items):
    """Work items per SM and shell class of the three-center queue (0 = by size, the default)."""
    check(load().pa_set_items_per_sm(int(items)))


def get_precision():
    return {PA_PRECISION_FP64: "fp64", PA_PRECISION_MIXED: "mixed"}[load().pa_get_precision()]


def set_screening(mode="schwarz"):
    """'schwarz' (default, the reference's schwarz_estimate) or 'qvl'
    (qvl_estimate, common/screening.f90:267-299) for the Coulomb-tensor path."""
    code = {"schwarz": PA_SCREEN_SCHWARZ, "qvl": PA_SCREEN_QVL}.get(mode, mode)
    check(load().pa_set_screening(int(code)))


def get_screening():
    return {PA_SCREEN_SCHWARZ: "schwarz", PA_SCREEN_QVL: "qvl"}[load().pa_get_screening()]


def set_metric_shift(shift):
    """Diagonal shift added to (P|Q) before the Cholesky factorization (0 = reference)."""
    check(load().pa_set_metric_shift(float(shift)))


def set_skip_metric(skip):
    check(load().pa_set_skip_metric(int(bool(skip))))


def set_class_timing(on):
    """Serialize and time the three-center class launches (profiling aid)."""
    check(load().pa_set_class_timing(int(bool(on))))


def get_class_times():
    """[(L_ab, L_c, ms)] of the class runs of the last single-molecule call in
    class-timing mode."""
    lib = load()
    n = lib.pa_get_class_times(0, None, None, None)
    lab, lc, ms = (ctypes.c_int * max(n, 1))(), (ctypes.c_int * max(n, 1))(), (ctypes.c_double * max(n, 1))()
    lib.pa_get_class_times(n, lab, lc, ms)
    return [(lab[i], lc[i], ms[i]) for i in range(n)]


TILE_VARIANTS = 3


def set_tile_variant(lab, lc, variant):
    """Tile-shape variant of the three-center class (L_ab, L_c) (0 = default)."""
    check(load().pa_set_tile_variant(int(lab), int(lc), int(variant)))


def get_tile_variant(lab, lc):
    v = ctypes.c_int()
    check(load().pa_get_tile_variant(int(lab), int(lc), ctypes.byref(v)))
    return v.value


def tile_shape(lab, lc, variant):
    """dict(tc, ub, lanes, blocks_per_sm, smem) of one class variant."""
    out = (ctypes.c_int * 5)()
    check(load().pa_tile_shape(int(lab), int(lc), int(variant), out))
    return dict(zip(("tc", "ub", "lanes", "blocks_per_sm", "smem"), list(out)))


def load_tile_table(path=None):
    """Applies a tile table ("L_ab L_c variant" lines); None = the default
    table beside the library. Returns the number of entries applied."""
    n = ctypes.c_int()
    check(load().pa_load_tile_table(None if path is None else str(path).encode(), ctypes.byref(n)))
    return n.value


def get_stats():
    st = PaStats()
    check(load().pa_get_stats(ctypes.byref(st)))
    return {name: getattr(st, name) for name, _ in PaStats._fields_}


def boys(nmax, T, mode="reference"):
    """F_0..F_nmax at the points T, evaluated on the device; shape (len(T), nmax+1)."""
    T = np.ascontiguousarray(np.atleast_1d(T), dtype=np.float64)
    out = np.zeros((len(T), nmax + 1))
    code = {"exact": PA_BOYS_EXACT, "reference": PA_BOYS_REFERENCE}.get(mode, mode)
    check(load().pa_boys_eval(int(code), int(nmax), len(T), ptr(T), ptr(out)))
    return out


class Basis:
    """A basis unpacked, normalized and resident in device memory (pa_basis)."""

    def __init__(self, shells, role="orbital", _args=None):
        lib = load()
        keep, args = _args if _args is not None else basis_args(shells)
        lmax = PA_LMAX_ORBITAL if role == "orbital" else PA_LMAX_AUX
        handle = _vp()
        check(lib.pa_basis_create(*args, lmax, ctypes.byref(handle)))
        self.handle = handle
        n, ns, lm = _i(), _i(), _i()
        check(lib.pa_basis_info(handle, ctypes.byref(n), ctypes.byref(ns), ctypes.byref(lm)))
        self.nshells, self.nsph, self.lmax = n.value, ns.value, lm.value
        self.role = role

    def close(self):
        if getattr(self, "handle", None):
            load().pa_basis_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def current_device():
    """The CUDA device the next library call runs on (of the calling thread)."""
    d = _i()
    check(load().pa_get_device(ctypes.byref(d)))
    return d.value


# Bases of the reference-facing functions: callers pass the same shells call
# after call, so the device copy (with its shell-pair lists, built on first use)
# is kept for later calls with byte-identical basis arrays on the same device;
# least recently used first out.
BASIS_CACHE_SIZE = 8
_basis_cache = OrderedDict()
_basis_lock = threading.Lock()


def cached_basis(shells, role="orbital"):
    keep, args = basis_args(shells)
    key = (current_device(), role) + tuple((a.shape, a.tobytes()) for a in keep)
    with _basis_lock:
        b = _basis_cache.get(key)
        if b is not None:
            _basis_cache.move_to_end(key)
            return b
    b = Basis(shells, role, _args=(keep, args))
    with _basis_lock:
        _basis_cache[key] = b
        while len(_basis_cache) > BASIS_CACHE_SIZE:
            _basis_cache.popitem(last=False)
    return b


def clear_basis_cache():
    """Frees the cached device bases of this module and of the f_* entry points."""
    with _basis_lock:
        _basis_cache.clear()
    check(load().pa_basis_cache_clear())


def count_triplets(orbital, aux):
    """(ntriplets, ncomputed, nints) of the Schwarz screening for two Basis objects."""
    a, b, c = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    check(load().pa_count_triplets(orbital.handle, aux.handle, ctypes.byref(a), ctypes.byref(b),
                                   ctypes.byref(c)))
    return a.value, b.value, c.value


def metric(aux):
    out = np.zeros((aux.nsph, aux.nsph), order="F")
    check(load().pa_metric(aux.handle, ptr(out)))
    return out


def cholesky_solve(A, B):
    """(L, L^-1 B) computed on the device, A = L L^T (L in the lower triangle
    of the first result; the linear algebra of the reference's inv_chol + dtrmm)."""
    A = np.array(A, dtype=np.float64, order="F", copy=True)
    B = np.array(B, dtype=np.float64, order="F", copy=True)
    n = A.shape[0]
    check(load().pa_cholesky_solve(n, ptr(A), B.shape[1] if B.ndim == 2 else 1, ptr(B)))
    return A, B


def df_4d_batch(orbitals, auxes, densities, nstates, outputs, layout=PA_LAYOUT_C, use_graph=True, stream=None):
    """Coulomb tensors of many molecules in one call (pa_df_4d_batch).

    orbitals, auxes: Basis objects; densities: device tensors (ndens, nbf, nbf);
    outputs: device tensors with nstates**4 elements each (column-major)."""
    n = len(orbitals)
    V = _vp * max(n, 1)
    I = ctypes.c_int * max(n, 1)
    orb = V(*[b.handle for b in orbitals])
    aux = V(*[b.handle for b in auxes])
    nd = I(*[int(d.shape[0]) for d in densities])
    dp = V(*[d.data_ptr() for d in densities])
    ns = I(*[int(x) for x in nstates])
    op = V(*[o.data_ptr() for o in outputs])
    check(load().pa_df_4d_batch(n, orb, aux, nd, dp, int(layout), ns, op, int(bool(use_graph)), stream))

