"""The C-ABI library loads and exports every symbol include/pa_b200.h declares
(no compute calls: this runs without a GPU)."""

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "pa_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(\w+)\s*\(", text, flags=re.M)))


def test_header_declares_reference_entry_points():
    names = declared_symbols()
    for ref_name in ("f_init", "f_int_schwarz_aux", "f_int_schwarz_bra",
                     "f_contract_coulomb_densities_2d", "f_contract_coulomb_densities_4d",
                     "f_intor_eri2c", "f_intor_df1c", "f_intor_df2c_mo"):
        assert ref_name in names


def test_library_exports_all_declared_symbols():
    from pysisyphus_addons import _native

    lib = ctypes.CDLL(str(_native.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from pysisyphus_addons import _native

    assert set(declared_symbols()) <= set(_native.SIGNATURES)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from pysisyphus_addons import _native

    monkeypatch.setattr(_native, "_lib", None)
    monkeypatch.setattr(_native, "LIB_PATH", tmp_path / "nope.so")
    with pytest.raises(ImportError):
        _native.load()
