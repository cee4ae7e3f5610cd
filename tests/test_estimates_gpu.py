"""The screening-estimator study (intor/benchmark.f90:15-132) on the GPU
against the oracle's restatement: same records in the same order, the
Schwarz estimates and distances to 1e-14 relative, the QVL estimates to 1e-12
relative (erf^-1 by different methods), the block norms ||(ab|c)||_2 to 1e-7
relative plus 1e-14 of the largest (the oracle's horizontal recurrence loses
~1e-8 on distant pairs with d shells), and the skip count exactly; the entry
point writes the records to int_estimates.bin."""

import numpy as np
import pytest

import oracle
from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.synthetic import config_workload
from pysisyphus_addons.intor import benchmark

pytestmark = pytest.mark.gpu


def test_estimates_vs_oracle():
    w = config_workload("cfg1")
    nat.set_boys_mode("reference")
    oracle.set_boys_mode("reference")
    rec, sk = benchmark.int3c2e_estimates(w.shells, w.shells_aux)
    ref, sk_ref = oracle.int3c2e_estimates(w.shells, w.shells_aux)
    assert rec.shape == ref.shape and sk == sk_ref
    np.testing.assert_allclose(rec[:, 0], ref[:, 0], rtol=1e-14, atol=0)
    np.testing.assert_allclose(rec[:, 3], ref[:, 3], rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(rec[:, 1], ref[:, 1], rtol=1e-12, atol=0)
    np.testing.assert_allclose(rec[:, 2], ref[:, 2], rtol=1e-7, atol=1e-14 * ref[:, 2].max())
    # the Schwarz estimate bounds the block norm on every record here
    assert (rec[:, 2] <= rec[:, 0] * (1 + 1e-12)).all()


def test_benchmark_entry_point_writes_records(tmp_path, monkeypatch, capsys):
    w = config_workload("cfg1")
    monkeypatch.chdir(tmp_path)
    benchmark.benchmark_int3c2e(w.shells, w.shells_aux)
    rec, _ = benchmark.int3c2e_estimates(w.shells, w.shells_aux)
    data = np.fromfile(tmp_path / "int_estimates.bin", dtype=np.float64).reshape(-1, 4)
    np.testing.assert_array_equal(data, rec)
