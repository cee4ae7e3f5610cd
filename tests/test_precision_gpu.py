"""Precision form of the three-center contraction (pa_set_precision): shell
triplets with Schwarz bound Q_ab * Q_c below a threshold run their recurrences
(Boys function, Hermite R, solid harmonics) in FP32 and are accumulated in FP64.

Every integral of such a triplet is bounded by its Schwarz value, so the FP32
rounding (~1e-7 relative, grown by the recurrences) perturbs the raw
contraction sum_(a>=b) (ab|P) Dsym by far less than the bound itself. The raw
contraction is compared with the FP64 oracle fixture at 1e-9 of its largest
element (measured: see the committed precision report in profiles/).
"""

import numpy as np
import pytest

import oracle
from pysisyphus_addons import _native as nat
from pysisyphus_addons.common.synthetic import config_workload
from pysisyphus_addons.diabatization import intor as dia

pytestmark = pytest.mark.gpu


def raw_df(w):
    nat.set_skip_metric(1)
    try:
        return dia.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    finally:
        nat.set_skip_metric(0)


@pytest.fixture(autouse=True)
def reset():
    yield
    nat.set_precision("fp64")
    nat.set_boys_mode("reference")


def test_threshold_zero_is_the_fp64_path():
    w = config_workload("cfg1")
    a = raw_df(w)
    nat.set_precision("mixed", 0.0)
    b = raw_df(w)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("mode", ["reference", "exact"])
def test_mixed_raw_contraction_cfg1(mode):
    w = config_workload("cfg1")
    nat.set_boys_mode(mode)
    oracle.set_boys_mode(mode)
    oracle.set_skip_metric(1)
    try:
        ref = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
    finally:
        oracle.set_skip_metric(0)
        oracle.set_boys_mode("reference")
    nat.set_precision("mixed", 1e-6)
    got = raw_df(w)
    err = np.abs(got - ref).max()
    assert err <= 1e-9 * np.abs(ref).max(), err
    # the FP32 path is really taken: with every triplet in FP32 the error grows
    nat.set_precision("mixed", 1e30)
    all32 = raw_df(w)
    assert np.abs(all32 - ref).max() > err


def test_mixed_raw_contraction_cfg2(golden_dir):
    w = config_workload("cfg2")
    fx = np.load(golden_dir / "oracle_cfg2_reference.npz")
    nat.set_precision("mixed", 1e-6)
    got = raw_df(w)
    err = np.abs(got - fx["raw"]).max()
    assert err <= 1e-9 * np.abs(fx["raw"]).max(), err
