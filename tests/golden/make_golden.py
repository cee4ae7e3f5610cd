"""Generate the golden fixtures under tests/golden/ (run in the build container).

Inputs, read from a checkout of the reference project (default
/root/reference, override with PA_REFERENCE):

* tests/test_coulomb_tensor/bena2_dcat.bson: ORCA wavefunction of BeNa2(2+)
  (basis, geometry, overlap matrix);
* tests/test_coulomb_tensor/bena2_dcat_densities_relaxed.npy: relaxed state and
  transition densities;
* tests/test_coulomb_tensor/test_coulomb_tensor.py: the hard-coded 2x2x2x2
  Coulomb tensor the reference asserts (atol 1e-12, rtol 1e-7).

Outputs:

* bena2_basis.json: shells (L, center in bohr, coefficients, exponents);
* bena2_overlap.npy: ORCA overlap matrix permuted to m = -l..l order;
* bena2_densities.npy: stack(D00, D01, D11) as the reference test builds it;
* bena2_coulomb_ref.json: the reference's golden Coulomb tensor;
* oracle_<cfg>_<mode>.npz: oracle results (Coulomb tensor, df tensor and the
  raw contraction before the metric solve) of the
  synthetic workloads, for GPU parity tests at sizes where re-running the
  oracle would dominate the test time.
"""

import json
import os
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "pysisyphus-addons_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

from pysisyphus_addons.common.orca import load_orca_bson  # noqa: E402
from pysisyphus_addons.common.synthetic import config_workload  # noqa: E402


def reference_fixtures(ref):
    tdir = ref / "tests" / "test_coulomb_tensor"
    shells, S = load_orca_bson(tdir / "bena2_dcat.bson")
    basis = [
        dict(L=s.L, center=s.center.tolist(), coeffs=s.coeffs.tolist(), exps=s.exps.tolist(),
             center_ind=s.center_ind, atomic_num=s.atomic_num)
        for s in shells
    ]
    (HERE / "bena2_basis.json").write_text(json.dumps(basis, indent=1))
    np.save(HERE / "bena2_overlap.npy", S)
    D = np.load(tdir / "bena2_dcat_densities_relaxed.npy")
    np.save(HERE / "bena2_densities.npy", np.stack((D[0, 0], D[0, 1], D[1, 1]), axis=0))
    src = (tdir / "test_coulomb_tensor.py").read_text()
    body = src[src.index("np.array(") :]
    body = body[: body.index("np.testing")]
    numbers = [float(x) for x in re.findall(r"[-+]?\d+\.\d+(?:[eE][-+]?\d+)?", body)]
    assert len(numbers) == 16, numbers
    ref_tensor = np.array(numbers).reshape(2, 2, 2, 2)
    (HERE / "bena2_coulomb_ref.json").write_text(json.dumps(
        {"tensor": ref_tensor.tolist(), "atol": 1e-12, "rtol": 1e-7,
         "source": "tests/test_coulomb_tensor/test_coulomb_tensor.py:17-32"}, indent=1))


def oracle_fixtures(keys):
    import oracle

    for key in keys:
        w = config_workload(key)
        for mode in ("reference", "exact"):
            oracle.set_boys_mode(mode)
            df = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
            oracle.set_skip_metric(1)
            raw = oracle.contract_coulomb_densities_2d(w.shells, w.shells_aux, w.densities)
            oracle.set_skip_metric(0)
            R = oracle.contract_coulomb_densities_4d(w.shells, w.shells_aux, w.densities)
            st = oracle.last_stats()
            extra = {"df": df} if key == "cfg1" else {}  # the cfg2 df is too ill-conditioned to compare
            np.savez_compressed(HERE / f"oracle_{key}_{mode}.npz", R=R, raw=raw, **extra,
                                ntriplets=st["ntriplets"], nskipped=st["nskipped"], nints=st["nints"])
            print(key, mode, st)


if __name__ == "__main__":
    ref = Path(os.environ.get("PA_REFERENCE", "/root/reference"))
    reference_fixtures(ref)
    oracle_fixtures(sys.argv[1:] or ["cfg1", "cfg2"])
