"""Host-side logic: basis packing, the synthetic workload generator."""

import numpy as np

from pysisyphus_addons.common.shells import Shell, Shells
from pysisyphus_addons.common.synthetic import CONFIGS, config_workload, random_molecule


def test_as_arrays_roundtrip():
    sh = Shells([Shell(0, [0, 0, 0], [0.5, 0.5], [3.0, 1.0], 0, 8),
                 Shell(2, [0, 0, 0], [1.0], [0.8], 0, 8),
                 Shell(1, [1, 2, 3], [1.0], [0.5], 1, 1)])
    bc, bs, bd = sh.as_arrays(fortran=True)
    assert bc.dtype == np.int32 and bs.dtype == np.int32 and bc.shape == (3, 3) and bs.shape == (3, 5)
    assert bs[:, 1].tolist() == [0, 2, 1] and bs[:, 2].tolist() == [2, 1, 1]
    back = Shells.from_arrays(bc, bs, bd, fortran=True)
    for a, b in zip(sh, back):
        assert a.L == b.L
        np.testing.assert_array_equal(a.center, b.center)
        np.testing.assert_array_equal(a.coeffs, b.coeffs)
        np.testing.assert_array_equal(a.exps, b.exps)
    # 1-based pointers (what the Fortran reads, common/shells.f90:151-167)
    assert bc[:, 2].min() == 1


def test_generator_sizes():
    w = config_workload("cfg1")
    assert len(w.mol.atomic_nums) == 8
    d = np.linalg.norm(w.mol.coords[:, None] - w.mol.coords[None], axis=-1)
    assert d[np.triu_indices(8, 1)].min() >= 1.8
    assert w.shells.l_max <= 2 and w.shells_aux.l_max <= 2
    assert w.densities.shape == (10, w.shells.sph_size, w.shells.sph_size)
    nheavy = int(np.sum(w.mol.atomic_nums > 1))
    assert w.shells.sph_size == nheavy * (1 + 2 + 6 + 5) + (8 - nheavy) * (2 + 3)
    assert w.shells_aux.sph_size == 8 * (6 + 12 + 15)


def test_generator_is_seeded():
    a = random_molecule(12, seed=5)
    b = random_molecule(12, seed=5)
    np.testing.assert_array_equal(a.coords, b.coords)
    assert set(CONFIGS) >= {"cfg1", "cfg2", "cfg5"}
