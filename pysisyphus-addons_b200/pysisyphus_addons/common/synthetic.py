"""Seeded synthetic molecules, basis sets and (transition) densities.

No public dataset is involved. The generator follows the workload
definitions of the density-fitting benchmarks:

* molecule: ``natoms`` atoms with Z uniform in {1, 6, 7, 8}, positions uniform
  in a cube of edge ``10 * (natoms / 8) ** (1/3)`` bohr (10 bohr for 8 atoms,
  constant number density for larger clusters), rejection-sampled to a minimum
  separation of 1.8 bohr;
* orbital basis, heavy atom: one s shell with 3 primitives (exponents
  log-uniform on [0.1, 80], random coefficients), 2 s, 2 p and 1 d single
  primitive shells, plus 1 f (lmax >= 3) and 1 g (lmax >= 4); hydrogen: 2 s
  and 1 p;
* auxiliary basis, every atom: even-tempered exponents 0.1 * 2.5**k with
  6 s (k = 0..5), 4 p (k = 0..3), 3 d (k = 0..2), 2 f (lauxmax >= 3),
  1 g (lauxmax >= 4), 1 h (lauxmax >= 5);
* states: random orthonormal MO coefficients (QR of a Gaussian matrix),
  normalized random CI vectors over ``nocc x nvirt`` orbital pairs, and the
  CIS-like state and transition densities built from them, in the lower
  triangular order (1,1), (2,1), (2,2), (3,1), ... that the reference expects
  (``diabatization/intor.f90:33-35``).
"""

from dataclasses import dataclass

import numpy as np

from .shells import Shell, Shells

ELEMENTS = np.array([1, 6, 7, 8])


@dataclass
class Molecule:
    atomic_nums: np.ndarray
    coords: np.ndarray  # (natoms, 3) in bohr


def cube_edge(natoms):
    return 10.0 * (natoms / 8.0) ** (1.0 / 3.0)


def random_molecule(natoms, seed=0, min_sep=1.8, edge=None):
    rng = np.random.default_rng(seed)
    edge = cube_edge(natoms) if edge is None else edge
    zs = rng.choice(ELEMENTS, size=natoms)
    coords = []
    tries = 0
    while len(coords) < natoms:
        tries += 1
        if tries > 1_000_000:
            raise RuntimeError("could not place atoms at the requested separation")
        x = rng.uniform(0.0, edge, size=3)
        if all(np.linalg.norm(x - c) >= min_sep for c in coords):
            coords.append(x)
    return Molecule(zs, np.array(coords))


def _loguniform(rng, lo, hi, size=None):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=size))


def orbital_basis(mol, lmax=2, seed=0):
    rng = np.random.default_rng(seed + 1_000_003)
    shells = []
    for ind, (z, xyz) in enumerate(zip(mol.atomic_nums, mol.coords)):
        if z == 1:
            spec = [0, 0, 1]
        else:
            spec = [0, 0, 1, 1, 2]
            if lmax >= 3:
                spec.append(3)
            if lmax >= 4:
                spec.append(4)
            # Contracted s shell with three primitives.
            exps = np.sort(_loguniform(rng, 0.1, 80.0, size=3))[::-1]
            coeffs = rng.uniform(0.2, 1.0, size=3)
            shells.append(Shell(0, xyz, coeffs, exps, ind, int(z)))
        for L in spec:
            exp = _loguniform(rng, 0.1, 80.0)
            shells.append(Shell(L, xyz, [1.0], [exp], ind, int(z)))
    return Shells(shells)


AUX_SPEC = ((0, 6), (1, 4), (2, 3), (3, 2), (4, 1), (5, 1))


def aux_basis(mol, lauxmax=2):
    shells = []
    for ind, (z, xyz) in enumerate(zip(mol.atomic_nums, mol.coords)):
        for L, count in AUX_SPEC:
            if L > lauxmax:
                continue
            for k in range(count):
                shells.append(Shell(L, xyz, [1.0], [0.1 * 2.5**k], ind, int(z)))
    return Shells(shells)


def random_states(nbf, nstates, nocc=6, nvirt=6, seed=0):
    """Return (densities[ndens, nbf, nbf], mo_coeffs[nbf, nbf])."""
    rng = np.random.default_rng(seed + 2_000_003)
    nocc = min(nocc, nbf // 2)
    nvirt = min(nvirt, nbf - nocc)
    C, _ = np.linalg.qr(rng.normal(size=(nbf, nbf)))
    Co = C[:, :nocc]
    Cv = C[:, nocc : nocc + nvirt]
    # State 0 is the ground state, states 1.. are excited (CIS-like vectors).
    X = rng.normal(size=(nstates, nocc, nvirt))
    X[0] = 0.0
    for J in range(1, nstates):
        X[J] /= np.linalg.norm(X[J])
    D00 = 2.0 * Co @ Co.T
    dens = []
    for I in range(nstates):
        for J in range(I + 1):
            if I == J == 0:
                D = D00
            elif J == 0:
                D = np.sqrt(2.0) * Co @ X[I] @ Cv.T
            elif I == J:
                D = D00 - Co @ X[I] @ X[I].T @ Co.T + Cv @ X[I].T @ X[I] @ Cv.T
            else:
                D = Cv @ X[I].T @ X[J] @ Cv.T - Co @ X[J] @ X[I].T @ Co.T
            dens.append(D)
    return np.ascontiguousarray(np.stack(dens)), C


@dataclass
class Workload:
    name: str
    mol: Molecule
    shells: Shells
    shells_aux: Shells
    densities: np.ndarray
    mo_coeffs: np.ndarray
    nstates: int


def make_workload(natoms, lmax, lauxmax, nstates, seed=0, name=None):
    mol = random_molecule(natoms, seed=seed)
    shells = orbital_basis(mol, lmax=lmax, seed=seed)
    shells_aux = aux_basis(mol, lauxmax=lauxmax)
    dens, C = random_states(shells.sph_size, nstates, seed=seed)
    name = name or f"df_coulomb_{natoms}atoms_lmax{lmax}_lauxmax{lauxmax}_{nstates}states"
    return Workload(name, mol, shells, shells_aux, dens, C, nstates)


# The five benchmark configurations: (natoms, lmax, lauxmax, nstates).
CONFIGS = {
    "cfg1": dict(natoms=8, lmax=2, lauxmax=2, nstates=4),
    "cfg2": dict(natoms=40, lmax=3, lauxmax=4, nstates=8),
    "cfg5": dict(natoms=200, lmax=4, lauxmax=5, nstates=8),
}


def config_workload(key, seed=0):
    return make_workload(seed=seed, **CONFIGS[key])


def batch_workloads(nmol=64, lmax=3, lauxmax=4, atoms=(5, 60), states=(4, 16), seed=4321):
    """The batched workload: nmol molecules with seeds 0..nmol-1, atom counts
    uniform in [atoms[0], atoms[1]] and state counts uniform in
    [states[0], states[1]] (drawn from one generator seeded with `seed`)."""
    rng = np.random.default_rng(seed)
    natoms = rng.integers(atoms[0], atoms[1] + 1, size=nmol)
    nstates = rng.integers(states[0], states[1] + 1, size=nmol)
    return [make_workload(int(n), lmax, lauxmax, int(k), seed=i,
                          name=f"batch{i}_{int(n)}atoms_{int(k)}states")
            for i, (n, k) in enumerate(zip(natoms, nstates))]
