"""Minimal stand-in for pysisyphus' ``Shells`` container.

pysisyphus (the caller of pysisyphus-addons) is not a dependency of this
package. Every public entry point only needs an object with
``as_arrays(fortran=True)`` returning ``(bas_centers, bas_spec, bas_data)``;
this module provides such an object, packed exactly the way the reference's
Fortran constructor unpacks it (``common/shells.f90:97-187``):

* ``bas_centers`` int32[nshells, 3]: (center index, atomic number,
  pointer to the three center coordinates in ``bas_data``);
* ``bas_spec`` int32[nshells, 5]: (shell index, L, number of primitives,
  number of contracted functions (always 1), pointer to the ``nprims``
  contraction coefficients, which are followed directly by the ``nprims``
  exponents);
* ``bas_data`` float64[m]: coordinates (bohr), coefficients, exponents.

Pointers are 1-based when ``fortran=True`` (what the Fortran and this
package's C-ABI read) and 0-based otherwise.

Contraction coefficients are given for *normalized primitives*; the
reference renormalizes them (``common/normalization.f90:10-38``) and so does
this package's native code.
"""

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Shell:
    L: int
    center: np.ndarray
    coeffs: np.ndarray
    exps: np.ndarray
    center_ind: int = 0
    atomic_num: int = 0

    def __post_init__(self):
        self.center = np.asarray(self.center, dtype=float).reshape(3)
        self.coeffs = np.atleast_1d(np.asarray(self.coeffs, dtype=float))
        self.exps = np.atleast_1d(np.asarray(self.exps, dtype=float))
        if self.coeffs.shape != self.exps.shape:
            raise ValueError("coeffs and exps must have the same size")
        if self.L < 0:
            raise ValueError("L must be >= 0")

    @property
    def nprims(self):
        return len(self.exps)

    @property
    def sph_size(self):
        return 2 * self.L + 1


@dataclass
class Shells:
    shells: list = field(default_factory=list)

    def __len__(self):
        return len(self.shells)

    def __iter__(self):
        return iter(self.shells)

    def __getitem__(self, i):
        return self.shells[i]

    @property
    def nshells(self):
        return len(self.shells)

    @property
    def sph_size(self):
        return sum(shell.sph_size for shell in self.shells)

    @property
    def l_max(self):
        return max((shell.L for shell in self.shells), default=-1)

    def sph_offsets(self):
        sizes = [shell.sph_size for shell in self.shells]
        return np.concatenate(([0], np.cumsum(sizes)[:-1])).astype(int)

    def as_arrays(self, fortran=False):
        """Pack the basis into (bas_centers, bas_spec, bas_data).

        Coordinates of each distinct center index are stored once, followed by
        per-shell coefficient and exponent blocks.
        """
        offset = 1 if fortran else 0
        nshells = len(self.shells)
        # rows are collected in Python lists and converted once (per-row numpy
        # assignment dominates the cost otherwise)
        data = []
        center_ptrs = {}
        cen_rows = []
        for shell in self.shells:
            xyz = shell.center.tolist()
            key = (shell.center_ind, *xyz)
            ptr = center_ptrs.get(key)
            if ptr is None:
                ptr = center_ptrs[key] = len(data)
                data.extend(xyz)
            cen_rows.append((shell.center_ind, shell.atomic_num, ptr + offset))
        spec_rows = []
        for i, shell in enumerate(self.shells):
            ptr = len(data)
            data.extend(shell.coeffs.tolist())
            data.extend(shell.exps.tolist())
            spec_rows.append((i, shell.L, len(shell.exps), 1, ptr + offset))
        bas_centers = np.array(cen_rows, dtype=np.int32).reshape(nshells, 3)
        bas_spec = np.array(spec_rows, dtype=np.int32).reshape(nshells, 5)
        bas_data = np.array(data, dtype=np.float64)
        return bas_centers, bas_spec, bas_data

    @staticmethod
    def from_arrays(bas_centers, bas_spec, bas_data, fortran=True):
        """Inverse of :meth:`as_arrays` (raw, un-normalized coefficients)."""
        offset = 1 if fortran else 0
        shells = []
        for (center_ind, atomic_num, cptr), (_, L, nprims, _, ptr) in zip(
            np.asarray(bas_centers), np.asarray(bas_spec)
        ):
            cptr -= offset
            ptr -= offset
            center = bas_data[cptr : cptr + 3]
            coeffs = bas_data[ptr : ptr + nprims]
            exps = bas_data[ptr + nprims : ptr + 2 * nprims]
            shells.append(Shell(int(L), center, coeffs, exps, int(center_ind), int(atomic_num)))
        return Shells(shells)
