"""Reader for ORCA wavefunctions stored as BSON (``orca_2json -bson`` output).

The reference's Coulomb-tensor test feeds such a file through pysisyphus
(``tests/test_coulomb_tensor/test_coulomb_tensor.py:7-32``). pysisyphus is not a
dependency here, so this module reads the BSON document itself and builds a
:class:`~pysisyphus_addons.common.shells.Shells` object in the ordering the
reference's kernels use: shells in file order, coordinates in bohr, contraction
coefficients as stored (they refer to normalized primitives).

It also returns the ORCA overlap matrix (``S-Matrix``) permuted from ORCA's
spherical order (p: z, x, y; d: z2, xz, yz, x2-y2, xy) into the m = -l..l order
used here (p: y, z, x; d: xy, yz, z2, xz, x2-y2), which pins the basis
normalization and ordering.
"""

import struct

import numpy as np

from .shells import Shell, Shells

# CODATA 2018 Bohr radius in Angstrom.
BOHR2ANG = 0.529177210903

_L_OF = {"s": 0, "p": 1, "d": 2, "f": 3, "g": 4, "h": 5}


def _cstring(buf, i):
    j = buf.index(b"\x00", i)
    return buf[i:j].decode(), j + 1


def _document(buf, i):
    (size,) = struct.unpack_from("<i", buf, i)
    end = i + size - 1
    i += 4
    out = {}
    while i < end:
        kind = buf[i]
        i += 1
        key, i = _cstring(buf, i)
        if kind == 0x01:
            (val,) = struct.unpack_from("<d", buf, i)
            i += 8
        elif kind == 0x02:
            (n,) = struct.unpack_from("<i", buf, i)
            i += 4
            val = buf[i : i + n - 1].decode()
            i += n
        elif kind in (0x03, 0x04):
            val, i = _document(buf, i)
            if kind == 0x04:
                val = [val[k] for k in sorted(val, key=int)]
        elif kind == 0x05:
            (n,) = struct.unpack_from("<i", buf, i)
            i += 5
            val = bytes(buf[i : i + n])
            i += n
        elif kind == 0x08:
            val = bool(buf[i])
            i += 1
        elif kind == 0x0A:
            val = None
        elif kind == 0x10:
            (val,) = struct.unpack_from("<i", buf, i)
            i += 4
        elif kind == 0x12:
            (val,) = struct.unpack_from("<q", buf, i)
            i += 8
        else:
            raise ValueError(f"unsupported BSON element type {kind:#x}")
        out[key] = val
    return out, end + 1


def read_bson(path):
    with open(path, "rb") as handle:
        buf = handle.read()
    doc, _ = _document(buf, 0)
    return doc


# Position, in ORCA's order, of each m = -l..l function.
_ORCA_TO_M = {0: [0], 1: [2, 0, 1], 2: [4, 2, 0, 1, 3]}


def shells_from_orca(doc):
    mol = doc["Molecule"]
    factor = 1.0 / BOHR2ANG if mol.get("CoordinateUnits", "Angs").startswith("Ang") else 1.0
    shells = []
    for atom in mol["Atoms"]:
        xyz = np.array(atom["Coords"], dtype=float) * factor
        z = int(atom["ElementNumber"])
        for bf in atom["BasisFunctions"]:
            L = _L_OF[bf["Shell"]]
            shells.append(Shell(L, xyz, bf["Coefficients"], bf["Exponents"], int(atom["Idx"]), z))
    return Shells(shells)


def orca_to_m_permutation(shells):
    """Index array ``perm`` with ``M_m = M_orca[perm][:, perm]`` (L <= 2)."""
    perm = []
    start = 0
    for shell in shells:
        if shell.L not in _ORCA_TO_M:
            raise NotImplementedError("ORCA reordering is implemented for L <= 2")
        perm.extend(start + k for k in _ORCA_TO_M[shell.L])
        start += shell.sph_size
    return np.array(perm)


def load_orca_bson(path):
    """Return (shells, S) with S in m = -l..l order."""
    doc = read_bson(path)
    shells = shells_from_orca(doc)
    S = np.array(doc["Molecule"]["S-Matrix"], dtype=float)
    perm = orca_to_m_permutation(shells)
    return shells, S[np.ix_(perm, perm)]
