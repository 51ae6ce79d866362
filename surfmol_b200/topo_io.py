"""Topology files of the reference, read and written.

Two formats, both produced by the reference's topology builder:

* TopologyData JSON (crates/libs/moltopo/src/export.rs:12-74): ``natoms``, ``elements`` (symbols),
  ``positions`` ([x, y, z] in A), ``bonds`` ([i, j]), ``angles`` ([i, j, k], centre j),
  ``dihedrals`` ([i, j, k, l]), ``inversions`` ([i, j, k, l], centre i) and optional parameter
  arrays (written empty by the reference).
* UFFTOPO binary (crates/apps/buildff/src/main.rs:10-28): the 7-byte magic ``UFFTOPO``, a version
  byte (1), seven little-endian int32 (natoms, nbonds, nangles, ndihedrals, ninversions, ntypes,
  flags), then positions (natoms x 3 float64), per-atom type indices (int32), bonds (x 2 int32),
  angles (x 3), dihedrals (x 4), inversions (x 4) and the type table (ntypes x 8 bytes, UFF type
  names padded with spaces).

A loaded molecule goes to the library with its lists as they are (``smr_add_listed_molecule``):
the reference's Uff::from_topology (crates/libs/molff/src/uff.rs:238-240) also takes the lists
from the file.  This is a host-side reader; files carry no charges, so those are passed apart.
"""
from __future__ import annotations

import json
import struct

import numpy as np

SYMBOLS = {1: "H", 6: "C", 7: "N", 8: "O", 9: "F", 11: "Na", 14: "Si", 15: "P", 16: "S", 17: "Cl"}
Z_OF = {v: k for k, v in SYMBOLS.items()}
MAGIC = b"UFFTOPO"


def _arr(x, w, dt):
    a = np.asarray(x if len(x) else np.zeros((0, w)), dtype=dt)
    return a.reshape(-1, w)


def read_json(path) -> dict:
    """TopologyData JSON -> dict(Z, elements, positions, bonds, angles, dihedrals, inversions)."""
    d = json.load(open(path))
    elements = list(d["elements"])
    if len(elements) != d["natoms"]:
        raise ValueError(f"{path}: {len(elements)} elements for natoms={d['natoms']}")
    Z = np.array([Z_OF[e] for e in elements], np.int32)
    return dict(Z=Z, elements=elements, types=None, positions=_arr(d["positions"], 3, np.float64),
                bonds=_arr(d["bonds"], 2, np.int32), angles=_arr(d["angles"], 3, np.int32),
                dihedrals=_arr(d["dihedrals"], 4, np.int32), inversions=_arr(d["inversions"], 4, np.int32))


def write_json(path, Z, positions, bonds, angles, dihedrals, inversions):
    """Write TopologyData JSON in the reference's field order (parameter arrays empty, as it does)."""
    elements = [SYMBOLS[int(z)] for z in Z]
    d = {"natoms": len(elements), "elements": elements,
         "positions": np.asarray(positions, float).reshape(-1, 3).tolist(),
         "bonds": np.asarray(bonds, int).reshape(-1, 2).tolist(),
         "angles": np.asarray(angles, int).reshape(-1, 3).tolist(),
         "dihedrals": np.asarray(dihedrals, int).reshape(-1, 4).tolist(),
         "inversions": np.asarray(inversions, int).reshape(-1, 4).tolist(),
         "bond_params": [], "angle_params": [], "dihedral_params": [], "inversion_params": [], "atom_params": []}
    with open(path, "w") as f:
        json.dump(d, f, indent=2)


def read_ufftopo(path) -> dict:
    """UFFTOPO binary -> dict(Z, types, positions, bonds, angles, dihedrals, inversions)."""
    b = open(path, "rb").read()
    if b[:7] != MAGIC:
        raise ValueError(f"{path}: not a UFFTOPO file")
    if b[7] != 1:
        raise ValueError(f"{path}: UFFTOPO version {b[7]} (reader knows 1)")
    na, nb, nang, ndih, ninv, nt, _flags = struct.unpack_from("<7i", b, 8)
    off = 36

    def take(count, dt, w):
        nonlocal off
        a = np.frombuffer(b, dtype=dt, count=count * w, offset=off).reshape(count, w) if count else np.zeros((0, w), dt)
        off += count * w * np.dtype(dt).itemsize
        return a.copy()
    pos = take(na, "<f8", 3)
    tidx = take(na, "<i4", 1)[:, 0]
    bonds = take(nb, "<i4", 2)
    angles = take(nang, "<i4", 3)
    dihs = take(ndih, "<i4", 4)
    invs = take(ninv, "<i4", 4)
    table = [b[off + 8 * k: off + 8 * k + 8].decode().rstrip(" \x00") for k in range(nt)]
    if off + 8 * nt != len(b):
        raise ValueError(f"{path}: {len(b) - off - 8 * nt} trailing bytes")
    types = [table[t] for t in tidx]
    Z = np.array([Z_OF[t.split("_")[0]] for t in types], np.int32)
    return dict(Z=Z, elements=[SYMBOLS[int(z)] for z in Z], types=types, positions=pos.astype(np.float64),
                bonds=bonds.astype(np.int32), angles=angles.astype(np.int32), dihedrals=dihs.astype(np.int32),
                inversions=invs.astype(np.int32))


def write_ufftopo(path, types, positions, bonds, angles, dihedrals, inversions):
    """Write a UFFTOPO file (type table sorted and deduplicated, as the reference writes it)."""
    table = sorted(set(types))
    idx = np.array([table.index(t) for t in types], "<i4")
    pos = np.asarray(positions, "<f8").reshape(-1, 3)
    arrs = [np.asarray(x, "<i4").reshape(-1, w) for x, w in ((bonds, 2), (angles, 3), (dihedrals, 4), (inversions, 4))]
    head = MAGIC + bytes([1]) + struct.pack("<7i", len(types), len(arrs[0]), len(arrs[1]), len(arrs[2]), len(arrs[3]),
                                            len(table), 0)
    body = pos.tobytes() + idx.tobytes() + b"".join(a.tobytes() for a in arrs)
    names = b"".join(t.encode()[:8].ljust(8, b" ") for t in table)
    with open(path, "wb") as f:
        f.write(head + body + names)


def read(path) -> dict:
    """Either format, by content."""
    with open(path, "rb") as f:
        magic = f.read(7)
    return read_ufftopo(path) if magic == MAGIC else read_json(path)
