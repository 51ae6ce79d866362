"""Topology files (the reference's TopologyData JSON and UFFTOPO binary): round trips, and molecules
loaded from their lists give bitwise the topology our own pipeline builds from the positions."""
import numpy as np
import pytest

from surfmol_b200 import synth
from surfmol_b200.relax import SmrError, Topology
from surfmol_b200.topo_io import read, read_json, read_ufftopo, write_json, write_ufftopo


def molecule(seed, n):
    rng = np.random.default_rng(seed)
    m = synth.ragged_molecule(rng, n) if n != 40 else synth.polyaromatic_40(rng)
    return m.Z, m.pos, synth.charges(rng, m.n)


@pytest.mark.parametrize("seed,n", [(1, 40), (2, 23), (3, 130)])
def test_files_round_trip_and_match_pipeline(tmp_path, seed, n):
    Z, P, q = molecule(seed, n)
    ref = Topology(Z, P, q).export()
    bonds, angs, dihs, invs = ref["bonds"], ref["angs"], ref["dihs"], ref["invs"]
    write_json(tmp_path / "t.json", Z, P, bonds, angs, dihs, invs)
    write_ufftopo(tmp_path / "t.bin", ref["types"], P, bonds, angs, dihs, invs)
    dj, db = read_json(tmp_path / "t.json"), read_ufftopo(tmp_path / "t.bin")
    assert read(tmp_path / "t.bin")["types"] == ref["types"]
    for d in (dj, db):
        assert np.array_equal(d["Z"], Z) and np.allclose(d["positions"], P, rtol=0, atol=0)
        for k, w in (("bonds", bonds), ("angles", angs), ("dihedrals", dihs), ("inversions", invs)):
            assert np.array_equal(d[k], w), k
    # typed from the bond graph (JSON) or from the file's type names (UFFTOPO): same topology
    for types in (None, db["types"]):
        t = Topology.from_lists(dj["Z"], dj["bonds"], dj["angles"], dj["dihedrals"], dj["inversions"], q, types).export()
        for k in ref:
            assert np.array_equal(np.asarray(ref[k]), np.asarray(t[k])), k


def test_bad_files_rejected(tmp_path):
    Z, P, q = molecule(4, 40)
    ref = Topology(Z, P, q).export()
    (tmp_path / "x.bin").write_bytes(b"NOTATOPO" + bytes(40))
    with pytest.raises(ValueError):
        read_ufftopo(tmp_path / "x.bin")
    write_ufftopo(tmp_path / "t.bin", ref["types"], P, ref["bonds"], ref["angs"], ref["dihs"], ref["invs"])
    (tmp_path / "t2.bin").write_bytes((tmp_path / "t.bin").read_bytes() + b"xx")
    with pytest.raises(ValueError):
        read_ufftopo(tmp_path / "t2.bin")
    bad = np.array(ref["angs"]).copy()
    bad[0] = [0, 1, 39]                                       # 0-1-39 is not an angle of the bond graph
    with pytest.raises(SmrError):
        Topology.from_lists(Z, ref["bonds"], bad, ref["dihs"], ref["invs"])
    with pytest.raises(SmrError):
        Topology.from_lists(Z, ref["bonds"], ref["angs"], ref["dihs"], ref["invs"], types=["Xx_9"] * len(Z))
