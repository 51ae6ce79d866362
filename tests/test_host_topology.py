"""The library's host-side molecule pipeline (typing, terms, parameters, round packing) vs the oracle (CPU)."""
import re
import os

import numpy as np
import pytest

from surfmol_b200 import synth

INT_KEYS = ["neighs", "neighBs", "bonds", "angs", "ang_ngs", "dihs", "dih_ngs", "invs", "inv_ngs"]
REAL_KEYS = ["bparams", "angp", "dihp", "invp", "req"]


def molecules():
    out = [synth.config0(0)]
    yield "config0", out[0].Z[0], out[0].pos[0], out[0].q[0]
    rng = np.random.default_rng(7)
    for n in [12, 20, 57, 133, 400, 1200]:
        m = synth.ragged_molecule(rng, n)
        p = synth.place(rng, m, (1.0, 2.0), 3.0)
        yield f"ragged{n}", m.Z, p, synth.charges(rng, m.n)


@pytest.mark.parametrize("name,Z,pos,q", list(molecules()))
def test_topology_matches_oracle(oracle, name, Z, pos, q):
    from surfmol_b200 import Topology
    T = Topology(Z, pos, q).export()
    O = oracle.System.from_molecule(Z, pos, q).export()
    for k in INT_KEYS:
        assert np.array_equal(T[k], O[k]), k
    for k in REAL_KEYS:
        assert np.array_equal(T[k], O[k]), k      # same formulas in the same order: bitwise
    assert T["types"] == O["types"]


def test_pentacene_types_and_counts(oracle):
    import json
    from surfmol_b200 import Topology
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "pentacene.json")))
    T = Topology(d["Z"], d["pos"])
    assert T.counts[1:] == [40, 66, 104, 66]


@pytest.mark.parametrize("team", [32, 64, 128, 256])
def test_round_packing_invariants(team):
    """Each term appears exactly once; inside a round the atoms of each role are distinct."""
    from surfmol_b200 import Topology
    rng = np.random.default_rng(3)
    for n in [40, 150, 420]:
        m = synth.ragged_molecule(rng, n)
        T = Topology(m.Z, synth.place(rng, m, (0, 0), 3.0))
        e = T.export()
        rounds, arrs = T.rounds(team)
        for kind, (cnt, arr, terms, R) in enumerate([(rounds[0], arrs[0], e["angs"], 3),
                                                      (rounds[1], arrs[1], e["dihs"], 4),
                                                      (rounds[2], arrs[2], e["invs"], 4)]):
            a = arr.reshape(cnt, team, 4)
            live = a[:, :, 0] >= 0
            # angles and dihedrals may be packed reversed (k-j-i, l-k-j-i): compare canonical forms
            canon = (lambda x: min(tuple(x), tuple(x[::-1]))) if kind < 2 else tuple
            got = sorted(canon(x[:R]) for x in a[live])
            assert got == sorted(canon(t) for t in terms)
            for r in range(cnt):
                rows = a[r][live[r]]
                for k in range(R):
                    assert len(set(rows[:, k])) == len(rows)


def test_rejects_unknown_element():
    from surfmol_b200 import Topology, SmrError
    with pytest.raises(SmrError):
        Topology([6, 92], [[0, 0, 0], [1.5, 0, 0]])


def test_rejects_overbonded_atom():
    from surfmol_b200 import Topology, SmrError
    pos = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1]], float)
    with pytest.raises(SmrError):
        Topology([6, 1, 1, 1, 1, 1], pos)


def test_autotuner_probe_copies_move_laterally():
    """Probe copies of a sample system keep its shape and height and sit at distinct lateral offsets."""
    from surfmol_b200.autotune import copy_start
    P = np.random.default_rng(0).normal(0, 3, (30, 3))
    assert copy_start(P, 0) is P
    shifts = []
    for c in range(1, 8):
        Q = copy_start(P, c)
        d = Q - P
        assert np.allclose(d, d[0]) and d[0, 2] == 0.0 and 0 <= d[0, 0] < 37 and 0 <= d[0, 1] < 37
        shifts.append(tuple(np.round(d[0, :2], 6)))
    assert len(set(shifts)) == len(shifts)
