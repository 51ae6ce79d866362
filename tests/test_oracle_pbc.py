"""The oracle's periodic systems (opencl/UFF.cl:141-236 bond shifts through neighCell, 1592-1650 NB
image sums) on the CPU: periodic topology building, forces as gradients, extensivity of a periodic
ribbon, and images that are too far to matter."""
import numpy as np
import pytest

from surfmol_b200 import synth


def ribbon(ncell, seed=0):
    m, lat = synth.polyacene_ribbon(ncell)
    rng = np.random.default_rng(seed)
    return m, lat, rng


def test_ribbon_topology_and_cells(oracle):
    m, lat, _ = ribbon(3)
    S = oracle.System.from_molecule(m.Z, m.pos, None, lattice=lat)
    assert (S.n, S.nbonds) == (18, 21)                                  # 7 bonds per C4H2 repeat
    cells = S.cells()
    ex = S.export()
    # a bond crossing the cell carries +1 at one end and -1 at the other (x field, 4-bit two's complement)
    crossing = [(a, s) for a in range(S.n) for s in range(4) if cells[a, s]]
    assert len(crossing) == 4                                           # 2 bonds cross, seen from both ends
    for a, s in crossing:
        b = ex["neighs"][a, s]
        back = [t for t in range(4) if ex["neighs"][b, t] == a][0]
        assert {cells[a, s], cells[b, back]} == {1, 15}
    assert set(ex["types"]) == {"C_R", "H_"}


def test_small_cells_refused(oracle):
    m, lat, _ = ribbon(1)
    with pytest.raises(ValueError, match="cell too small"):
        oracle.System.from_molecule(m.Z, m.pos, None, lattice=lat)


@pytest.mark.parametrize("npbc,rcut", [((1, 0, 0), 0.0), ((2, 0, 0), 0.0), ((1, 0, 0), 6.0)])
def test_forces_are_gradients(oracle, npbc, rcut):
    m, lat, rng = ribbon(3, seed=1)
    q = synth.charges(rng, m.n)
    P = m.pos + rng.normal(0, 0.05, m.pos.shape)
    S = oracle.System.from_molecule(m.Z, m.pos, q, lattice=lat)
    nb = dict(lvec=lat, npbc=npbc, rcut=rcut)
    F, _, Ec = S.eval(P, **nb)
    h = 1e-6
    for a in (0, 2, 5, 17):                                              # crossing-bond atoms among them
        for k in range(3):
            d = np.zeros_like(P); d[a, k] = h
            Ep = S.eval(P + d, **nb)[2][0]
            Em = S.eval(P - d, **nb)[2][0]
            assert abs(-(Ep - Em) / (2 * h) - F[a, k]) < 2e-5 * max(1.0, abs(F[a, k])), (a, k)


def test_extensive_over_cells(oracle):
    """With a cutoff shorter than the 3-repeat cell, a 6-repeat cell holds exactly twice the energy
    and each atom the force of its copy in the 3-repeat cell."""
    m3, lat3, rng = ribbon(3, seed=2)
    m6, lat6 = synth.polyacene_ribbon(6)
    q3 = synth.charges(rng, m3.n)
    P3 = m3.pos + rng.normal(0, 0.03, m3.pos.shape)
    per = lat3[0, 0]
    P6 = np.concatenate([P3, P3 + [per, 0.0, 0.0]])
    q6 = np.concatenate([q3, q3])
    S3 = oracle.System.from_molecule(m3.Z, m3.pos, q3, lattice=lat3)
    # the 6-repeat cell built from its own ideal geometry; the ideal 3-repeat atoms map to k and k+18
    Z6 = np.concatenate([m3.Z, m3.Z])
    S6 = oracle.System.from_molecule(Z6, np.concatenate([m3.pos, m3.pos + [per, 0, 0]]), q6, lattice=lat6)
    F3, _, E3 = S3.eval(P3, lvec=lat3, npbc=(1, 0, 0), rcut=6.0)
    F6, _, E6 = S6.eval(P6, lvec=lat6, npbc=(1, 0, 0), rcut=6.0)
    assert abs(E6[0] - 2 * E3[0]) < 1e-10 * abs(E3[0])
    for c in range(1, 7):
        assert abs(E6[c] - 2 * E3[c]) < 1e-10 * max(1.0, abs(E3[c])), c
    assert np.abs(F6[:18] - F3).max() < 1e-10 and np.abs(F6[18:] - F3).max() < 1e-10


def test_far_images_change_nothing(oracle):
    rng = np.random.default_rng(3)
    m = synth.polyaromatic_40(rng)
    P = synth.place(rng, m, (0.0, 0.0), 0.0, z_top=0.0)
    S = oracle.System.from_molecule(m.Z, P, np.zeros(m.n))
    F0, _, E0 = S.eval(P)
    lat = np.diag([1e4, 1e4, 0.0])
    F1, _, E1 = S.eval(P, lvec=lat, npbc=(1, 1, 0))
    assert np.abs(F1 - F0).max() < 1e-12 and abs(E1[0] - E0[0]) < 1e-12
    # with images nearer than the molecule's size they do act
    F2, _, E2 = S.eval(P, lvec=np.diag([12.0, 12.0, 0.0]), npbc=(1, 1, 0))
    assert abs(E2[5] - E0[5]) > 1e-3
