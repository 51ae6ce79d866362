"""Multi-replica RAFF on the CPU: the host preparation of crates/libs/oclff/src/pack.rs (oracle
restatement pinned to the reference's own unit tests, the library's native builders against it)
and the FP64 oracle step on cases with known answers."""
import math

import numpy as np
import pytest

from surfmol_b200 import synth

WATER_BONDS = [(0, 1), (0, 2)]


def water():
    """O at the origin, H at 0.96 A, 104.5 degrees (the geometry of pack.rs:319-330's tests)."""
    a = math.radians(104.5)
    return np.array([8, 1, 1]), np.array([[0, 0, 0], [0.96 * math.cos(a / 2), 0.96 * math.sin(a / 2), 0],
                                          [0.96 * math.cos(a / 2), -0.96 * math.sin(a / 2), 0]])


def methanol():
    t = math.radians(109.5)
    c, o = [0, 0, 0], [1.43, 0, 0]
    h = [[-1.09, 0, 0], [1.09 * math.cos(t), 1.09 * math.sin(t), 0],
         [1.09 * math.cos(t), 1.09 * math.sin(t) * math.cos(2.0944), 1.09 * math.sin(t) * math.sin(2.0944)]]
    ho = [1.43 + 0.96 * math.cos(math.pi - math.radians(108.5)), 0.96 * math.sin(math.pi - math.radians(108.5)), 0]
    return np.array([6, 8, 1, 1, 1, 1]), np.array([c, o] + h + [ho]), [(0, 1), (0, 2), (0, 3), (0, 4), (1, 5)]


def test_oracle_builders_match_reference_tests(oracle):
    """pack.rs:362-433: node order, neighbours, exclusions, back-slots and ports of water."""
    Z, P = water()
    perm, nnode = oracle.raff_node_order(3, WATER_BONDS)
    assert list(perm) == [0, 1, 2] and nnode == 1                 # O is the node (degree 2)
    ng = oracle.raff_build_neighs(3, WATER_BONDS)
    assert list(ng[0]) == [1, 2, -1, -1] and list(ng[1]) == [0, -1, -1, -1] and list(ng[2]) == [0, -1, -1, -1]
    e1, e2 = oracle.raff_exclusions(ng)
    assert list(e1[0][:2]) == [1, 2] and e2[0][0] == -1
    assert e1[1][0] == 0 and e2[1][0] == 2
    bk = oracle.raff_bk_slots(ng, nnode)
    assert bk[1][0] == 0 and bk[2][0] == 1
    pl, k = oracle.raff_ports(P, ng, 200.0)
    assert abs(pl[0, 0, 0] - P[1, 0]) < 1e-5 and abs(pl[0, 0, 1] - P[1, 1]) < 1e-5 and k[0, 0] == 200.0


@pytest.mark.parametrize("which", ["water", "methanol", "pentitol", "random"])
def test_library_builders_match_oracle(oracle, which):
    from surfmol_b200.raff import prepare
    if which == "water":
        Z, P = water(); B = WATER_BONDS
    elif which == "methanol":
        Z, P, B = methanol()
    elif which == "pentitol":
        m = synth.pentitol(); Z, P, B = m.Z, m.pos, m.bonds
    else:                                                          # a random tree of degree <= 4
        rng = np.random.default_rng(4)
        n = 30
        B, deg = [], np.zeros(n, int)
        for i in range(1, n):
            j = int(rng.choice([j for j in range(i) if deg[j] < 4]))
            B.append((j, i)); deg[i] += 1; deg[j] += 1
        Z = rng.choice([1, 6, 7, 8], n); P = rng.normal(0, 3, (n, 3))
    prep = prepare(Z, P, B, k_stiff=150.0)
    perm, nnode = oracle.raff_node_order(len(Z), B)
    assert np.array_equal(prep.perm, perm) and prep.nnode == nnode
    inv = np.empty(len(Z), int); inv[perm] = np.arange(len(Z))
    Bp = [(inv[i], inv[j]) for i, j in B]
    ng = oracle.raff_build_neighs(len(Z), Bp)
    assert np.array_equal(prep.neighs, ng)
    e1, e2 = oracle.raff_exclusions(ng)
    assert np.array_equal(prep.excl1, e1) and np.array_equal(prep.excl2, e2)
    assert np.array_equal(prep.bk_slots, oracle.raff_bk_slots(ng, nnode))
    pl, k = oracle.raff_ports(np.asarray(P, np.float32)[perm], ng, 150.0)
    assert np.array_equal(prep.port_local, pl) and np.array_equal(prep.k, k)
    masses = {1: 1.008, 6: 12.011, 7: 14.007, 8: 15.999}
    assert np.allclose(prep.inv_mass, [1.0 / masses[int(z)] for z in prep.Z], rtol=1e-6)


def topo_of(prep, radius=None, fixmask=None):
    n = prep.natoms
    return dict(radius=np.zeros(n) if radius is None else radius, neighs=prep.neighs, excl1=prep.excl1, excl2=prep.excl2,
                fixmask=np.zeros(n, int) if fixmask is None else fixmask, port_local=prep.port_local[:prep.nnode],
                k=prep.k[:prep.nnode], bk=prep.bk_slots)


def state_of(prep, P, nsys=1):
    pos4 = np.zeros((nsys, prep.natoms, 4))
    pos4[..., :3] = P
    pos4[..., 3] = prep.inv_mass
    quat = np.zeros((nsys, prep.natoms, 4)); quat[..., 3] = 1.0
    return pos4, quat


def test_rest_geometry_is_a_fixed_point(oracle):
    from surfmol_b200.raff import prepare
    m = synth.pentitol()
    prep = prepare(m.Z, m.pos, m.bonds)
    pos4, quat = state_of(prep, prep.pos.astype(np.float64))
    out = oracle.raff_step(pos4, quat, prep.natoms, prep.nnode, 20, topo_of(prep))
    assert np.abs(out["pos"] - pos4).max() < 1e-6 and np.abs(out["dnode"]).max() < 1e-6


def test_perturbed_geometry_relaxes(oracle):
    """From 0.2 A of noise the Jacobi XPBD iteration contracts steadily (about 2.3x per 500 steps
    for this molecule) back to the rest bond lengths."""
    from surfmol_b200.raff import prepare
    m = synth.pentitol()
    prep = prepare(m.Z, m.pos, m.bonds)
    rng = np.random.default_rng(1)
    P = prep.pos + rng.uniform(-0.2, 0.2, prep.pos.shape)
    pos4, quat = state_of(prep, P)
    out = oracle.raff_step(pos4, quat, prep.natoms, prep.nnode, 500, topo_of(prep))
    r0 = np.abs(out["dnode"]).max()
    out = oracle.raff_step(out["pos"], out["quat"], prep.natoms, prep.nnode, 2500, topo_of(prep),
                           dmom=out["dmom"], dqmom=out["dqmom"])
    assert np.abs(out["dnode"]).max() < r0 / 6
    d0 = [np.linalg.norm(prep.pos[i] - prep.pos[j]) for i, j in prep.bonds]
    d1 = [np.linalg.norm(out["pos"][0, i, :3] - out["pos"][0, j, :3]) for i, j in prep.bonds]
    assert np.abs(np.array(d1) - d0).max() < 5e-4


def test_collision_known_answer(oracle):
    """Two free unbonded spheres of radius 1 at distance 1.5: each moves 0.125 apart per unit
    relaxation (half the overlap split by equal inverse masses, halved again)."""
    n = 2
    topo = dict(radius=np.ones(n), neighs=-np.ones((n, 4), int), excl1=-np.ones((n, 4), int),
                excl2=-np.ones((n, 4), int), fixmask=np.zeros(n, int), port_local=np.zeros((0, 4, 4)), k=np.zeros((0, 4)),
                bk=-np.ones((n, 4), int))
    pos4 = np.array([[[0, 0, 0, 1.0], [1.5, 0, 0, 1.0]]])
    quat = np.zeros((1, 2, 4)); quat[..., 3] = 1
    out = oracle.raff_step(pos4, quat, n, 0, 1, topo, relaxation=1.0)
    assert abs(out["coll"][0, 0, 0] + 0.125) < 1e-9 and abs(out["coll"][0, 1, 0] - 0.125) < 1e-9
    assert abs(out["pos"][0, 1, 0] - out["pos"][0, 0, 0] - 1.75) < 1e-9


def test_fixmask_and_plane(oracle):
    from surfmol_b200.raff import prepare
    m = synth.pentitol()
    prep = prepare(m.Z, m.pos, m.bonds)
    rng = np.random.default_rng(2)
    P = prep.pos + rng.uniform(-0.2, 0.2, prep.pos.shape)
    fix = np.zeros(prep.natoms, int)
    fix[0] = 7                                                      # frozen node
    fix[prep.nnode] = 8                                             # a cap pulled onto z = 0
    pos4, quat = state_of(prep, P)
    out = oracle.raff_step(pos4, quat, prep.natoms, prep.nnode, 30, topo_of(prep, fixmask=fix))
    assert np.array_equal(out["pos"][0, 0], pos4[0, 0]) and np.array_equal(out["quat"][0, 0], quat[0, 0])
    # bit 8 moves z onto the plane plus that step's relaxed correction (RRsp3.cl:1999-2003): one
    # step takes the cap from 1.2 A to the size of one correction
    one = oracle.raff_step(pos4, quat, prep.natoms, prep.nnode, 1, topo_of(prep, fixmask=fix))
    assert abs(P[prep.nnode, 2]) > 0.3 and abs(one["pos"][0, prep.nnode, 2]) < 0.05
