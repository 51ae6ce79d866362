"""Periodic systems on the GPU against the FP64 oracle: bonds to a partner's image in the next cell
(opencl/UFF.cl:141-236) and NB sums over PBC images (UFF.cl:1592-1650), per-system lattices."""
import numpy as np
import pytest

from surfmol_b200 import synth
from tests.gpu_helpers import F_RTOL, build_device_grid, force_err, small_slab_grid

pytestmark = pytest.mark.gpu
E_NB, E_GRID = 5, 6


@pytest.fixture(scope="module")
def env():
    from surfmol_b200 import RelaxMulti
    slab, dims, p0, step = small_slab_grid()
    R = RelaxMulti(max_systems=256, max_atoms=40000)
    R.set_nb(1.0, 1.5)
    g = build_device_grid(R, slab, dims, p0, step)
    yield R, slab, g
    R.finish()


def ribbon_on_slab(rng, ncell, slab, jitter=0.05):
    m, lat = synth.polyacene_ribbon(ncell)
    lat = lat.astype(np.float32).astype(np.float64)          # the lattice the GPU sees
    P = m.pos + [0.4 * slab.Lx, 0.4 * slab.Ly, slab.z_top + 3.2] + rng.normal(0, jitter, m.pos.shape)
    return m.Z, P, lat, synth.charges(rng, m.n)


def oracle_eval(oracle, g, Z, P, q, lat, npbc, rcut=0.0, build_lat=None):
    S = oracle.System.from_molecule(Z, P, q, lattice=build_lat)
    return S, S.eval(P.astype(np.float32).astype(np.float64), oracle.Grid(g["coef"], g["p0"], g["step"]),
                     lvec=lat, npbc=npbc, rcut=rcut)


def test_topology_matches_oracle(env, oracle):
    R, slab, _ = env
    Z, P, lat, q = ribbon_on_slab(np.random.default_rng(0), 3, slab)
    tid = R.add_molecule_pbc(Z, P, lat, q)
    S = oracle.System.from_molecule(Z, P, q, lattice=lat)
    ex = S.export()
    assert np.array_equal(R.topology_cells(tid), S.cells())
    assert R.topology_counts(tid)[:5] == [S.n, S.nbonds, S.nang, S.ndih, S.ninv]
    got = R.topology_export(tid)
    for k in ("neighs", "bonds", "angs", "dihs", "invs", "type_id"):
        assert np.array_equal(got[k], ex[k]), k


@pytest.mark.parametrize("ncell,npbc,rcut,team", [(3, (1, 0, 0), 0.0, 32), (3, (2, 0, 0), 0.0, 64), (4, (1, 0, 0), 6.0, 128),
                                                  (6, (1, 0, 0), 0.0, 256), (3, (0, 0, 0), 0.0, 32)])
def test_periodic_ribbon_matches_oracle(env, oracle, ncell, npbc, rcut, team):
    R, slab, g = env
    R.set_nb(1.0, 1.5, rcut)
    R.set_team_size(1 << 20, team)
    try:
        Z, P, lat, q = ribbon_on_slab(np.random.default_rng(ncell + team), ncell, slab)
        tid = R.add_molecule_pbc(Z, P, lat, q, npbc=npbc)
        sl = R.add_systems([tid], [P])
        lv, nimg = R.get_pbc(sl[0])
        assert np.array_equal(nimg, npbc) and np.allclose(lv, lat)
        F, E = R.eval_forces(sl)
        _, (Fo, Eao, Eco) = oracle_eval(oracle, g, Z, P, q, lat, npbc, rcut, build_lat=lat)
        assert force_err(F[0], Fo) < F_RTOL
        assert np.abs(F[0][:, 3] - Eao).max() < 1e-5 * max(1.0, np.abs(Eao).max())
        for c in range(1, 7):
            assert abs(E[0, c] - Eco[c]) < 2e-6 * max(1.0, abs(Eco[c])), (c, E[0, c], Eco[c])
        R.remove_systems(sl)
    finally:
        R.set_nb(1.0, 1.5)
        R.set_team_size(1 << 20, 0)


def test_isolated_molecule_meets_its_images(env, oracle):
    """smr_set_pbc on a molecule without periodic bonds: NB over its copies in a 2D cell."""
    R, slab, g = env
    rng = np.random.default_rng(5)
    m = synth.polyaromatic_40(rng)
    P = synth.place(rng, m, (0.5 * slab.Lx, 0.5 * slab.Ly), 3.0, z_top=slab.z_top)
    q = synth.charges(rng, m.n)
    lat = np.array([[13.5, 0.0, 0.0], [1.25, 12.75, 0.0], [0.0, 0.0, 0.0]])
    sl = R.add_systems([R.add_molecule(m.Z, P, q)], [P])
    F0, E0 = R.eval_forces(sl)
    R.set_pbc(sl, lat, (1, 1, 0))
    F, E = R.eval_forces(sl)
    _, (Fo, Eao, Eco) = oracle_eval(oracle, g, m.Z, P, q, lat, (1, 1, 0))
    assert force_err(F[0], Fo) < F_RTOL
    assert abs(E[0, E_NB] - Eco[E_NB]) < 2e-6 * max(1.0, abs(Eco[E_NB]))
    assert abs(E[0, E_NB] - E0[0, E_NB]) > 1e-3                       # the images act
    R.set_pbc(sl, np.zeros((3, 3)), (0, 0, 0))                         # off again
    F1, E1 = R.eval_forces(sl)
    assert force_err(F1[0], F0[0][:, :3]) < 1e-6
    R.remove_systems(sl)


def test_relax_periodic_ribbon_in_a_mix(env, oracle):
    """A periodic ribbon relaxes to the oracle's minimum, and bit for bit as in a mix with isolated
    molecules (which keep their own forms)."""
    R, slab, g = env
    rng = np.random.default_rng(7)
    Z, P, lat, q = ribbon_on_slab(rng, 4, slab, jitter=0.08)
    tid = R.add_molecule_pbc(Z, P, lat, q)
    a = R.add_systems([tid], [P])
    R.run_fire(3000, step_budget=3000, fconv=1e-3)
    alone = R.download(a)
    assert alone["status"][0] == 1, alone
    S = oracle.System.from_molecule(Z, P, q, lattice=lat)
    Fo, _, _ = S.eval(R.download_pos64(a)[0], oracle.Grid(g["coef"], g["p0"], g["step"]), lvec=lat, npbc=(1, 0, 0))
    assert np.sqrt((Fo ** 2).sum(1)).max() < 3e-3
    R.remove_systems(a)
    others = [synth.polyaromatic_40(rng) for _ in range(3)]
    Ps = [synth.place(rng, o, (rng.uniform(0, slab.Lx), rng.uniform(0, slab.Ly)), 3.0, z_top=slab.z_top) for o in others]
    tids = [R.add_molecule(o.Z, p, synth.charges(rng, o.n)) for o, p in zip(others, Ps)]
    b = R.add_systems(tids[:2] + [tid] + tids[2:], Ps[:2] + [P] + Ps[2:])
    R.run_fire(3000, step_budget=3000, fconv=1e-3)
    mix = R.download(b)
    assert np.array_equal(mix["pos"][2], alone["pos"][0]) and mix["steps"][2] == alone["steps"][0]
    R.remove_systems(b)


def test_pbc_errors(env):
    from surfmol_b200.relax import SmrError
    R, slab, _ = env
    m, lat = synth.polyacene_ribbon(1)
    with pytest.raises(SmrError, match="cell too small"):
        R.add_molecule_pbc(m.Z, m.pos, lat)
    Z, P, lat, q = ribbon_on_slab(np.random.default_rng(9), 3, slab)
    with pytest.raises(SmrError):
        R.add_molecule_pbc(Z, P, lat, q, npbc=(8, 0, 0))
    tid = R.add_molecule_pbc(Z, P, lat, q)
    sl = R.add_systems([tid], [P])
    with pytest.raises(SmrError, match="cross"):
        R.set_pbc(sl, np.zeros((3, 3)), (0, 0, 0))                     # its bonds cross axis a
    with pytest.raises(SmrError):
        R.set_pbc(sl, lat, (0, -1, 0))
    R.set_pbc(sl, lat, (2, 0, 0))
    assert list(R.get_pbc(sl[0])[1]) == [2, 0, 0]
    R.remove_systems(sl)
