"""Folded-surface substrate (SurfaceFolded, crates/libs/surfff/src/lib.rs:126-351) on the GPU
against the FP64 oracle: per-atom forces and energies, the force clamp, relaxation, and batched vs
plain trajectories bit for bit."""
import numpy as np
import pytest

from surfmol_b200 import synth
from surfmol_b200.folded import FoldedSurface, nacl
from tests.gpu_helpers import F_RTOL, force_err

pytestmark = pytest.mark.gpu
E_GRID = 6


@pytest.fixture(scope="module")
def R():
    from surfmol_b200 import RelaxMulti
    r = RelaxMulti(max_systems=2048, max_atoms=200000)
    r.set_nb(1.0, 1.5)
    yield r
    r.finish()


def skewed():
    """Oblique lattice, non-integer harmonics and 5 z decays with coefficients on every channel."""
    rng = np.random.default_rng(2)
    s = FoldedSurface(6.1, 2.3, 0.4, 5.2, [0.0, 1.0, 2.0, 0.5], [0.0, 1.0, 3.0], [2.4, 1.2, 0.6, 0.3, 0.9],
                      [0.0, 0.0, 0.0, 0.0, -0.5])
    # the fastest decay (kz = 2.4, basis 0..11) is Pauli only: a constant 40 above harmonics
    # summing to less, so the wall is repulsive everywhere; charge, London and small Pauli terms
    # on the slower decays
    s.cq[:] = rng.normal(0, 0.5, s.nbasis)
    s.cl[:] = -rng.uniform(0, 1.0, s.nbasis)
    s.cp[:] = rng.uniform(-0.5, 0.5, s.nbasis)
    s.cq[:12] = 0.0
    s.cl[:12] = 0.0
    s.cp[:12] = rng.uniform(-2.5, 2.5, 12)
    s.cp[0] = 40.0
    return s


def on_surface(rng, n, height=2.5):
    m = synth.ragged_molecule(rng, n) if n != 40 else synth.polyaromatic_40(rng)
    p = synth.place(rng, m, (rng.uniform(0, 12), rng.uniform(0, 12)), height, z_top=0.0)
    return m.Z, p, synth.charges(rng, m.n)


@pytest.mark.parametrize("surf", ["nacl", "skewed"])
@pytest.mark.parametrize("n,team,form", [(40, 32, 0), (90, 64, 0), (250, 128, 1), (40, 32, 2), (600, 512, 0)])
def test_forces_energies_match_oracle(R, oracle, surf, n, team, form):
    s = nacl() if surf == "nacl" else skewed()
    R.set_surface_folded(s)
    R.set_team_size(1 << 20, team)
    R.set_schedule(0, team, form)
    try:
        rng = np.random.default_rng(n + team)
        Z, P, q = on_surface(rng, n)
        sl = R.add_systems([R.add_molecule(Z, P, q)], [P])
        F, E = R.eval_forces(sl)
        S = oracle.System.from_molecule(Z, P, q)
        Fo, Eao, Eco = S.eval(P.astype(np.float32).astype(np.float64), oracle.Folded(**s.as_dict()))
        assert force_err(F[0], Fo) < F_RTOL
        assert np.abs(F[0][:, 3] - Eao).max() < 1e-5 * max(1.0, np.abs(Eao).max())
        assert abs(Eco[E_GRID]) > 1e-4                                     # the surface acts
        assert abs(E[0, E_GRID] - Eco[E_GRID]) < 2e-6 * max(1.0, abs(Eco[E_GRID]))
        R.remove_systems(sl)
    finally:
        R.set_team_size(1 << 20, 0)
        R.set_schedule(0, 0, 0)
        R.set_surface_folded(None)


@pytest.mark.parametrize("fmax", [100.0, 0.02])
def test_lone_atoms_and_clamp(R, oracle, fmax):
    """Lone atoms (only the surface acts) from deep inside the repulsive wall, where the clamp holds
    |F| at fmax, to far above the surface; positions on both sides of the cell's edges."""
    s = nacl()
    s.fmax = fmax
    R.set_surface_folded(s)
    try:
        rng = np.random.default_rng(7)
        pts = np.column_stack([rng.uniform(-12, 24, 64), rng.uniform(-12, 24, 64), np.linspace(-15.0, 12.0, 64)])
        tids, Ps, Zs = [], [], []
        for k, p in enumerate(pts):
            Z = np.array([(6, 8, 1, 7)[k % 4]])
            tids.append(R.add_molecule(Z, p[None, :], np.array([0.3 * np.sin(k)])))
            Ps.append(p[None, :]); Zs.append(Z)
        sl = R.add_systems(tids, Ps)
        F, E = R.eval_forces(sl)
        folded = oracle.Folded(**s.as_dict())
        nclamp = 0
        for k in range(len(pts)):
            S = oracle.System.from_molecule(Zs[k], Ps[k], np.array([0.3 * np.sin(k)]))
            Fo, Eao, _ = S.eval(Ps[k].astype(np.float32).astype(np.float64), folded)
            nclamp += abs(np.linalg.norm(Fo[0]) - fmax) < 1e-9 * fmax
            assert np.abs(F[k][0, :3] - Fo[0]).max() < F_RTOL * max(1.0, np.abs(Fo[0]).max()), k
            assert abs(F[k][0, 3] - Eao[0]) < 1e-5 * max(1.0, abs(Eao[0])), k
        assert nclamp >= 8                                                  # the clamp was exercised
        R.remove_systems(sl)
    finally:
        R.set_surface_folded(None)


def test_relaxed_structure_is_oracle_minimum(R, oracle):
    s = nacl()
    R.set_surface_folded(s)
    try:
        rng = np.random.default_rng(11)
        Z, P, q = on_surface(rng, 40, height=3.0)
        sl = R.add_systems([R.add_molecule(Z, P, q)], [P])
        R.run_fire(4000, step_budget=4000, fconv=1e-3)
        out = R.download(sl)
        assert out["status"][0] == 1, out
        S = oracle.System.from_molecule(Z, P, q)
        Fo, _, _ = S.eval(R.download_pos64(sl)[0], oracle.Folded(**s.as_dict()))
        assert np.sqrt((Fo ** 2).sum(1)).max() < 3e-3
        ro = S.relax(P.astype(np.float32).astype(np.float64), oracle.Folded(**s.as_dict()), max_steps=4000, fconv=1e-3)
        assert ro["conv"]
        R.remove_systems(sl)
    finally:
        R.set_surface_folded(None)


def test_batched_plain_alone_mix_bitwise(R):
    R.set_surface_folded(skewed())
    try:
        rng = np.random.default_rng(12)
        mols = [on_surface(rng, n) for n in (40, 25, 130, 300)]
        tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
        a = R.add_systems(tids, [m[1] for m in mols])
        R.run_fire(150, step_budget=150, fconv=1e-6)
        mix = R.download(a)
        R.remove_systems(a)
        b = R.add_systems([tids[2]], [mols[2][1]])
        for _ in range(3):
            R.run_fire(50, step_budget=150, fconv=1e-6)
        alone = R.download(b)
        R.remove_systems(b)
        c = R.add_systems([tids[2]], [mols[2][1]])
        R.run_fire(150, step_budget=150, fconv=1e-6, mode=1)
        plain = R.download(c)
        R.remove_systems(c)
        assert np.array_equal(mix["pos"][2], alone["pos"][0])
        assert np.array_equal(mix["pos"][2], plain["pos"][0])
        assert np.array_equal(mix["forces"][2], plain["forces"][0])
        assert mix["steps"][2] == alone["steps"][0] == plain["steps"][0] == 150
    finally:
        R.set_surface_folded(None)


def test_switching_substrates(R, oracle):
    """Folded surface on, then off again: the grid path returns unchanged; without a grid the
    substrate is absent."""
    from tests.gpu_helpers import build_device_grid, small_slab_grid
    slab, dims, p0, step = small_slab_grid()
    g = build_device_grid(R, slab, dims, p0, step)
    rng = np.random.default_rng(13)
    m = synth.polyaromatic_40(rng)
    P = synth.place(rng, m, (3.0, 3.0), 3.0, z_top=slab.z_top)
    q = synth.charges(rng, m.n)
    sl = R.add_systems([R.add_molecule(m.Z, P, q)], [P])
    F0, E0 = R.eval_forces(sl)
    R.set_surface_folded(nacl(z0=slab.z_top))
    F1, E1 = R.eval_forces(sl)
    R.set_surface_folded(None)
    F2, E2 = R.eval_forces(sl)
    assert np.array_equal(F0[0], F2[0]) and np.array_equal(E0, E2)
    assert not np.array_equal(F0[0], F1[0])
    S = oracle.System.from_molecule(m.Z, P, q)
    Fo, _, _ = S.eval(P.astype(np.float32).astype(np.float64), oracle.Folded(**nacl(z0=slab.z_top).as_dict()))
    assert force_err(F1[0], Fo) < F_RTOL
    R.remove_systems(sl)


def test_bad_surfaces_rejected(R):
    from surfmol_b200.relax import SmrError
    s = nacl()
    s.bx, s.by = s.ax, s.ay                                                 # b parallel to a
    with pytest.raises(SmrError):
        R.set_surface_folded(s)
    s = nacl()
    s.fmax = 0.0
    with pytest.raises(SmrError):
        R.set_surface_folded(s)
    with pytest.raises(ValueError):
        R.set_surface_folded(FoldedSurface(5, 0, 0, 5, [0.0], [0.0], [1.0, 2.0], [0.0]))    # z0 shorter than kz
