"""CUDA path vs the FP64 oracle through the C ABI (needs a GPU)."""
import json
import os

import numpy as np
import pytest

from surfmol_b200 import synth
from tests.gpu_helpers import F_RTOL, small_slab_grid, build_device_grid, decode, force_err, molecule_on_slab

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
E_BOND, E_ANG, E_DIH, E_INV, E_NB, E_GRID = 1, 2, 3, 4, 5, 6


@pytest.fixture(scope="module")
def R():
    from surfmol_b200 import RelaxMulti
    r = RelaxMulti(max_systems=2048, max_atoms=400000)
    yield r
    r.finish()


@pytest.fixture(scope="module")
def grid_data(R):
    slab, dims, p0, step = small_slab_grid()
    g = build_device_grid(R, slab, dims, p0, step)
    return slab, g


@pytest.fixture
def slab_grid(R, grid_data):
    slab, g = grid_data
    R.set_grid(g["coef"], g["p0"], g["step"])      # other tests rebuild the device grid
    return slab, g


def test_h2_bond(R, oracle):
    """crates/libs/oclff/tests/test_uff_cl.rs:8-56 through smr_add_topology: fx=+-20, E=1 per atom."""
    g = json.load(open(os.path.join(GOLD, "h2.json")))
    R.set_nb(rcut=1e-6)
    kl = np.zeros((2, 8)); kl[0, :2] = (g["k"], g["l0"]); kl[1, :2] = (g["k"], g["l0"])
    tid = R.add_topology(np.zeros((2, 4)), [[1, -1, -1, -1], [0, -1, -1, -1]], kl)
    s = R.add_systems([tid], [np.array(g["pos"], float)])
    F, E = R.eval_forces(s)
    assert abs(F[0][0, 0] - 20.0) < g["tol"] and abs(F[0][1, 0] + 20.0) < g["tol"]
    assert abs(F[0][0, 3] - 1.0) < g["tol"] and abs(F[0][1, 3] - 1.0) < g["tol"]
    R.remove_systems(s)
    R.set_nb()


def test_pentacene_bonded(R, oracle):
    d = json.load(open(os.path.join(GOLD, "pentacene.json")))
    R.set_nb(rcut=1e-6)
    P = np.array(d["pos"])
    tid = R.add_molecule(d["Z"], P)
    P2 = P.copy(); P2[0, 2] = 0.5
    s = R.add_systems([tid, tid], [P, P2])
    F, E = R.eval_forces(s)
    assert abs(2 * E[0, E_BOND] - d["planar"]["E_bond"]) < 5e-4
    assert abs(E[0, E_ANG] - d["planar"]["E_angle"]) < 5e-4
    assert abs(2 * E[1, E_BOND] - d["displaced"]["E_bond"]) < 5e-4
    assert abs(E[1, E_INV] - d["displaced"]["E_inv"]) < 5e-4
    S = oracle.System.from_molecule(d["Z"], P)
    Fo, Eao, Eco = S.eval(P2, rcut=1e-6)
    assert force_err(F[1], Fo) < F_RTOL
    assert np.abs(E[1, 1:7] - Eco[1:7]).max() < 1e-5 * max(1.0, np.abs(Eco).max())
    R.remove_systems(s)
    R.set_nb()


@pytest.mark.parametrize("n,team,form", [(40, 32, 0), (40, 64, 0), (21, 32, 0), (90, 64, 0), (90, 128, 0), (250, 128, 0),
                                         (250, 256, 0), (600, 512, 0), (40, 128, 1), (40, 32, 1), (90, 256, 1), (250, 512, 1),
                                         (40, 32, 2), (21, 32, 2), (90, 32, 2), (90, 64, 2), (250, 128, 2), (600, 512, 2),
                                         (40, 256, 2)])
def test_forces_energies_match_oracle(R, oracle, slab_grid, n, team, form):
    """Rounds form (bonded terms in conflict-free rounds), gather form (pieces + per-atom sums) and
    owner form (terms evaluated by their owner atom, pieces gathered over bond back-slots)."""
    slab, g = slab_grid
    R.set_team_size(1 << 20, team)
    R.set_schedule(0, team, form)
    rng = np.random.default_rng(n * 31 + team)
    Z, P, q = molecule_on_slab(rng, n, slab)
    tid = R.add_molecule(Z, P, q)
    s = R.add_systems([tid], [P])
    F, E = R.eval_forces(s)
    P32 = P.astype(np.float32).astype(np.float64)
    grid = oracle.Grid(g["coef"], g["p0"], g["step"])
    S = oracle.System.from_molecule(Z, P, q)
    Fo, Eao, Eco = S.eval(P32, grid)
    err = force_err(F[0], Fo)
    assert err < F_RTOL, err
    assert np.abs(F[0][:, 3] - Eao).max() < 1e-5 * max(1.0, np.abs(Eao).max())
    # energy components: each bonded term's energy is FP32, a small sum of coefficients that are
    # large and nearly cancel near equilibrium (angle terms of sp2 carbon: ~2e-6 relative to the
    # component for a 90-atom benzenoid); the total energy's bar below is 1e-6 relative
    for c in range(1, 7):
        assert abs(E[0, c] - Eco[c]) < 5e-6 * max(1.0, abs(Eco[c])), (c, E[0, c], Eco[c])
    assert abs(E[0, 0] - Eco[0]) < 2e-6 * max(1.0, np.abs(Eco[1:7]).sum())
    assert abs(E[0, 0] - Eco[0]) < 1e-6 * abs(Eco[0])            # total energy within 1e-6 relative
    R.remove_systems(s)
    R.set_team_size(1 << 20, 0)
    R.set_schedule(0, 0, 0)


@pytest.mark.parametrize("ncell,nlayers,nxy,nz", [(1, 2, 16, 20), (2, 3, 24, 16)])
def test_grid_build_matches_oracle(R, oracle, ncell, nlayers, nxy, nz):
    slab, dims, p0, step = small_slab_grid(ncell=ncell, nlayers=nlayers, nxy=nxy, nz=nz, dz=0.25)
    g = build_device_grid(R, slab, dims, p0, step)
    co = oracle.build_grid_fast(slab.ions, slab.req(), slab.Lx, slab.Ly, dims[0], dims[1], dims[2], p0, step,
                                alpha=1.5, npbc=1)
    cg = g["coef"].astype(np.float64)
    for c in range(3):
        scale = np.abs(co[..., c]).max()
        assert scale > 0
        assert np.abs(cg[..., c] - co[..., c]).max() < 2e-6 * scale, c


@pytest.mark.parametrize("dtype", [1, 2])
def test_reduced_precision_grid_decodes_exactly(R, oracle, dtype):
    """fp16 / bf16 storage: the kernel's interpolation equals the oracle's on the decoded values."""
    from surfmol_b200 import GRID_F32
    slab, dims, p0, step = small_slab_grid()
    build_device_grid(R, slab, dims, p0, step, dtype=dtype)
    g = R.get_grid()
    assert g["dtype"] == dtype
    rng = np.random.default_rng(5)
    Z, P, q = molecule_on_slab(rng, 40, slab)
    tid = R.add_molecule(Z, P, q)
    s = R.add_systems([tid], [P])
    F, E = R.eval_forces(s)
    S = oracle.System.from_molecule(Z, P, q)
    Fo, _, _ = S.eval(P.astype(np.float32).astype(np.float64), oracle.Grid(decode(g), g["p0"], g["step"]))
    assert force_err(F[0], Fo) < F_RTOL
    R.remove_systems(s)
    build_device_grid(R, slab, dims, p0, step, dtype=GRID_F32)


def test_relaxed_structure_is_oracle_minimum(R, oracle, slab_grid):
    """FIRE on the GPU converges; the FP64 oracle finds max|F| at the result below fconv + 1e-4."""
    slab, g = slab_grid
    rng = np.random.default_rng(11)
    Z, P, q = molecule_on_slab(rng, 40, slab)
    tid = R.add_molecule(Z, P, q)
    s = R.add_systems([tid], [P])
    R.run_fire(2000, step_budget=2000, fconv=1e-3)
    out = R.download(s)
    assert out["status"][0] == 1, out
    S = oracle.System.from_molecule(Z, P, q)
    # at the float32 positions alone one ulp of a stiff bond moves |F| by ~1e-3 eV/A; at the
    # compensated positions the oracle sees the state FIRE converged
    Fo, _, Eco = S.eval(R.download_pos64(s)[0], oracle.Grid(g["coef"], g["p0"], g["step"]))
    # the convergence test uses the forces before the step's last move (relax_fire order,
    # crates/apps/molengine/src/main.rs:242-275), so the returned structure is one move further on
    assert np.sqrt((out["forces"][0][:, :3].astype(np.float64) ** 2).sum(1)).max() < 1e-3
    assert np.sqrt((Fo ** 2).sum(1)).max() < 3e-3
    ro = S.relax(P.astype(np.float32).astype(np.float64), oracle.Grid(g["coef"], g["p0"], g["step"]), max_steps=2000,
                 fconv=1e-3)
    assert ro["conv"]
    R.remove_systems(s)


def test_batched_plain_alone_mix_bitwise(R, oracle, slab_grid):
    """Same trajectories bit for bit: batched vs one-launch-per-step, alone vs in a ragged mix, chunked."""
    slab, g = slab_grid
    rng = np.random.default_rng(12)
    mols = [molecule_on_slab(rng, n, slab) for n in (40, 25, 130, 300)]
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


@pytest.mark.parametrize("starts,forms,teams", [([0, 60], [0, 1], [0, 128]), ([0, 1], [0, 1], [0, 256]),
                                                ([0, 60], [0, 1], [0, 32]), ([0, 30, 80], [0, 1, 1], [0, 64, 256]),
                                                ([0, 50, 90], [2, 0, 2], [0, 0, 64]), ([0, 70], [2, 1], [0, 128])])
def test_staged_schedule_bitwise(R, oracle, slab_grid, starts, forms, teams):
    """Stages of different forms and team sizes: batched, plain and chunked-alone runs agree bit for bit
    (chunk ends fall inside and on stage boundaries), and the relaxed structure is an oracle minimum."""
    slab, g = slab_grid
    if forms == [0, 1]:
        R.set_schedule(starts[1], teams[1], 0)
        assert R.get_schedule() == (starts[1], teams[1], 0)
    else:
        R.set_stages(starts, forms, teams)
    assert R.get_stages() == (starts, forms, teams)
    rng = np.random.default_rng(21 + starts[1])
    mols = [molecule_on_slab(rng, n, slab) for n in (40, 30, 120)]
    tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
    a = R.add_systems(tids, [m[1] for m in mols])
    R.run_fire(140, step_budget=140, fconv=1e-6)
    mix = R.download(a)
    R.remove_systems(a)
    b = R.add_systems([tids[0]], [mols[0][1]])
    for _ in range(4):
        R.run_fire(35, step_budget=140, fconv=1e-6)
    alone = R.download(b)
    R.remove_systems(b)
    c = R.add_systems([tids[0]], [mols[0][1]])
    R.run_fire(140, step_budget=140, fconv=1e-6, mode=1)
    plain = R.download(c)
    R.remove_systems(c)
    assert np.array_equal(mix["pos"][0], alone["pos"][0]) and np.array_equal(mix["pos"][0], plain["pos"][0])
    assert mix["steps"][0] == alone["steps"][0] == plain["steps"][0] == 140
    d = R.add_systems([tids[1]], [mols[1][1]])
    R.run_fire(3000, step_budget=3000, fconv=1e-3)
    out = R.download(d)
    assert out["status"][0] in (1, 2)
    S = oracle.System.from_molecule(*mols[1])
    P64 = R.download_pos64(d)[0]                           # the compensated positions FIRE converged
    assert np.abs(P64 - out["pos"][0]).max() < 1e-5
    Fo, _, _ = S.eval(P64, oracle.Grid(g["coef"], g["p0"], g["step"]))
    Fe, _ = R.eval_forces(d)                               # forces at the final positions
    assert force_err(Fe[0], Fo) < F_RTOL
    if out["status"][0] == 1:
        # relax_fire tests the forces of the step and then still moves the atoms
        # (crates/apps/molengine/src/main.rs:242-275): the reported forces are below fconv, the
        # returned structure is one FIRE move further on
        assert np.sqrt((out["forces"][0][:, :3].astype(np.float64) ** 2).sum(1)).max() < 1e-3
        assert np.sqrt((Fo ** 2).sum(1)).max() < 3e-3
    R.remove_systems(d)
    R.set_schedule(0, 0, 0)


def test_nonfinite_system_is_isolated(R, oracle, slab_grid):
    slab, g = slab_grid
    rng = np.random.default_rng(13)
    mols = [molecule_on_slab(rng, 40, slab) for _ in range(3)]
    tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
    bad = mols[1][1].copy(); bad[3, 0] = np.nan
    s = R.add_systems(tids, [mols[0][1], bad, mols[2][1]])
    R.run_fire(100, step_budget=100, fconv=1e-6)
    out = R.download(s)
    assert out["status"][1] == 3
    ref = R.add_systems([tids[0], tids[2]], [mols[0][1], mols[2][1]])
    R.run_fire(100, step_budget=100, fconv=1e-6)
    out2 = R.download(ref)
    assert np.array_equal(out["pos"][0], out2["pos"][0]) and np.array_equal(out["pos"][2], out2["pos"][1])
    R.remove_systems(s)
    R.remove_systems(ref)


def test_full_config_grid_matches_oracle(R, oracle):
    """The 226x226x121 grid of the benchmark workload (2-layer 4x4-cell slab) against the FP64 builder."""
    slab = synth.rocksalt_slab(4, 2)
    g = synth.grid_for(slab, nz=121)
    R.build_grid(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step)
    cg = R.get_grid()["coef"].astype(np.float64)
    co = oracle.build_grid_fast(slab.ions, slab.req(), slab.Lx, slab.Ly, g.nx, g.ny, g.nz, g.p0, g.step)
    # Morse node values are sums of FP32 terms (as make_MorseFF computes them) and the exact
    # B-spline fit amplifies node errors by up to 3 per axis: 1e-5 for P, L; FP64 Ewald: 2e-6
    for c, tol in zip(range(3), (1e-5, 1e-5, 2e-6)):
        scale = np.abs(co[..., c]).max()
        assert scale > 0
        assert np.abs(cg[..., c] - co[..., c]).max() < tol * scale, c
