"""Langevin drive of the MD update (the TDrives input of updateAtomsMMFFf4, opencl/UFF.cl:982-991) on
the GPU: FIRE trajectories under the drive (alone and with constraint springs) follow the FP64
oracle; a fixed-seed drive relaxes to a loaded structure whose returned forces stay physical;
chunked, mixed and switched-off runs are bitwise; bad inputs are refused."""
import numpy as np
import pytest

from tests.gpu_helpers import build_device_grid, molecule_on_slab, small_slab_grid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    from surfmol_b200 import RelaxMulti
    slab, dims, p0, step = small_slab_grid()
    R = RelaxMulti(max_systems=64, max_atoms=20000)
    R.set_nb(1.0, 1.5)
    g = build_device_grid(R, slab, dims, p0, step)
    yield R, slab, g
    R.finish()


DRIVES = {
    "fixed_seed": (40.0, 0.05, 2.5, 0.0),             # T [K], gamma, seed, seed increment per step
    "stepping_seed": (40.0, 0.05, 0.37, 1.0),
    "hot_negative_seed": (300.0, 0.02, -7.3, 0.25),
}


@pytest.mark.parametrize("name", list(DRIVES))
@pytest.mark.parametrize("with_cons", [False, True])
def test_trajectory_matches_oracle(env, oracle, name, with_cons):
    """40 FIRE steps with the drive (and springs) from the same float32 start: positions within 2e-4 A of
    the FP64 oracle's trajectory."""
    R, slab, g = env
    T, gamma, seed, dseed = DRIVES[name]
    rng = np.random.default_rng(5 + len(name) + 7 * with_cons)
    Z, P, q = molecule_on_slab(rng, 40, slab)
    P32 = P.astype(np.float32).astype(np.float64)
    sl = R.add_systems([R.add_molecule(Z, P, q)], [P])
    cons = None
    if with_cons:
        atoms = np.array([1, 9, 30])
        target = P32[atoms] + [[0.3, 0.0, 0.2], [0.0, -0.25, 0.1], [-0.2, 0.2, 0.0]]
        k = np.array([[4.0, 4.0, 4.0], [0.0, 2.0, 6.0], [3.0, -1.0, 3.0]])
        R.set_constraints(sl[0], atoms, target, k)
        cons = (atoms, target, k)
    R.set_thermal_drive(sl, T, gamma, seed=seed, seed_step=dseed)
    R.run_fire(40, step_budget=40, fconv=1e-9)
    out = R.download(sl)
    assert out["steps"][0] == 40 and out["status"][0] == 2
    S = oracle.System.from_molecule(Z, P, q)
    ro = S.relax_drive(P32, oracle.Grid(g["coef"], g["p0"], g["step"]), max_steps=40, cons=cons,
                       tdrive=(T, gamma, dseed, seed), fconv=1e-9)
    assert ro["steps"] == 40
    moved = np.abs(ro["pos"] - P32).max()
    assert moved > 1e-2                                                 # the drive moved the atoms
    assert np.abs(R.download_pos64(sl)[0] - ro["pos"]).max() < 2e-4
    R.remove_systems(sl)


def test_fixed_seed_drive_relaxes_under_load(env, oracle):
    """With a fixed seed the noise is a constant per-atom load: FIRE converges, the returned forces are
    the physical ones at the result (oracle), and the load keeps them well away from zero."""
    R, slab, g = env
    rng = np.random.default_rng(8)
    Z, P, q = molecule_on_slab(rng, 40, slab)
    sl = R.add_systems([R.add_molecule(Z, P, q)], [P])
    R.set_thermal_drive(sl, 20.0, 0.05, seed=1.75)
    R.run_fire(6000, step_budget=6000, fconv=1e-3)
    out = R.download(sl)
    assert out["status"][0] == 1, out
    S = oracle.System.from_molecule(Z, P, q)
    Fo, _, _ = S.eval(R.download_pos64(sl)[0], oracle.Grid(g["coef"], g["p0"], g["step"]))
    assert np.abs(out["forces"][0][:, :3] - Fo).max() < 3e-3
    assert np.abs(Fo).max() > 2e-2
    R.remove_systems(sl)


def test_chunked_mixed_and_off_bitwise(env):
    """The seed of step s depends on s alone: a run in chunks equals one call; a driven system inside a
    mixed batch equals it alone; gamma = 0 gives the undriven trajectory bit for bit."""
    R, slab, _ = env
    rng = np.random.default_rng(4)
    mols = [molecule_on_slab(rng, n, slab) for n in (40, 25, 60)]
    tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
    Ps = [m[1] for m in mols]

    def run(idx, chunks, drive=True, budget=90):
        sl = R.add_systems([tids[i] for i in idx], [Ps[i] for i in idx])
        if drive:
            R.set_thermal_drive(sl[idx.index(0)], 30.0, 0.04, seed=0.9, seed_step=0.5)
        for c in chunks:
            R.run_fire(c, step_budget=budget, fconv=1e-9)
        out = R.download(sl)
        R.remove_systems(sl)
        return out

    one = run([0], [90])
    chunked = run([0], [25, 40, 25])
    mixed = run([1, 0, 2], [90])
    assert np.array_equal(one["pos"][0], chunked["pos"][0]) and chunked["steps"][0] == 90
    assert np.array_equal(one["pos"][0], mixed["pos"][1])
    plain = run([0], [90], drive=False)
    sl = R.add_systems([tids[0]], [Ps[0]])
    R.set_thermal_drive(sl, 30.0, 0.04, seed=0.9, seed_step=0.5)
    R.set_thermal_drive(sl, 30.0, 0.0)                                   # switched off again
    R.run_fire(90, step_budget=90, fconv=1e-9)
    off = R.download(sl)
    R.remove_systems(sl)
    assert np.array_equal(off["pos"][0], plain["pos"][0])
    assert not np.array_equal(one["pos"][0], plain["pos"][0])


def test_thermal_drive_errors(env):
    from surfmol_b200.relax import SmrError
    R, slab, _ = env
    rng = np.random.default_rng(6)
    Z, P, q = molecule_on_slab(rng, 40, slab)
    sl = R.add_systems([R.add_molecule(Z, P, q)], [P])
    with pytest.raises(SmrError):
        R.set_thermal_drive(sl, np.nan, 0.1)
    with pytest.raises(SmrError):
        R.set_thermal_drive(sl, -1.0, 0.1)
    R.remove_systems(sl)
    with pytest.raises(SmrError):
        R.set_thermal_drive(sl, 10.0, 0.1)                               # inactive slot
