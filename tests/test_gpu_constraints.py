"""Position constraints (the constr / constrK springs of updateAtomsMMFFf4, opencl/UFF.cl:974-982)
on the GPU: a constrained relaxation ends where the physical force (FP64 oracle) and the springs
balance; constraints leave the returned forces physical; mixes and removal are bitwise."""
import numpy as np
import pytest

from surfmol_b200 import synth
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


def springs(P, atoms, target, k):
    F = np.zeros_like(P)
    F[atoms] = (target - P[atoms]) * np.maximum(k, 0.0)
    return F


@pytest.mark.parametrize("kvec", [(5.0, 5.0, 5.0), (0.0, 0.0, 8.0), (2.0, -1.0, 3.0)])
def test_constrained_minimum(env, oracle, kvec):
    R, slab, g = env
    rng = np.random.default_rng(int(10 * sum(abs(x) for x in kvec)))
    Z, P, q = molecule_on_slab(rng, 40, slab)
    atoms = np.array([0, 7, 19])
    target = P[atoms] + [[0.5, 0.0, 0.3], [-0.2, 0.4, 0.0], [0.0, -0.3, 0.6]]
    k = np.tile(kvec, (3, 1))
    sl = R.add_systems([R.add_molecule(Z, P, q)], [P])
    R.set_constraints(sl[0], atoms, target, k)
    R.run_fire(4000, step_budget=4000, fconv=1e-3)
    out = R.download(sl)
    assert out["status"][0] == 1, out
    P64 = R.download_pos64(sl)[0]
    S = oracle.System.from_molecule(Z, P, q)
    Fo, _, _ = S.eval(P64, oracle.Grid(g["coef"], g["p0"], g["step"]))
    Ft = Fo + springs(P64, atoms, target, k)
    assert np.sqrt((Ft ** 2).sum(1)).max() < 3e-3
    # returned forces are the physical ones (the springs are not stored with them)
    Fs = springs(P64, atoms, target, k)
    assert np.abs(out["forces"][0][:, :3] - Fo).max() < 3e-3
    assert np.abs(Fs).max() > 1e-2                                     # the springs hold a real load
    R.remove_systems(sl)


def test_mix_alone_and_removal_bitwise(env):
    R, slab, _ = env
    rng = np.random.default_rng(3)
    mols = [molecule_on_slab(rng, n, slab) for n in (40, 25, 60)]
    tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
    Ps = [m[1] for m in mols]
    tgt = Ps[1][[2, 5]] + 0.3

    def run(ids, cons):
        sl = R.add_systems([tids[i] for i in ids], [Ps[i] for i in ids])
        for j, i in enumerate(ids):
            if cons and i == 1:
                R.set_constraints(sl[j], [2, 5], tgt, 4.0)
        R.run_fire(600, step_budget=600, fconv=1e-6)
        out = R.download(sl)
        R.remove_systems(sl)
        return out

    mix = run([0, 1, 2], True)
    alone = run([1], True)
    free0 = run([0], False)
    assert np.array_equal(mix["pos"][1], alone["pos"][0])
    assert np.array_equal(mix["pos"][0], free0["pos"][0])
    # set, then removed before running: the unconstrained trajectory
    sl = R.add_systems([tids[1]], [Ps[1]])
    R.set_constraints(sl[0], [2, 5], tgt, 4.0)
    R.set_constraints(sl[0], [])
    R.run_fire(600, step_budget=600, fconv=1e-6)
    removed = R.download(sl)
    R.remove_systems(sl)
    free1 = run([1], False)
    assert np.array_equal(removed["pos"][0], free1["pos"][0])
    assert not np.array_equal(alone["pos"][0], free1["pos"][0])


def test_constraint_errors(env):
    from surfmol_b200.relax import SmrError
    R, slab, _ = env
    Z, P, q = molecule_on_slab(np.random.default_rng(4), 40, slab)
    sl = R.add_systems([R.add_molecule(Z, P, q)], [P])
    with pytest.raises(SmrError):
        R.set_constraints(sl[0], [40], [[0, 0, 0]], 1.0)                # atom outside the system
    with pytest.raises(SmrError):
        R.set_constraints(sl[0], [1], [[np.nan, 0, 0]], 1.0)
    R.remove_systems(sl)
    with pytest.raises(SmrError):
        R.set_constraints(sl[0], [1], [[0, 0, 0]], 1.0)                 # inactive slot
