"""CUDA path vs the oracle and vs the reference's own kernels for the NB variants and the force
limit (needs a GPU).

* 1-3 exclusion (smr_nb_params.excl13, getNonBond_GridFF_Bspline_ex2, opencl/UFF.cl:1722-1930):
  forces and energies vs the FP64 oracle's excl13 evaluation, <= 64 atoms (mask) and above
  (explicit 1-3 partners), with and without a cutoff, and relaxation to the oracle's minimum.
* NB + grid against the reference's kernels built for the host (oracle/_ref): a topology with
  zero bonded parameters isolates getNonBond_GridFF_Bspline (1-2) and its _ex2 form (1-2 + 1-3),
  compared FP32 to FP32.  Skipped where oracle/_ref was not built.
* Force limit (updateAtomsMMFFf4 Flimit, UFF.cl:946-948): trajectories over the first steps, where
  the clamp acts, and the clamped forces smr_download returns, vs the oracle's relax_fire.
"""
import numpy as np
import pytest

from tests.gpu_helpers import F_RTOL, small_slab_grid, build_device_grid, force_err, molecule_on_slab

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R():
    from surfmol_b200 import RelaxMulti
    r = RelaxMulti(max_systems=256, max_atoms=200000)
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
    R.set_grid(g["coef"], g["p0"], g["step"])
    yield slab, g
    R.set_nb()


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as Rf
    if not Rf.available(build_if_missing=False):
        pytest.skip("oracle/_ref (the reference's kernels built for the host) is not built")
    return Rf


@pytest.mark.parametrize("n,rcut", [(21, 0.0), (40, 0.0), (64, 0.0), (90, 0.0), (90, 6.0), (250, 10.0), (600, 0.0)])
def test_excl13_matches_oracle(R, oracle, slab_grid, n, rcut):
    slab, g = slab_grid
    R.set_nb(rcut=rcut, excl13=True)
    rng = np.random.default_rng(1300 + n)
    Z, P, q = molecule_on_slab(rng, n, slab)
    P32 = P.astype(np.float32).astype(np.float64)
    tid = R.add_molecule(Z, P, q)
    s = R.add_systems([tid], [P32])
    F, E = R.eval_forces(s)
    S = oracle.System.from_molecule(Z, P, q)
    grid = oracle.Grid(g["coef"], g["p0"], g["step"])
    Fo, Eao, Eco = S.eval(P32, grid, rcut=rcut, excl13=1)
    assert force_err(F[0], Fo) < F_RTOL
    assert np.abs(F[0][:, 3] - Eao).max() < 1e-5 * max(1.0, np.abs(Eao).max())
    assert abs(E[0, 0] - Eco[0]) < 1e-6 * max(1.0, abs(Eco[0]))
    # and it differs from the 1-2-only evaluation, so the test sees the exclusion
    F12, _, _ = S.eval(P32, grid, rcut=rcut, excl13=0)
    assert np.abs(F12 - Fo).max() > 100 * F_RTOL * max(1.0, np.abs(Fo).max())
    R.remove_systems(s)


def test_excl13_relaxes_to_oracle_minimum(R, oracle, slab_grid):
    slab, g = slab_grid
    R.set_nb(excl13=True)
    rng = np.random.default_rng(77)
    Z, P, q = molecule_on_slab(rng, 40, slab)
    tid = R.add_molecule(Z, P, q)
    s = R.add_systems([tid], [P])
    R.run_fire(3000, step_budget=3000, fconv=1e-3)
    out = R.download(s)
    assert out["status"][0] == 1
    S = oracle.System.from_molecule(Z, P, q)
    Pr = R.download_pos64(s)[0]
    Fo, _, _ = S.eval(Pr, oracle.Grid(g["coef"], g["p0"], g["step"]), excl13=1)
    assert np.sqrt((Fo ** 2).sum(1)).max() < 3e-3
    R.remove_systems(s)


def test_excl13_refused_with_pbc_images(R, slab_grid):
    """1-3 exclusion is defined for systems without PBC images: both entry points refuse the mix
    with an error and run the same systems again once it is off."""
    from surfmol_b200.relax import SmrError
    slab, g = slab_grid
    rng = np.random.default_rng(3)
    Z, P, q = molecule_on_slab(rng, 40, slab)
    tid = R.add_molecule(Z, P, q)
    s = R.add_systems([tid], [P])
    R.set_pbc(s, np.diag([40.0, 40.0, 0.0]), (1, 1, 0))
    R.set_nb(excl13=True)
    with pytest.raises(SmrError):
        R.eval_forces(s)
    with pytest.raises(SmrError):
        R.run_fire(10)
    R.set_nb()
    R.eval_forces(s)
    R.set_pbc(s, np.zeros((3, 3)), (0, 0, 0))
    R.remove_systems(s)


@pytest.mark.parametrize("excl13,n", [(False, 40), (False, 97), (True, 40), (True, 97)])
def test_nb_grid_matches_reference_kernel(R, oracle, ref, slab_grid, excl13, n):
    """NB + grid only (zero bonded parameters) vs getNonBond_GridFF_Bspline / _ex2 from the
    reference's own source, both FP32, on 3 placements of one molecule."""
    slab, g = slab_grid
    R.set_nb(excl13=excl13)
    rng = np.random.default_rng(900 + n + int(excl13))
    Z, P, q = molecule_on_slab(rng, n, slab)
    e = oracle.System.from_molecule(Z, P, q).export()
    tid = R.add_topology(e["req"], e["neighs"], np.zeros((len(Z), 8)))
    Ps = [P] + [P + np.array([rng.uniform(-3, 3), rng.uniform(-3, 3), rng.uniform(-0.6, 0.8)]) for _ in range(2)]
    Ps = [p.astype(np.float32).astype(np.float64) for p in Ps]      # both sides at the same FP32 positions
    s = R.add_systems([tid] * 3, Ps)
    F, _ = R.eval_forces(s)
    A = np.zeros((3, len(Z), 4), np.float32)
    A[:, :, :3] = np.array(Ps, np.float32)
    Rq = np.tile(e["req"].astype(np.float32), (3, 1, 1))
    if excl13:
        Fr = ref.nb_grid_ex2(A, Rq, np.tile(ref.second_neighs(e["neighs"]), (3, 1, 1)), g["coef"], g["p0"], g["step"])
    else:
        Fr = ref.nb_grid(A, Rq, np.tile(e["neighs"], (3, 1, 1)), g["coef"], g["p0"], g["step"])
    for k in range(3):
        assert np.abs(F[k][:, :3] - Fr[k, :, :3]).max() < F_RTOL * max(1.0, np.abs(Fr[k, :, :3]).max())
        assert np.abs(F[k][:, 3] - Fr[k, :, 3]).max() < 1e-5 * max(1.0, np.abs(Fr[k, :, 3]).max())
    R.remove_systems(s)


@pytest.mark.parametrize("flimit,steps", [(1.0, 1), (1.0, 8), (0.3, 25)])
def test_force_limit_follows_oracle(R, oracle, slab_grid, flimit, steps):
    """updateAtomsMMFFf4's |f| <= Flimit clamp (UFF.cl:946-948): a molecule started 2.1 A above
    the surface with 0.1 A of jitter has forces well above the limit; over the first steps the
    GPU trajectory follows the oracle's, and the forces smr_download returns are the clamped ones."""
    from surfmol_b200 import synth
    slab, g = slab_grid
    rng = np.random.default_rng(int(100 * flimit) + steps)
    m = synth.polyaromatic_40(rng)
    q = synth.charges(rng, m.n)
    P = synth.place(rng, m, (rng.uniform(0, slab.Lx), rng.uniform(0, slab.Ly)), 2.1, jitter=0.1, z_top=slab.z_top)
    grid = oracle.Grid(g["coef"], g["p0"], g["step"])
    S = oracle.System.from_molecule(m.Z, P, q)
    P32 = P.astype(np.float32).astype(np.float64)
    F0, _, _ = S.eval(P32, grid)
    assert np.sqrt((F0 ** 2).sum(1)).max() > 3 * flimit          # the clamp acts from the first step
    tid = R.add_molecule(m.Z, P, q)
    s = R.add_systems([tid], [P32])
    R.run_fire(steps, step_budget=steps, flimit=flimit, fconv=1e-6)
    out = R.download(s)
    o = S.relax(P32, grid, max_steps=steps, flimit=flimit, fconv=1e-6)
    Pg = R.download_pos64(s)[0]
    assert np.abs(Pg - o["pos"]).max() < 2e-4
    Fg = out["forces"][0][:, :3].astype(np.float64)
    assert np.sqrt((Fg ** 2).sum(1)).max() <= flimit * (1 + 1e-5)        # stored clamped
    assert np.sqrt((o["F"] ** 2).sum(1)).max() <= flimit * (1 + 1e-12)
    assert np.abs(Fg - o["F"]).max() < 1e-3 * flimit
    R.remove_systems(s)
