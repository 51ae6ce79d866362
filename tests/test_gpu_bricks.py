"""The brick copy of the substrate grid (SMR_TUNE_GRID_BRICKS) against the z-fastest grid
(needs a GPU).  The copy only changes where the kernel reads each voxel; the values and the
order of the sums are the same, so forces, energies and whole FIRE trajectories must agree
bit for bit, for float32, float16 and bfloat16 storage, on a grid whose stencils wrap the
periodic x / y bounds and reach the z bounds."""
import numpy as np
import pytest

from tests.gpu_helpers import small_slab_grid, build_device_grid, molecule_on_slab

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R():
    from surfmol_b200 import RelaxMulti
    r = RelaxMulti(max_systems=64, max_atoms=20000)
    yield r
    r.finish()


@pytest.mark.parametrize("dtype", [0, 1, 2])
def test_bricks_bitwise_equal_to_plain_grid(R, dtype):
    slab, dims, p0, step = small_slab_grid(ncell=1, nlayers=2, nxy=20, nz=30, dz=0.3)
    build_device_grid(R, slab, dims, p0, step, dtype=dtype)
    rng = np.random.default_rng(40 + dtype)
    mols = [molecule_on_slab(rng, n, slab, height=h) for n, h in ((40, 1.35), (90, 3.2), (21, 9.1), (150, 2.9))]
    tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
    slots = R.add_systems(tids, [m[1] for m in mols])
    out = {}
    for mode in (0, 1):
        R.set_grid_bricks(mode)
        R.set_positions(slots, [m[1] for m in mols])
        R.reset_fire(slots)
        F, E = R.eval_forces(slots)
        R.run_fire(300, step_budget=300, fconv=1e-4)
        d = R.download(slots)
        out[mode] = (F, E, d, R.download_pos64(slots))
    for k in range(len(slots)):
        assert np.array_equal(out[0][0][k], out[1][0][k])
        assert np.array_equal(out[0][3][k], out[1][3][k])
        assert np.array_equal(out[0][2]["forces"][k], out[1][2]["forces"][k])
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2]["steps"], out[1][2]["steps"])
    R.remove_systems(slots)
    R.set_grid_bricks(-1)
