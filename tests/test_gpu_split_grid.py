"""16-bit grid with FP32 near-surface planes (smr_convert_grid_split) against the plain FP32 and
16-bit grids and the FP64 oracle (needs a GPU).  An atom whose stencil starts below the split plane
reads the FP32 copy, every other atom the 16-bit grid, with the same arithmetic as the plain grids:
its force and per-atom energy must equal, bit for bit, those of the FP32 grid below the split and
those of the 16-bit grid above it, in the z-fastest layout and through the brick copy."""
import numpy as np
import pytest

from tests.gpu_helpers import F_RTOL, small_slab_grid, build_device_grid, molecule_on_slab

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def R():
    from surfmol_b200 import RelaxMulti
    r = RelaxMulti(max_systems=64, max_atoms=20000)
    yield r
    r.finish()


def _cells(P, p0, step):
    """stencil start plane iz - 1 of each atom, and whether it lies clear of a rounding decision"""
    u = (np.asarray(P, np.float64)[:, 2] - p0[2]) / step[2]
    iz = np.floor(u).astype(int)
    return iz - 1, np.abs(u - np.round(u)) > 1e-3


@pytest.mark.parametrize("dtype,bricks", [(1, 0), (1, 1), (2, 0), (2, 1)])
def test_split_grid_equals_fp32_below_and_16bit_above(R, dtype, bricks):
    slab, dims, p0, step = small_slab_grid(ncell=1, nlayers=2, nxy=20, nz=40, dz=0.25)
    rng = np.random.default_rng(70 + dtype)
    # heights spread over both sides of the split (planes 0-39 span z_gap .. z_gap + 9.75 A)
    mols = [molecule_on_slab(rng, n, slab, height=h) for n, h in ((40, 1.6), (90, 3.0), (60, 4.2), (21, 6.5), (40, 8.0))]
    tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
    slots = R.add_systems(tids, [m[1] for m in mols])
    R.set_grid_bricks(bricks)
    zsplit = 12
    F = {}
    for mode in ("f32", "f16", "split"):
        build_device_grid(R, slab, dims, p0, step, dtype=0)
        if mode == "f16":
            R.convert_grid(dtype)
        elif mode == "split":
            R.convert_grid_split(dtype, zsplit)
            assert R.get_grid_split()[0] == zsplit
            assert R.get_grid()["dtype"] == dtype
        R.set_positions(slots, [m[1] for m in mols])
        F[mode], _ = R.eval_forces(slots)
    assert R.grid_bricks_active() == bool(bricks)
    nlo = nhi = 0
    for k, (Z, P, q) in enumerate(mols):
        start, clear = _cells(P.astype(np.float32), p0, step)
        lo, hi = clear & (start < zsplit), clear & (start >= zsplit)
        nlo += lo.sum(); nhi += hi.sum()
        assert np.array_equal(F["split"][k][lo], F["f32"][k][lo])
        assert np.array_equal(F["split"][k][hi], F["f16"][k][hi])
    assert nlo > 50 and nhi > 50
    R.remove_systems(slots)
    R.set_grid_bricks(-1)


def test_split_grid_meets_fp32_accuracy_near_the_surface(R, oracle):
    """Molecules at the relaxed height: against the FP64 oracle on the FP64 grid the split grid's
    forces carry the FP32 grid's error, and the FP32 copy it returns is the FP32 grid's planes."""
    slab, dims, p0, step = small_slab_grid(ncell=1, nlayers=2, nxy=28, nz=48, dz=0.2)
    co = oracle.build_grid_fast(slab.ions, slab.req(), slab.Lx, slab.Ly, dims[0], dims[1], dims[2], p0, step,
                                alpha=1.5, npbc=1)
    rng = np.random.default_rng(77)
    mols = [molecule_on_slab(rng, 40, slab, height=h) for h in (2.8, 3.1, 3.4)]
    tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
    slots = R.add_systems(tids, [m[1] for m in mols])
    err = {}
    for mode in ("f32", "f16", "split"):
        g32 = build_device_grid(R, slab, dims, p0, step, dtype=0)
        if mode == "f16":
            R.convert_grid(1)
        elif mode == "split":
            R.convert_grid_split(1, 30)
            zs, lo = R.get_grid_split(planes=True)
            assert zs == 30 and np.array_equal(lo, g32["coef"][:, :, :33, :])
        R.set_positions(slots, [m[1] for m in mols])
        F, _ = R.eval_forces(slots)
        e = 0.0
        for k, (Z, P, q) in enumerate(mols):
            S = oracle.System.from_molecule(Z, P, q)
            Fo, _, _ = S.eval(P.astype(np.float32).astype(np.float64), oracle.Grid(co, p0, step))
            e = max(e, np.abs(np.asarray(F[k], float)[:, :3] - Fo).max())
        err[mode] = e
    assert err["split"] == err["f32"]
    assert err["split"] < F_RTOL
    assert err["f16"] > 3 * err["split"]
    # any later conversion drops the copy
    R.convert_grid(2)
    assert R.get_grid_split()[0] == 0
    R.remove_systems(slots)
    build_device_grid(R, slab, dims, p0, step, dtype=0)


def test_split_grid_rejects_bad_requests(R):
    from surfmol_b200.relax import SmrError
    slab, dims, p0, step = small_slab_grid(ncell=1, nlayers=2, nxy=16, nz=20, dz=0.25)
    build_device_grid(R, slab, dims, p0, step, dtype=0)
    for dt, zs in ((0, 5), (1, 0), (1, 18)):
        with pytest.raises(SmrError):
            R.convert_grid_split(dt, zs)
    R.convert_grid(1)
    with pytest.raises(SmrError):
        R.convert_grid_split(1, 5)                   # needs an FP32 grid
    build_device_grid(R, slab, dims, p0, step, dtype=0)


def test_graph_replay_follows_the_split(R):
    """With graph replay on, relaxing on the plain 16-bit grid and then on its split form gives the
    split form's own trajectory (the launch plan includes the FP32 copy, so the first plan's graph is
    not replayed), and repeating the split call replays it bit for bit."""
    slab, dims, p0, step = small_slab_grid(ncell=1, nlayers=2, nxy=20, nz=40, dz=0.25)
    rng = np.random.default_rng(91)
    mols = [molecule_on_slab(rng, n, slab, height=h) for n, h in ((40, 2.8), (60, 3.2))]
    tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
    slots = R.add_systems(tids, [m[1] for m in mols])
    out = {}
    try:
        for graph in (False, True):
            R.set_graph(graph)
            for mode in ("f16", "split", "split"):
                build_device_grid(R, slab, dims, p0, step, dtype=0)
                if mode == "f16":
                    R.convert_grid(1)
                else:
                    R.convert_grid_split(1, 20)
                R.set_positions(slots, [m[1] for m in mols])
                R.reset_fire(slots)
                R.run_fire(60, step_budget=60, fconv=1e-9)
                out.setdefault((graph, mode), []).append(R.download(slots)["pos"])
        ref = out[(False, "split")][0]
        for pos in out[(True, "split")] + out[(False, "split")][1:]:
            for k in range(len(mols)):
                assert np.array_equal(pos[k], ref[k])
        assert any(not np.array_equal(out[(True, "f16")][0][k], ref[k]) for k in range(len(mols)))
    finally:
        R.set_graph(False)
        R.remove_systems(slots)
