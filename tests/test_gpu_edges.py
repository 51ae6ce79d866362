"""Edge cases through the C ABI on the GPU: empty calls, a lone atom, bond-free and disconnected
molecules, atoms outside the grid's z range, uncharged systems, mixed sizes in one launch, and the
error paths (bad slots, unknown topologies, capacity)."""
import numpy as np
import pytest

from surfmol_b200 import synth
from tests.gpu_helpers import F_RTOL, build_device_grid, force_err, molecule_on_slab, small_slab_grid

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    from surfmol_b200 import RelaxMulti
    slab, dims, p0, step = small_slab_grid()
    R = RelaxMulti(max_systems=64, max_atoms=20000)
    R.set_nb(1.0, 1.5)
    build_device_grid(R, slab, dims, p0, step)
    yield R, slab, R.get_grid()
    R.finish()


def oracle_forces(oracle, Z, P, q, g, **nb):
    S = oracle.System.from_molecule(Z, P, q)
    return S.eval(np.asarray(P, np.float32).astype(np.float64), oracle.Grid(g["coef"], g["p0"], g["step"]), **nb)


def test_empty_calls(env):
    R, _, _ = env
    assert R.run_fire(100, step_budget=100) == 0                   # no systems: nothing to do, no error
    F, E = R.eval_forces([])
    assert len(F) == 0 and E.shape == (0, 8)
    out = R.download([])
    assert len(out["steps"]) == 0
    R.remove_systems([])


def test_zero_steps_leave_state(env):
    R, slab, _ = env
    rng = np.random.default_rng(1)
    Z, P, q = molecule_on_slab(rng, 40, slab)
    s = R.add_systems([R.add_molecule(Z, P, q)], [P])
    R.run_fire(0, step_budget=100)
    out = R.download(s)
    assert out["steps"][0] == 0 and out["status"][0] == 0
    assert np.array_equal(out["pos"][0], P.astype(np.float32))
    R.remove_systems(s)


def test_lone_atom_and_bond_free(env, oracle):
    """A single atom (no bonds, no pairs) and two unbonded atoms: only NB and grid act."""
    R, slab, g = env
    c = np.array([0.5 * slab.Lx, 0.5 * slab.Ly, slab.z_top + 3.2])
    cases = [(np.array([6]), c[None, :], np.array([0.0])),
             (np.array([8, 6]), np.stack([c, c + [3.3, 0.0, 0.1]]), np.array([-0.2, 0.2]))]
    for Z, P, q in cases:
        tid = R.add_molecule(Z, P, q)
        s = R.add_systems([tid], [P])
        F, E = R.eval_forces(s)
        Fo, _, Eo = oracle_forces(oracle, Z, P, q, g)
        assert force_err(F[0], Fo) < F_RTOL
        assert abs(E[0, 0] - Eo[0]) < 1e-5 * max(1.0, abs(Eo[0]))
        R.run_fire(200, step_budget=200, fconv=1e-4)
        out = R.download(s)
        assert out["status"][0] in (1, 2) and np.all(np.isfinite(out["pos"][0]))
        R.remove_systems(s)


def test_disconnected_fragments(env, oracle):
    """Two molecules in one topology (no bond between them): NB acts across the fragments."""
    R, slab, g = env
    rng = np.random.default_rng(3)
    a = synth.ragged_molecule(rng, 24)
    b = synth.ragged_molecule(rng, 24)
    pa = synth.place(rng, a, (0.3 * slab.Lx, 0.3 * slab.Ly), 3.0, z_top=slab.z_top)
    pb = synth.place(rng, b, (0.3 * slab.Lx + 9.0, 0.3 * slab.Ly), 3.5, z_top=slab.z_top)
    Z = np.concatenate([a.Z, b.Z]); P = np.concatenate([pa, pb]); q = synth.charges(rng, len(Z))
    tid = R.add_molecule(Z, P, q)
    s = R.add_systems([tid], [P])
    F, _ = R.eval_forces(s)
    Fo, _, _ = oracle_forces(oracle, Z, P, q, g)
    assert force_err(F[0], Fo) < F_RTOL
    R.remove_systems(s)


def test_outside_grid_z_range(env, oracle):
    """Atoms below the grid's second plane or above its third-last get no substrate force (UFF.cl
    returns 0 there): the GPU agrees with the oracle on both sides."""
    R, slab, g = env
    rng = np.random.default_rng(4)
    m = synth.polyaromatic_40(rng)
    top = g["p0"][2] + g["step"][2] * (g["coef"].shape[2] - 1)
    for z in (g["p0"][2] + 0.05, top + 1.0):
        P = synth.place(rng, m, (2.0, 2.0), 0.0, jitter=0.0, z_top=0.0)
        P[:, 2] = z
        q = synth.charges(rng, m.n)
        s = R.add_systems([R.add_molecule(m.Z, P, q)], [P])
        F, E = R.eval_forces(s)
        Fo, _, Eo = oracle_forces(oracle, m.Z, P, q, g)
        assert force_err(F[0], Fo) < F_RTOL
        assert abs(E[0, 6]) < 1e-12 and abs(Eo[6]) < 1e-12          # no grid energy
        R.remove_systems(s)


def test_uncharged_and_mixed_sizes(env, oracle):
    """Q = 0 everywhere (pure LJ + grid Pauli/London) and systems of 5-600 atoms in one launch."""
    R, slab, g = env
    rng = np.random.default_rng(5)
    mols = [molecule_on_slab(rng, n, slab) for n in (12, 40, 130, 600)]
    mols = [(Z, P, np.zeros_like(q)) for Z, P, q in mols]
    tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
    s = R.add_systems(tids, [m[1] for m in mols])
    F, _ = R.eval_forces(s)
    for k, (Z, P, q) in enumerate(mols):
        Fo, _, _ = oracle_forces(oracle, Z, P, q, g)
        assert force_err(F[k], Fo) < F_RTOL, len(Z)
    R.remove_systems(s)


def test_error_paths(env):
    from surfmol_b200.relax import SmrError
    R, slab, _ = env
    rng = np.random.default_rng(6)
    Z, P, q = molecule_on_slab(rng, 40, slab)
    tid = R.add_molecule(Z, P, q)
    with pytest.raises(SmrError):
        R.add_systems([tid + 1000], [P])                            # unknown topology
    with pytest.raises(SmrError):
        R.remove_systems([63])                                       # inactive slot
    with pytest.raises(SmrError):
        R.download([5000])                                           # out of range
    with pytest.raises(SmrError):
        R.add_systems([tid] * 65, [P] * 65)                          # more slots than the capacity
    with pytest.raises(ValueError):
        R.add_systems([tid], [P[:10]])                               # positions of the wrong size
    with pytest.raises(SmrError):
        R.set_stages([5], [0], [0])                                  # first stage must start at 0
    with pytest.raises(SmrError):
        R.set_stages([0, 10], [0, 7], [0, 0])                        # unknown form
    with pytest.raises(SmrError):
        R.set_nb_lanes(3)                                            # not a power of two
    s = R.add_systems([tid], [P])                                    # the handle still works
    R.run_fire(10, step_budget=10)
    assert R.download(s)["steps"][0] == 10
    with pytest.raises(SmrError):
        R.remove_topology(tid)                                       # still used by a slot
    R.remove_systems(s)
    R.remove_topology(tid)
    with pytest.raises(SmrError):
        R.add_systems([tid], [P])                                    # released topology


def test_watchdog_timeout_and_recovery():
    """A call whose device work outlasts the watchdog returns SMR_ERR_TIMEOUT (-6) with the work still
    running; the next call waits for it and refreshes the per-system state, so the results equal
    those of a run without the timeout, bit for bit.  Only host waits are bounded here: the kernels
    have no device-side waits."""
    from surfmol_b200 import RelaxMulti
    from surfmol_b200.relax import SmrError
    slab, dims, p0, step = small_slab_grid()
    rng = np.random.default_rng(9)
    mols = [molecule_on_slab(rng, 40, slab) for _ in range(16)]
    outs = []
    for watchdog in (None, 1):
        R = RelaxMulti(max_systems=2048, max_atoms=2048 * 40)
        try:
            R.set_nb(1.0, 1.5)
            build_device_grid(R, slab, dims, p0, step)
            tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
            reps = [k % len(mols) for k in range(2048)]
            s = R.add_systems([tids[k] for k in reps], [mols[k][1] for k in reps])
            if watchdog:
                R.set_watchdog(watchdog)
                with pytest.raises(SmrError, match=r"\(-6\)"):
                    R.run_fire(1500, step_budget=1500, fconv=1e-4)
                R.set_watchdog(600000)
            else:
                R.run_fire(1500, step_budget=1500, fconv=1e-4)
            outs.append(R.download(s))
        finally:
            R.finish()
    a, b = outs
    assert np.array_equal(a["steps"], b["steps"]) and np.array_equal(a["status"], b["status"])
    assert all(np.array_equal(x, y) for x, y in zip(a["pos"], b["pos"]))


def test_topology_file_relaxes_like_pipeline(env, tmp_path):
    """A molecule loaded from a UFFTOPO file relaxes bit for bit like the same molecule added from
    elements and positions (same lists, types and parameters)."""
    from surfmol_b200.relax import Topology
    from surfmol_b200.topo_io import write_ufftopo
    R, slab, _ = env
    rng = np.random.default_rng(8)
    Z, P, q = molecule_on_slab(rng, 60, slab)
    ref = Topology(Z, P, q).export()
    write_ufftopo(tmp_path / "m.bin", ref["types"], P, ref["bonds"], ref["angs"], ref["dihs"], ref["invs"])
    t1 = R.add_molecule(Z, P, q)
    t2, P2 = R.add_topology_file(tmp_path / "m.bin", charges=q)
    s = R.add_systems([t1, t2], [P, P2])
    R.run_fire(200, step_budget=200, fconv=1e-6)
    out = R.download(s)
    assert np.array_equal(out["pos"][0], out["pos"][1]) and out["steps"][0] == out["steps"][1] == 200
    R.remove_systems(s)


@pytest.mark.parametrize("world", [1, 3, 4])
def test_sharded_grid_build_equals_single_build(world):
    """The sharded build's two halves (raw x-slabs, then the fit of the gathered whole) give the
    single-call grid bit for bit; the ranks' slabs are built one after another on this GPU into
    the buffer an all-gather would fill (3 ranks: slabs reach past nx, the extra planes dropped)."""
    import torch
    from surfmol_b200 import RelaxMulti
    from surfmol_b200.shard import build_grid_sharded, grid_slabs
    slab, dims, p0, step = small_slab_grid()
    nx, ny, nz = dims
    R = RelaxMulti(max_systems=4, max_atoms=400)
    try:
        ref = build_device_grid(R, slab, dims, p0, step)
        w, slabs = grid_slabs(nx, world)
        full = torch.empty(world * 3 * w * ny * nz, dtype=torch.float64, device="cuda")
        for k, (x0, _) in enumerate(slabs):
            part = full[k * 3 * w * ny * nz:(k + 1) * 3 * w * ny * nz]
            R.grid_raw_slab(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, nx, ny, nz, p0, step, x0, w, part.data_ptr(),
                            alpha_morse=1.5, npbc=1)
        torch.cuda.synchronize()
        R.grid_from_raw(full.data_ptr(), nx, ny, nz, p0, step)
        got = R.get_grid()
        assert np.array_equal(got["coef"], ref["coef"])
        build_grid_sharded(R, slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, nx, ny, nz, p0, step, alpha_morse=1.5, npbc=1)
        assert np.array_equal(R.get_grid()["coef"], ref["coef"])
    finally:
        R.finish()


def test_set_grid_from_device_memory():
    """smr_set_grid_device: a grid held by torch on the GPU goes in device to device and reads back
    unchanged; host memory is refused."""
    import torch
    from surfmol_b200 import RelaxMulti
    from surfmol_b200.relax import SmrError
    slab, dims, p0, step = small_slab_grid()
    R = RelaxMulti(max_systems=4, max_atoms=400)
    try:
        g = build_device_grid(R, slab, dims, p0, step)
        t = torch.from_numpy(g["coef"].copy()).cuda()
        R2 = RelaxMulti(max_systems=4, max_atoms=400)
        try:
            R2.set_grid_device(t.data_ptr(), dims, p0, step)
            assert np.array_equal(R2.get_grid()["coef"], g["coef"])
            with pytest.raises(SmrError, match="device memory"):
                R2.set_grid_device(g["coef"].ctypes.data, dims, p0, step)
        finally:
            R2.finish()
    finally:
        R.finish()
