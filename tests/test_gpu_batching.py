"""Ragged batching on the GPU: batch admission, concurrent size classes, interaction tiling and the
autotuner, through the C ABI, against one-by-one admission and the FP64 oracle."""
import numpy as np
import pytest

from tests.gpu_helpers import F_RTOL, build_device_grid, force_err, molecule_on_slab, small_slab_grid

pytestmark = pytest.mark.gpu


def make_handle(ms, ma, slab, dims, p0, step, rcut=0.0):
    from surfmol_b200 import RelaxMulti
    R = RelaxMulti(max_systems=ms, max_atoms=ma)
    R.set_nb(1.0, 1.5, rcut)
    build_device_grid(R, slab, dims, p0, step)
    return R


@pytest.fixture(scope="module")
def setup():
    slab, dims, p0, step = small_slab_grid()
    rng = np.random.default_rng(314)
    mols = [molecule_on_slab(rng, n, slab) for n in (22, 40, 57, 90, 150, 210, 330)]
    return slab, dims, p0, step, mols


def test_batch_admission_matches_one_by_one(setup):
    """smr_add_molecules (parallel host typing and packing, one upload) gives the topologies and the
    trajectories of smr_add_molecule, bit for bit, with the size classes running concurrently."""
    slab, dims, p0, step, mols = setup
    tot = sum(len(m[0]) for m in mols)
    A = make_handle(16, tot, slab, dims, p0, step)
    B = make_handle(16, tot, slab, dims, p0, step)
    try:
        ta = [A.add_molecule(Z, P, q) for Z, P, q in mols]
        tb = list(B.add_molecules([m[0] for m in mols], [m[1] for m in mols], [m[2] for m in mols]))
        for a, b in zip(ta, tb):
            ea, eb = A.topology(a), B.topology(b)
            for k in ea:
                assert np.array_equal(np.asarray(ea[k]), np.asarray(eb[k])), k
        sa = A.add_systems(ta, [m[1] for m in mols])
        sb = B.add_systems(tb, [m[1] for m in mols])
        for R in (A, B):
            R.set_stages([0, 40], [0, 1], [0, 0])
            R.run_fire(120, step_budget=120, fconv=1e-6)
        oa, ob = A.download(sa), B.download(sb)
        for i in range(len(mols)):
            assert np.array_equal(oa["pos"][i], ob["pos"][i]) and oa["steps"][i] == ob["steps"][i] == 120
    finally:
        A.finish()
        B.finish()


@pytest.mark.parametrize("lanes", [1, 2, 8, 32])
def test_nb_lanes_forces_match_oracle(setup, oracle, lanes):
    """Every NB interaction tiling gives oracle forces (with and without the 10 A cutoff)."""
    slab, dims, p0, step, mols = setup
    from oracle import oracle as O
    for rcut in (0.0, 10.0):
        R = make_handle(4, 2000, slab, dims, p0, step, rcut)
        try:
            R.set_nb_lanes(lanes)
            assert R.get_nb_lanes() == lanes
            g = R.get_grid()
            for Z, P, q in (mols[1], mols[5]):
                s = R.add_systems([R.add_molecule(Z, P, q)], [P])
                F, _ = R.eval_forces(s)
                Fo, _, _ = O.System.from_molecule(Z, P, q).eval(P.astype(np.float32).astype(np.float64),
                                                                O.Grid(g["coef"], g["p0"], g["step"]), rcut=rcut)
                assert force_err(F[0], Fo) < F_RTOL, (lanes, rcut, len(Z))
                R.remove_systems(s)
        finally:
            R.finish()


def test_autotuner_runs_and_applies(setup):
    """The autotuner measures candidates on the device and its result applies to a handle; the tuned
    launch shape gives the same relaxation as any other up to rounding (same step counts within a few)."""
    slab, dims, p0, step, mols = setup
    from surfmol_b200.autotune import Autotuner
    fire = dict(dt0=0.001, dt_max=0.05, fconv=1e-3)
    mk = lambda ms, ma: make_handle(ms, ma, slab, dims, p0, step)
    res = Autotuner(mk, fire, probe_steps=30, max_steps=400).tune([m[0] for m in mols], [m[1] for m in mols],
                                                                  [m[2] for m in mols])
    assert res.nb_lanes in (0, 1, 2, 4, 8)
    assert res.timings["relax_ms_tuned"] <= res.timings["relax_ms_single_stage"] + 1e-9
    # the whole tuned shape is kept only when it beats the library's default shape (else: defaults)
    t, d = res.timings["relax_ms_tuned_shape"], res.timings["relax_ms_default_shape"]
    assert res.timings["relax_ms_single_stage"] == min(t, d)
    assert bool(res.team_by_class) == (t <= d)
    R = mk(16, 4000)
    try:
        res.apply(R)
        st = R.get_stages()
        assert tuple(st[0]) == tuple(res.stages[0]) and tuple(st[1]) == tuple(res.stages[1])
        tids = R.add_molecules([m[0] for m in mols], [m[1] for m in mols], [m[2] for m in mols])
        s = R.add_systems(tids, [m[1] for m in mols])
        R.run_fire(400, step_budget=400, **fire)
        out = R.download(s)
        assert np.all(np.isfinite(np.concatenate(out["pos"])))
    finally:
        R.finish()


def test_large_systems_global_state(setup, oracle):
    """Systems whose team state exceeds shared memory (1800 atoms: ~280 KB) keep it in global memory:
    forces match the oracle, and batched (mixed with a shared-memory system) and plain runs agree bit
    for bit."""
    from oracle import oracle as O
    from tests.gpu_helpers import molecule_on_slab
    slab, dims, p0, step, _ = setup
    rng = np.random.default_rng(1800)
    mols = [molecule_on_slab(rng, n, slab) for n in (1800, 1200)]
    assert len(mols[0][0]) > 1500
    R = make_handle(8, 8000, slab, dims, p0, step, rcut=10.0)
    try:
        g = R.get_grid()
        tids = [R.add_molecule(Z, P, q) for Z, P, q in mols]
        s = R.add_systems(tids, [m[1] for m in mols])
        F, _ = R.eval_forces(s)
        for i, (Z, P, q) in enumerate(mols):
            Fo, _, _ = O.System.from_molecule(Z, P, q).eval(P.astype(np.float32).astype(np.float64),
                                                            O.Grid(g["coef"], g["p0"], g["step"]), rcut=10.0)
            assert force_err(F[i], Fo) < F_RTOL, (len(Z), force_err(F[i], Fo))
        R.run_fire(30, step_budget=30, fconv=1e-6)
        mix = R.download(s)
        R.remove_systems(s)
        c = R.add_systems([tids[0]], [mols[0][1]])
        R.run_fire(30, step_budget=30, fconv=1e-6, mode=1)
        plain = R.download(c)
        assert np.array_equal(mix["pos"][0], plain["pos"][0]) and plain["steps"][0] == 30
    finally:
        R.finish()


def test_graph_replay_bitwise(setup):
    """With graph replay on, a repeated relaxation call replays the captured launch sequence and gives
    bit for bit the trajectories of directly issued launches (several stages, concurrent classes)."""
    slab, dims, p0, step, mols = setup
    R = make_handle(16, 4000, slab, dims, p0, step)
    try:
        tids = R.add_molecules([m[0] for m in mols], [m[1] for m in mols], [m[2] for m in mols])
        s = R.add_systems(tids, [m[1] for m in mols])
        R.set_stages([0, 30, 60], [0, 1, 1], [0, 64, 128])
        outs = []
        for graph in (False, True, True, True):
            R.set_graph(graph)
            R.set_positions(s, [m[1] for m in mols])
            R.reset_fire(s)
            R.run_fire(90, step_budget=90, fconv=1e-6)
            assert R.last_timing()[1] > 0
            outs.append(R.download(s))
        assert R.graph_replays() == 2
        for o in outs[1:]:
            for i in range(len(mols)):
                assert np.array_equal(o["pos"][i], outs[0]["pos"][i]) and o["steps"][i] == 90
    finally:
        R.finish()


@pytest.mark.parametrize("cap", [256, 32])
def test_nblist_forces_and_bitwise(setup, oracle, cap):
    """NB neighbour lists (systems >= 128 atoms under the 10 A cutoff): the forces of the first FIRE
    step match the oracle (cap 32 forces row overflow, i.e. the all-pairs fallback for crowded
    atoms), and batched, chunked and plain runs stay bitwise identical across list rebuilds."""
    from oracle import oracle as O
    slab, dims, p0, step, mols = setup
    big = [mols[4], mols[5], mols[6]]                       # 150-330 atoms
    R = make_handle(8, 4000, slab, dims, p0, step, rcut=10.0)
    try:
        R.set_nblist(min_atoms=128, skin=1.0, cap=cap)
        g = R.get_grid()
        tids = [R.add_molecule(Z, P, q) for Z, P, q in big]
        s = R.add_systems(tids, [m[1] for m in big])
        R.run_fire(1, step_budget=1, fconv=1e-9)
        out = R.download(s)
        for k, (Z, P, q) in enumerate(big):
            Fo, _, _ = O.System.from_molecule(Z, P, q).eval(P.astype(np.float32).astype(np.float64),
                                                            O.Grid(g["coef"], g["p0"], g["step"]), rcut=10.0)
            assert force_err(out["forces"][k], Fo) < F_RTOL, (len(Z), cap)
        R.remove_systems(s)
        runs = []
        for mode, chunks in ((0, [150]), (0, [40, 40, 70]), (1, [150])):
            s = R.add_systems(tids, [m[1] for m in big])
            for c in chunks:
                R.run_fire(c, step_budget=150, fconv=1e-6, mode=mode)
            runs.append(R.download(s))
            R.remove_systems(s)
        for o in runs[1:]:
            for k in range(len(big)):
                assert np.array_equal(o["pos"][k], runs[0]["pos"][k]) and o["steps"][k] == runs[0]["steps"][k] == 150
    finally:
        R.finish()


def test_nblist_complete_while_molecules_move(setup):
    """The lists stay complete between rebuilds: a list is rebuilt once an atom has moved more than
    half the skin, so no pair's separation changes by more than the skin before it is (atoms of
    these placements move up to ~3 A in 300 steps; one copy starts 2 A higher).  Every 60 FIRE
    steps the next step's forces
    (partner loop over the lists) equal an all-pairs evaluation at the same positions up to FP32
    summation order; a pair missing inside the 10 A cutoff would add its Coulomb force (~1e-3 eV/A)."""
    slab, dims, p0, step, mols = setup
    big = [mols[4], mols[5], mols[6]]                       # 150-330 atoms
    R = make_handle(8, 4000, slab, dims, p0, step, rcut=10.0)
    try:
        R.set_nblist(min_atoms=128, skin=1.0, cap=256)
        tids = [R.add_molecule(Z, P, q) for Z, P, q in big]
        starts = [m[1] for m in big] + [big[0][1] + np.array([0.0, 0.0, 2.0])]
        s = R.add_systems(tids + [tids[0]], starts)
        for _ in range(5):
            R.run_fire(60, fconv=1e-9)
            F_all, _ = R.eval_forces(s)                     # the evaluation entry point uses no lists
            R.run_fire(1, fconv=1e-9)                       # forces at the same positions, over the lists
            F_list = R.download(s, pos=False)["forces"]
            for k in range(len(s)):
                ref = F_all[k][:, :3].astype(np.float64)
                assert np.abs(F_list[k][:, :3] - ref).max() < 2e-5 * max(1.0, np.abs(ref).max()), k
    finally:
        R.finish()
