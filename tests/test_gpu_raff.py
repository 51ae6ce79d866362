"""Multi-replica RAFF on the GPU against the FP64 oracle (opencl/RRsp3.cl:1774-2048 restated):
one and many steps under every option of the step, replicas independent of the batch and of how
the steps are chunked, padding atoms, block teams for larger molecules, and the error paths."""
import numpy as np
import pytest

from surfmol_b200 import synth

pytestmark = pytest.mark.gpu


def replicas(prep, nsys, seed, amp=0.2):
    rng = np.random.default_rng(seed)
    P = np.repeat(prep.pos[None].astype(np.float64), nsys, 0)
    scale = np.where(prep.Z == 1, 1.5, 1.0)[None, :, None]
    return (P + amp * scale * rng.uniform(-1, 1, P.shape)).astype(np.float32)


def tree(seed, n=100):
    """A random bonded tree of degree <= 4 with its own geometry (1.0-1.5 A bonds)."""
    rng = np.random.default_rng(seed)
    Z = np.zeros(n, np.int32)
    P = np.zeros((n, 3))
    B, deg = [], np.zeros(n, int)
    for i in range(1, n):
        j = int(rng.choice([j for j in range(i) if deg[j] < 4]))
        B.append((j, i)); deg[i] += 1; deg[j] += 1
        v = rng.normal(size=3)
        P[i] = P[j] + rng.uniform(1.0, 1.5) * v / np.linalg.norm(v)
    for i in range(n):
        Z[i] = 6 if deg[i] > 1 else 1
    return Z, P, B


def setup(prep, nsys, seed, radius=None, fixmask=None):
    from surfmol_b200.raff import RaffMulti
    R = RaffMulti(prep.natoms, nsys)
    P = replicas(prep, nsys, seed)
    R.upload_prepared(prep, P, radius=radius, fixmask=fixmask)
    return R, P


def oracle_run(oracle, prep, P, nsteps, radius=None, fixmask=None, **cfg):
    n = prep.natoms
    pos4 = np.zeros((len(P), n, 4))
    pos4[..., :3] = P
    pos4[..., 3] = prep.inv_mass
    quat = np.zeros((len(P), n, 4)); quat[..., 3] = 1
    topo = dict(radius=np.zeros(n) if radius is None else radius, neighs=prep.neighs, excl1=prep.excl1, excl2=prep.excl2,
                fixmask=np.zeros(n, int) if fixmask is None else fixmask, port_local=prep.port_local[:prep.nnode],
                k=prep.k[:prep.nnode], bk=prep.bk_slots)
    return oracle.raff_step(pos4, quat, n, prep.nnode, nsteps, topo, **cfg)


CASES = {
    "default": dict(),
    "momentum": dict(cfg=dict(momentum_beta=0.4)),
    "collisions": dict(radius=1.3),
    "fixmask": dict(fix=True),
    "rot_mass": dict(cfg=dict(rot_mass_scale=2.5, dt=0.05, relaxation=0.8)),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("nsteps,tol", [(1, 2e-6), (200, 2e-4)])
def test_steps_match_oracle(oracle, case, nsteps, tol):
    from surfmol_b200.raff import prepare
    c = CASES[case]
    m = synth.pentitol()
    prep = prepare(m.Z, m.pos, m.bonds)
    radius = None if "radius" not in c else np.full(prep.natoms, c["radius"], np.float32)
    fix = None
    if c.get("fix"):
        fix = np.zeros(prep.natoms, np.int32); fix[0] = 7; fix[3] = 2; fix[prep.nnode] = 8; fix[prep.nnode + 1] = 5
    cfg = dict(c.get("cfg", {}))
    R, P = setup(prep, 64, 11, radius=radius, fixmask=fix)
    try:
        R.step_cluster_multi(nsteps, **cfg)
        ref_cfg = dict(dt=cfg.get("dt", 0.1), relaxation=cfg.get("relaxation", 0.5), beta=cfg.get("momentum_beta", 0.0),
                       rot_mass_scale=cfg.get("rot_mass_scale", 1.0))
        o = oracle_run(oracle, prep, P.astype(np.float64), nsteps, radius=radius, fixmask=fix, **ref_cfg)
        assert np.abs(R.download_pos_multi() - o["pos"][..., :3]).max() < tol
        assert np.abs(R.download_quat_multi() - o["quat"]).max() < tol
        scale = max(1.0, np.abs(o["dnode"]).max())
        got = np.stack([R.download_dpos_node_replica(k) for k in range(0, 64, 9)])
        assert np.abs(got - o["dnode"][::9]).max() < tol * scale
        if radius is not None:
            cg = np.stack([R.download_dpos_coll_replica(k) for k in range(0, 64, 9)])
            assert np.abs(o["coll"]).max() > 1e-3                       # collisions happened
            assert np.abs(cg - o["coll"][::9]).max() < tol
    finally:
        R.finish()


def test_replicas_independent_of_batch_and_chunks():
    from surfmol_b200.raff import prepare
    m = synth.pentitol()
    prep = prepare(m.Z, m.pos, m.bonds)
    R, P = setup(prep, 1000, 5)
    R.step_cluster_multi(100, momentum_beta=0.3)
    R.step_cluster_multi(150, momentum_beta=0.3)
    big = R.download_pos_multi()
    R.finish()
    from surfmol_b200.raff import RaffMulti
    for k in (0, 517, 999):
        one = RaffMulti(prep.natoms, 1)
        one.upload_prepared(prep, P[k:k + 1])
        one.step_cluster_multi(250, momentum_beta=0.3)
        assert np.array_equal(one.download_pos_replica(0), big[k]), k
        one.finish()


def test_padding_atoms_change_nothing():
    """Replicas padded to 32 atoms (inverse mass 0, NaN positions, as pack_molecules lays them out)
    give bit for bit the unpadded result."""
    from surfmol_b200.raff import RaffMulti, prepare
    m = synth.pentitol()
    prep = prepare(m.Z, m.pos, m.bonds)
    R, P = setup(prep, 16, 7)
    R.step_cluster_multi(120)
    ref = R.download_pos_multi()
    R.finish()
    n, npad = prep.natoms, 32
    pad = lambda a, fill: np.concatenate([a, np.full((npad - n,) + a.shape[1:], fill, a.dtype)])
    Rp = RaffMulti(npad, 16)
    Rp.upload_radius(np.zeros(npad))
    Rp.upload_neighs_and_exclusions(pad(prep.neighs, -1), pad(prep.excl1, -1), pad(prep.excl2, -1))
    Rp.upload_cluster_ports_multi(prep.port_local[:prep.nnode], prep.k[:prep.nnode], prep.nnode)
    Rp.upload_bk_slots_multi(pad(prep.bk_slots, -1))
    Pp = np.concatenate([P, np.zeros((16, npad - n, 3), np.float32)], 1)
    Rp.upload_state_multi(Pp, pad(prep.inv_mass, 0.0))
    Rp.step_cluster_multi(120)
    got = Rp.download_pos_multi()
    assert np.array_equal(got[:, :n], ref) and np.isnan(got[:, n:]).all()
    Rp.finish()


@pytest.mark.parametrize("natoms", [100, 300])
def test_block_teams_match_oracle(oracle, natoms):
    from surfmol_b200.raff import prepare
    Z, P0, B = tree(natoms, natoms)
    prep = prepare(Z, P0, B)
    R, P = setup(prep, 24, 3)
    try:
        R.step_cluster_multi(50, momentum_beta=0.2)
        o = oracle_run(oracle, prep, P.astype(np.float64), 50, beta=0.2)
        assert np.abs(R.download_pos_multi() - o["pos"][..., :3]).max() < 1e-4
    finally:
        R.finish()


def test_errors():
    from surfmol_b200.raff import RaffError, RaffMulti, prepare
    with pytest.raises(RaffError):
        RaffMulti(2000, 4)                                              # more atoms than a team holds
    m = synth.pentitol()
    prep = prepare(m.Z, m.pos, m.bonds)
    R = RaffMulti(prep.natoms, 4)
    with pytest.raises(RaffError, match="ports"):
        R.step_cluster_multi(1)                                         # ports not uploaded
    with pytest.raises(RaffError):
        R.upload_radius(np.full(prep.natoms, -1.0))
    bad = prep.neighs.copy(); bad[0, 0] = prep.natoms
    with pytest.raises(RaffError):
        R.upload_neighs_and_exclusions(bad, prep.excl1, prep.excl2)
    R.finish()
