"""Continuous-batching server on the GPU: every served result is bitwise the result of the same request
relaxed alone, whatever else was resident; admission respects the HBM budget; topologies of retired
requests are released (and their device records compacted away) without disturbing resident ones."""
import numpy as np
import pytest

from tests.gpu_helpers import build_device_grid, molecule_on_slab, small_slab_grid

pytestmark = pytest.mark.gpu

FIRE = dict(dt0=0.001, dt_max=0.05, fconv=1e-3)
MAX_STEPS = 300


def make_handle(ms, ma, slab, dims, p0, step):
    from surfmol_b200 import RelaxMulti
    R = RelaxMulti(max_systems=ms, max_atoms=ma)
    R.set_nb(1.0, 1.5, 10.0)
    build_device_grid(R, slab, dims, p0, step)
    return R


@pytest.fixture(scope="module")
def reqs():
    from surfmol_b200.serve import Request
    slab, dims, p0, step = small_slab_grid()
    rng = np.random.default_rng(2024)
    sizes = np.exp(rng.uniform(np.log(20), np.log(260), 48)).astype(int)
    arrivals = np.sort(rng.uniform(0.0, 0.3, len(sizes)))
    out = []
    for i, (n, t) in enumerate(zip(sizes, arrivals)):
        Z, P, q = molecule_on_slab(rng, int(n), slab)
        out.append(Request(i, Z, P, q, float(t)))
    return (slab, dims, p0, step), out


def serve(geom, reqs, budget_atoms, chunk):
    from surfmol_b200.serve import Request, Server
    slab, dims, p0, step = geom
    R = make_handle(64, 40000, slab, dims, p0, step)
    try:
        mine = [Request(r.rid, r.Z, r.pos, r.q, r.arrival) for r in reqs]
        S = Server(R, 64, 40000, hbm_budget_bytes=budget_atoms * 1024, chunk_steps=chunk, max_steps=MAX_STEPS,
                   fire=FIRE, keep_pos64=True)
        st = S.run(mine)
        return mine, st
    finally:
        R.finish()


def test_served_results_equal_alone(reqs):
    geom, rs = reqs
    served, st = serve(geom, rs, budget_atoms=10 ** 6, chunk=40)
    assert st.n == len(rs) and all(r.t_done >= r.arrival and r.status in (1, 2) for r in served)
    assert st.max_resident > 1                                    # requests overlapped on the device
    slab, dims, p0, step = geom
    R = make_handle(4, 4000, slab, dims, p0, step)
    try:
        for k in (0, 7, 21, 40, len(rs) - 1):
            r = rs[k]
            s = R.add_systems([R.add_molecule(r.Z, r.pos, r.q)], [r.pos])
            R.run_fire(MAX_STEPS, step_budget=MAX_STEPS, **FIRE)
            alone = R.download(s)
            p64 = R.download_pos64(s)[0]
            assert np.array_equal(alone["pos"][0], served[k].out_pos), k
            assert np.array_equal(p64, served[k].out_pos64), k
            assert alone["steps"][0] == served[k].steps and alone["status"][0] == served[k].status
            assert alone["energy"][0] == served[k].energy
            R.remove_systems(s)
    finally:
        R.finish()


def test_budget_bounds_residency_and_keeps_results(reqs):
    """A budget of ~600 atoms keeps only a few systems resident; results stay bitwise the same."""
    geom, rs = reqs
    a, _ = serve(geom, rs, budget_atoms=10 ** 6, chunk=40)
    b, st = serve(geom, rs, budget_atoms=600, chunk=25)
    assert st.max_resident <= 600 // 20
    for x, y in zip(a, b):
        if len(x.Z) <= 600:
            assert np.array_equal(x.out_pos, y.out_pos) and x.steps == y.steps
        else:
            assert y.status == -1
