"""The FP64 oracle against the reference's own OpenCL kernels (CPU).

Two sources of reference outputs:
* tests/golden/ref_kernels.json, made by tests/golden/make_ref_fixtures.py from oracle/_ref
  (the reference's kernels built for the host); always available;
* oracle/_ref itself, where it is built (it needs the reference tree once), on larger seeded
  cases: many atoms, several systems, points across the periodic wraps and the z bounds.

The reference runs in FP32, the oracle in FP64, so the bar is FP32 rounding:
REF_RTOL relative to max(1, max|value|) for forces, energies and potentials.  The Ewald-2D
potential is a sum of ~1e5 G x ion terms whose phases the reference builds by repeated complex
multiplication in FP32; its FP32 error reaches ~1.2e-5 of max|phi|, so EWALD_RTOL applies there.
"""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REF_RTOL = 1e-5
EWALD_RTOL = 5e-5


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


@pytest.fixture(scope="module")
def fx():
    return json.load(open(os.path.join(GOLD, "ref_kernels.json")))


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref not built and no reference tree")
    return R


def _nb_system(oracle, d):
    """The oracle system of a fixture: bonds with zero stiffness, so only NB + grid act."""
    bonds = np.array(d["bonds"])
    n = len(d["req"])
    return oracle.System.from_bonds(n, bonds, np.zeros((len(bonds), 2)), np.array(d["req"]))


# ------------------------------------------------------------------ fixtures (no reference tree needed)
def test_fixture_ljqh(oracle, fx):
    d = fx["ljqh"]
    mixed = np.array(d["mixed"])
    ri, rj = np.array(d["reqi"]), np.array(d["reqj"])
    # mixREQ_arithmetic: R0 = Ri + Rj, E0 = Ei Ej (pre-square-rooted), Q = Qi Qj, H = min(Hi Hj, 0)
    want = np.c_[ri[:, 0] + rj[:, 0], ri[:, 1] * rj[:, 1], ri[:, 2] * rj[:, 2], np.minimum(ri[:, 3] * rj[:, 3], 0)]
    assert np.abs(mixed - want).max() < 1e-6
    out = oracle.ljqh_pairs(d["dp"], mixed, d["rdamp"])
    assert rel(d["out"], out) < REF_RTOL


def test_fixture_sampler(oracle, fx):
    d = fx["sample"]
    g = np.array(d["grid"], np.float32)
    out = oracle.sample_points(oracle.Grid(g, (0, 0, 0), (1, 1, 1)), d["u"], d["plqh"])
    ref = np.array(d["out"])
    assert rel(ref, out) < REF_RTOL
    # outside 1 <= iz < nz - 2 both return exactly zero
    assert np.array_equal(np.all(ref == 0, 1), np.all(out == 0, 1))
    assert np.all(ref == 0, 1).any() and not np.all(ref == 0, 1).all()


@pytest.mark.parametrize("case", ["nb_grid", "nb_ex2"])
def test_fixture_nb_grid(oracle, fx, case):
    d = fx["nb_grid"]
    S = _nb_system(oracle, d)
    grid = oracle.Grid(np.array(d["grid"], np.float32), d["p0"], d["step"])
    A = np.array(d["atoms"])
    ref = np.array(fx[case]["out"])
    if case == "nb_ex2":   # the fixture's exclusion lists are make_second_neighs of the topology
        from oracle.ref import second_neighs
        assert np.array_equal(np.array(fx[case]["excl"]), second_neighs(np.array(d["neighs"])))
    for s in range(len(A)):
        F, Ea, _ = S.eval(A[s, :, :3], grid, rdamp=d["rdamp"], alpha=d["alpha"], excl13=int(case == "nb_ex2"))
        assert rel(ref[s, :, :3], F) < REF_RTOL
        assert rel(ref[s, :, 3], Ea) < REF_RTOL


def test_fixture_morse(oracle, fx):
    d = fx["morse"]
    nx, ny, nz = d["ngrid"]
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    p0 = d["p0"]
    pts = np.c_[p0[0] + ix.ravel() * d["Lx"] / nx, p0[1] + iy.ravel() * d["Ly"] / ny, p0[2] + iz.ravel() * d["cz"] / nz]
    o = oracle.morse_points(pts, np.array(d["ions"]), np.array(d["req"]), d["Lx"], d["Ly"], npbc=d["npbc"], alpha=d["alpha"])
    assert np.abs(np.ravel(d["paul"]) - o[:, 0]).max() < REF_RTOL * np.abs(o[:, 0]).max()
    assert np.abs(np.ravel(d["lond"]) - o[:, 1]).max() < REF_RTOL * np.abs(o[:, 1]).max()


def test_fixture_bspline_conv(oracle, fx):
    d = fx["conv"]
    c = np.array(d["coef_xfast"])                     # (nz, ny, nx)
    out = oracle.bspline_conv(c.transpose(2, 1, 0))   # oracle layout (nx, ny, nz)
    assert np.abs(out.transpose(2, 1, 0) - np.array(d["out"])).max() < 1e-5


def test_fixture_ewald_and_image_sum(oracle, fx):
    d = fx["ewald"]
    pts, ions = np.array(d["pts"]), np.array(d["ions"])
    pe = oracle.ewald_points(pts, ions, d["Lx"], d["Ly"], gcut=d["gcut"])
    assert rel(d["phi"], pe) < EWALD_RTOL
    pb = oracle.brute_coulomb_points(pts, ions, d["Lx"], d["Ly"], nrep=fx["brute"]["nrep"])
    assert rel(fx["brute"]["phi"], pb) < REF_RTOL


# ------------------------------------------------------------------ live reference build
def test_live_ljqh_and_sampler(oracle, ref):
    rng = np.random.default_rng(7)
    n = 400
    ri = np.c_[rng.uniform(1.3, 2.1, n), np.sqrt(rng.uniform(1e-3, 1e-2, n)), rng.normal(0, .4, n), np.zeros(n)]
    rj = np.c_[rng.uniform(1.3, 2.1, n), np.sqrt(rng.uniform(1e-3, 1e-2, n)), rng.normal(0, .4, n), np.zeros(n)]
    mixed = ref.mix_req(ri, rj)
    dp = rng.normal(0, 4.0, (n, 3)).astype(np.float32)
    for rd in (0.5, 1.0):
        assert rel(ref.ljqh(dp, mixed, rd), oracle.ljqh_pairs(dp, mixed, rd)) < REF_RTOL
    nx, ny, nz = 13, 11, 17
    g = rng.normal(size=(nx, ny, nz, 4)).astype(np.float32)
    # lateral coordinates across both periodic wraps; z through both bounds (iz = 0, 1, nz-3, nz-2)
    u = np.c_[rng.uniform(-2 * nx, 2 * nx, 2000), rng.uniform(-ny, 2 * ny, 2000), rng.uniform(-1, nz + 1, 2000)]
    u = np.r_[u, [[0.0, 0.0, 1.0], [nx - 1e-3, ny - 1e-3, nz - 3 + 0.5], [-1e-3, -1e-3, nz - 2.0], [nx, ny, 0.999]]]
    u = u.astype(np.float32)
    plqh = rng.normal(size=(len(u), 4)).astype(np.float32)
    a = ref.sample(g, u, plqh)
    b = oracle.sample_points(oracle.Grid(g, (0, 0, 0), (1, 1, 1)), u, plqh)
    assert rel(a, b) < REF_RTOL
    assert np.array_equal(np.all(a == 0, 1), np.all(b == 0, 1))


@pytest.mark.parametrize("natoms", [22, 40, 97])
def test_live_nb_grid_kernels(oracle, ref, natoms):
    """getNonBond_GridFF_Bspline and its _ex2 form over 4 systems of one molecule, vs the oracle
    (1-2 exclusion; 1-2 + 1-3 exclusion) on a grid built from a NaCl slab."""
    from surfmol_b200 import synth
    rng = np.random.default_rng(natoms)
    slab = synth.rocksalt_slab(2, 2)
    dims, p0 = (24, 24, 40), (0.0, 0.0, slab.z_top + 1.0)
    step = (slab.Lx / 24, slab.Ly / 24, 0.2)
    coef = oracle.build_grid_fast(slab.ions, slab.req(), slab.Lx, slab.Ly, *dims, p0, step).astype(np.float32)
    grid = oracle.Grid(coef, p0, step)
    m = synth.polyaromatic_40(rng) if natoms == 40 else synth.ragged_molecule(rng, natoms)
    q = synth.charges(rng, m.n)
    P = [synth.place(rng, m, (rng.uniform(0, slab.Lx), rng.uniform(0, slab.Ly)), rng.uniform(1.8, 5.5)) for _ in range(4)]
    e = oracle.System.from_molecule(m.Z, P[0], q).export()
    S = oracle.System.from_bonds(m.n, e["bonds"], np.zeros((len(e["bonds"]), 2)), e["req"])
    A = np.zeros((4, m.n, 4), np.float32)
    A[:, :, :3] = np.array(P)
    Rq = np.tile(e["req"].astype(np.float32), (4, 1, 1))
    F12 = ref.nb_grid(A, Rq, np.tile(e["neighs"], (4, 1, 1)), coef, p0, step)
    F13 = ref.nb_grid_ex2(A, Rq, np.tile(ref.second_neighs(e["neighs"]), (4, 1, 1)), coef, p0, step)
    Fg = ref.nb_grid(A, Rq, np.tile(e["neighs"], (4, 1, 1)), coef, p0, step, nbff=False)
    for s in range(4):
        for F, ex in ((F12, 0), (F13, 1)):
            Fo, Ea, _ = S.eval(A[s, :, :3].astype(np.float64), grid, rdamp=1.0, alpha=1.5, excl13=ex)
            assert rel(F[s, :, :3], Fo) < REF_RTOL
            assert rel(F[s, :, 3], Ea) < REF_RTOL
        # the grid part alone (ns.w < 0 skips the atom-atom loop)
        Fo, Ea, _ = S.eval(A[s, :, :3].astype(np.float64), grid, rdamp=1.0, alpha=1.5, rcut=1e-6)
        assert rel(Fg[s, :, :3], Fo) < REF_RTOL


def test_live_grid_build_kernels(oracle, ref):
    """make_MorseFF, BsplineConv3D (and the oracle's exact fit through it), Ewald-2D, image sum."""
    from surfmol_b200 import synth
    rng = np.random.default_rng(11)
    slab = synth.rocksalt_slab(3, 3)
    nx, ny, nz = 24, 24, 10
    P, L = ref.morse(np.c_[slab.ions[:, :3], np.zeros(len(slab.ions))], slab.req(), np.diag([slab.Lx, slab.Ly, 3.0]),
                     (nx, ny, nz), (0.0, 0.0, 0.8), alpha=1.5)
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    pts = np.c_[ix.ravel() * slab.Lx / nx, iy.ravel() * slab.Ly / ny, 0.8 + iz.ravel() * 3.0 / nz]
    o = oracle.morse_points(pts, slab.ions, slab.req(), slab.Lx, slab.Ly, npbc=1, alpha=1.5)
    assert np.abs(P.ravel() - o[:, 0]).max() < REF_RTOL * np.abs(o[:, 0]).max()
    assert np.abs(L.ravel() - o[:, 1]).max() < REF_RTOL * np.abs(o[:, 1]).max()
    v = rng.normal(size=(9, 8, 12))
    c = oracle.bspline_fit(v)
    assert np.abs(ref.bspline_conv(c.transpose(2, 1, 0)).transpose(2, 1, 0) - v).max() < 1e-5
    pts = np.c_[rng.uniform(0, slab.Lx, 24), rng.uniform(0, slab.Ly, 24), rng.uniform(0.5, 7.0, 24)]
    for gcut in (3.0, 7.0):
        assert rel(ref.ewald_full(pts, slab.ions, slab.Lx, slab.Ly, gcut),
                   oracle.ewald_points(pts, slab.ions, slab.Lx, slab.Ly, gcut=gcut)) < EWALD_RTOL
    assert rel(ref.coulomb_brute(pts, slab.ions, slab.Lx, slab.Ly, 8),
               oracle.brute_coulomb_points(pts, slab.ions, slab.Lx, slab.Ly, nrep=8)) < REF_RTOL
