"""Synthetic workload generator (CPU): the compact benzenoids of the ragged and served sets."""
import numpy as np

from surfmol_b200 import synth


def test_benzenoid_atom_count_formula():
    """benzenoid_atoms (n_C + n_H from the count of carbons shared by three rings) equals the ring
    graph built explicitly: its vertices plus one H per two-coordinated carbon."""
    rng = np.random.default_rng(0)
    for _ in range(60):
        A, B = int(rng.integers(1, 9)), int(rng.integers(1, 9))
        m = min(A, B) - 1
        c1 = int(rng.integers(0, m + 1))
        c2 = A + B - 2 - int(rng.integers(0, m + 1))
        hexes = synth.convex_hexes(A, B, c1, c2)
        xy, adj = synth._ring_graph(hexes)
        assert synth.benzenoid_atoms(hexes) == xy.shape[0] + int((adj.sum(1) == 2).sum()), (A, B, c1, c2)


def test_ragged_molecules_are_compact_and_clean():
    """Sizes near the target, every ring carbon 2- or 3-coordinated, no non-bonded contact below
    the construction margin, the largest flakes far shorter than a ribbon of the same size."""
    rng = np.random.default_rng(1)
    for target in (12, 20, 57, 133, 400, 1000):
        m = synth.ragged_molecule(rng, target)
        assert abs(m.n - target) <= max(6, 0.15 * target), (target, m.n)
        n = m.n
        bonded = np.zeros((n, n), bool)
        for i, j in m.bonds:
            bonded[i, j] = bonded[j, i] = True
        deg = bonded.sum(1)
        heavy = m.Z != synth.Z_H
        assert np.all(deg[m.Z == synth.Z_H] == 1) and np.all(deg[m.Z == synth.Z_O] == 1)
        assert np.all((deg[heavy & (m.Z != synth.Z_O)] >= 2) & (deg[heavy & (m.Z != synth.Z_O)] <= 3))
        d = np.linalg.norm(m.pos[:, None] - m.pos[None], axis=-1)
        np.fill_diagonal(d, 1e9)
        assert d[~bonded].min() >= synth.MIN_NONBONDED
        if target >= 400:
            # a one-row ribbon of this size would be ~2.46 A per 4 atoms long
            assert np.ptp(m.pos[:, :2], axis=0).max() < 0.4 * 2.46 * n / 4
