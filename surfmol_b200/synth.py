"""Seeded synthetic workloads: planar polyaromatic molecules over a rock-salt slab.

The reference measures nothing on a public dataset; these generators stand in
for its inputs with the shapes of the relaxation configurations:

* ``polyaromatic_40`` -- one 40-atom planar polyaromatic: a hexacene
  skeleton (26 ring sites at 1.40 A: 24 C + 2 pyridinic N on edge sites) with
  14 edge substituents (12 H at 1.09 A, 2 carbonyl O at 1.22 A).
* ``ragged_molecule`` -- compact convex hexagonal cores of a target size with
  H capping, ~5 % N (pyridinic, edge sites) and ~5 % O (carbonyl).
* ``rocksalt_slab`` -- (100) slab, a = 5.64 A, +-q ions, 4 ions per cell and
  layer, top layer at z = 0.

All geometry is float64 and fully determined by the integer seed.  Typing of
these molecules by the reference's hybridisation rule
(crates/libs/moltopo/src/assign_uff.rs:8-125) is clean: ring C -> C_R,
edge N (2 neighbours) -> N_R, carbonyl O (1 neighbour) -> O_2, H -> H_.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

Z_H, Z_C, Z_N, Z_O, Z_NA, Z_CL = 1, 6, 7, 8, 11, 17

B_CC = 1.40      # ring bond length (A)
B_CH = 1.09      # C-H (A)
B_CO = 1.22      # C=O (A)
BOND_CUT = 1.8   # bond-by-cutoff radius used by the reference topology builder
MIN_NONBONDED = 2.0    # geometric margin so the 1.8 A cutoff finds exactly the intended bonds
JITTER_CLIP = 0.05     # per-component clip of the Gaussian jitter: distances move by < 0.18 A

# (R_vdW, E_vdW) of the substrate ions, rows "Na" and "Cl" of the reference's
# data/AtomTypes.dat; Morse uses (R, sqrt(E)).
ION_RE = {Z_NA: (1.4915, 0.00130092313), Z_CL: (1.9735, 0.00984365166)}

_HEX_DIRS = [(1, 0), (1, -1), (0, -1), (-1, 0), (-1, 1), (0, 1)]


@dataclass
class Molecule:
    Z: np.ndarray          # (n,) int32 atomic numbers
    pos: np.ndarray        # (n,3) float64, molecule frame (centroid at origin, z=0)
    bonds: list = field(default_factory=list)   # construction bonds (i<j)

    @property
    def n(self) -> int:
        return int(self.Z.shape[0])


def _hex_vertices(hexes):
    """Vertices (rounded keys) of a set of axial hexagon centres, and the hex count per vertex."""
    verts = {}
    for (q, r) in hexes:
        cx = math.sqrt(3.0) * B_CC * (q + 0.5 * r)
        cy = 1.5 * B_CC * r
        for k in range(6):
            th = math.radians(30.0 + 60.0 * k)
            x, y = cx + B_CC * math.cos(th), cy + B_CC * math.sin(th)
            key = (round(x * 1000), round(y * 1000))
            if key not in verts:
                verts[key] = [x, y, 0]
            verts[key][2] += 1
    return verts


def _ring_graph(hexes):
    v = _hex_vertices(hexes)
    keys = sorted(v.keys())
    xy = np.array([[v[k][0], v[k][1]] for k in keys], dtype=np.float64)
    n = len(keys)
    d = np.linalg.norm(xy[:, None, :] - xy[None, :, :], axis=-1)
    adj = (d < B_CC * 1.05) & (d > 0.1)
    return xy, adj


def _assemble(rng, xy, adj, n_N, n_O):
    """Ring sites + substituents.  Returns Molecule or None if the geometry is crowded."""
    nring = xy.shape[0]
    deg = adj.sum(1)
    edge = [i for i in range(nring) if deg[i] == 2]
    if len(edge) < n_N + n_O + 1:
        return None
    perm = list(rng.permutation(edge))
    n_sites = []
    for i in perm:
        if len(n_sites) == n_N:
            break
        if not any(adj[i, j] for j in n_sites):
            n_sites.append(int(i))
    if len(n_sites) < n_N:
        return None
    rest = [int(i) for i in perm if i not in n_sites]
    o_sites = rest[:n_O]
    Z = [Z_N if i in n_sites else Z_C for i in range(nring)]
    P = [[xy[i, 0], xy[i, 1], 0.0] for i in range(nring)]
    bonds = [(i, j) for i in range(nring) for j in range(i + 1, nring) if adj[i, j]]
    for i in edge:
        if i in n_sites:
            continue
        nb = np.nonzero(adj[i])[0]
        d = (xy[i] - xy[nb[0]]) + (xy[i] - xy[nb[1]])
        d /= np.linalg.norm(d)
        if i in o_sites:
            z, b = Z_O, B_CO
        else:
            z, b = Z_H, B_CH
        bonds.append((i, len(Z)))
        Z.append(z)
        P.append([xy[i, 0] + b * d[0], xy[i, 1] + b * d[1], 0.0])
    P = np.array(P, dtype=np.float64)
    n = len(Z)
    bonded = np.zeros((n, n), dtype=bool)
    for i, j in bonds:
        bonded[i, j] = bonded[j, i] = True
    dd = np.linalg.norm(P[:, None, :] - P[None, :, :], axis=-1)
    np.fill_diagonal(dd, 1e9)
    if np.any(dd[~bonded] < MIN_NONBONDED):
        return None
    P -= P.mean(0)
    return Molecule(np.array(Z, dtype=np.int32), P, bonds)


def parallelogram_core(A: int, B: int):
    """Ring graph of an A x B parallelogram of hexagons (acenes for B=1).

    Parallelogram benzenoids have zigzag edges only: no bay or fjord regions,
    so with C-H = 1.09 A every non-bonded distance stays above 2.16 A and the
    1.8 A bond cutoff recovers exactly the construction bonds."""
    return _ring_graph([(q, r) for q in range(A) for r in range(B)])


def polyaromatic_40(rng) -> Molecule:
    """Hexacene skeleton (26 ring sites: 24 C + 2 pyridinic N), 12 H + 2 carbonyl O = 40 atoms."""
    xy, adj = parallelogram_core(6, 1)
    for _ in range(1000):
        m = _assemble(rng, xy, adj, n_N=2, n_O=2)
        if m is not None and m.n == 40:
            return m
    raise RuntimeError("could not generate the 40-atom polyaromatic")


def convex_hexes(A: int, B: int, c1: int, c2: int):
    """Axial hexagon centres of a convex benzenoid: the A x B parallelogram (0 <= q < A, 0 <= r < B)
    without the corners q + r < c1 and q + r > c2.  Its edges are zigzag only (no bay, cove or
    fjord regions), so with C-H = 1.09 A every non-bonded distance stays above 2.16 A."""
    return [(q, r) for q in range(A) for r in range(B) if c1 <= q + r <= c2]


def benzenoid_atoms(hexes) -> int:
    """C + H of the benzenoid hydrocarbon on these hexagons: n_C = 4h + 2 - n_i, n_H = 2h + 4 - n_i,
    n_i the carbons shared by three rings (one per triangle of mutually adjacent centres)."""
    s = set(hexes)
    ni = 0
    for (q, r) in s:
        ni += ((q + 1, r) in s and (q, r + 1) in s) + ((q - 1, r) in s and (q, r - 1) in s)
    return 6 * len(s) + 6 - 2 * ni


def _compact_shape(rng, target: int):
    """A random convex benzenoid of about ``target`` atoms (C + H): aspect ratio log-uniform in
    [1, 3], corner cuts uniform; its scale found by bisection on the atom count."""
    rho = math.exp(rng.uniform(0.0, math.log(3.0)))
    f1, f2 = rng.uniform(), rng.uniform()

    def shape(sc):
        A = max(1, int(round(sc * math.sqrt(rho))))
        B = max(1, int(round(sc / math.sqrt(rho))))
        m = min(A, B) - 1
        c1, c2 = int(round(f1 * m)), A + B - 2 - int(round(f2 * m))
        return A, B, c1, c2

    lo, hi = 0.5, 2.0
    while benzenoid_atoms(convex_hexes(*shape(hi))) < target:
        hi *= 2.0
    for _ in range(24):
        mid = 0.5 * (lo + hi)
        if benzenoid_atoms(convex_hexes(*shape(mid))) < target:
            lo = mid
        else:
            hi = mid
    a, b = shape(lo), shape(hi)
    na, nb = benzenoid_atoms(convex_hexes(*a)), benzenoid_atoms(convex_hexes(*b))
    return a if abs(na - target) <= abs(nb - target) else b


def ragged_molecule(rng, target: int) -> Molecule:
    """Compact hexagonal core with H capping near ``target`` atoms: a convex benzenoid (zigzag
    edges, aspect ratio 1-3, corners cut at random, from benzene and acenes up to coronene-like
    flakes), with ~5 % of the atoms pyridinic N on edge sites and ~5 % carbonyl O (together at
    most a third of the edge sites).  Large flakes are carbon-rich: the edge, which carries every
    H, N and O, grows like the square root of the size."""
    target = max(int(target), 12)
    for _ in range(1000):
        # the pyridinic N (about 3 % of the atoms) replace edge CH: aim the core that much higher
        hexes = convex_hexes(*_compact_shape(rng, round(target / 0.97)))
        xy, adj = _ring_graph(hexes)
        nedge = int((adj.sum(1) == 2).sum())
        tot = xy.shape[0] + nedge
        # N and O each ~5 % of the atoms, together at most a third of the edge sites
        n_sub = min(int(round(0.05 * tot)), nedge // 6)
        m = _assemble(rng, xy, adj, n_N=n_sub, n_O=n_sub)
        if m is not None:
            return m
    raise RuntimeError("could not generate a ragged molecule")


def _tetra_rest(a, b):
    """The two remaining unit directions of an ideal tetrahedron given two bond directions a, b."""
    m = -(a + b) / 2.0
    u = np.cross(a, b)
    u /= np.linalg.norm(u)
    return m + u * math.sqrt(2.0 / 3.0), m - u * math.sqrt(2.0 / 3.0)


def pentitol(cc: float = 1.53, co: float = 1.43, ch: float = 1.09, oh: float = 0.96):
    """A xylitol-like pentitol, HOCH2-(CHOH)3-CH2OH (C5H12O5, 22 atoms, 21 bonds, 10 nodes: the C
    and O atoms), on an ideal tetrahedral zigzag chain.  Returns a Molecule with its bonds."""
    dx, dy = cc * math.sin(math.radians(109.4712 / 2.0)), cc * math.cos(math.radians(109.4712 / 2.0))
    Cp = [np.array([k * dx, (k % 2) * dy, 0.0]) for k in range(5)]
    Z, P, bonds = [6] * 5, list(Cp), [(k, k + 1) for k in range(4)]

    def add(z, p, to):
        Z.append(z)
        P.append(p)
        bonds.append((to, len(Z) - 1))
        return len(Z) - 1

    for k in range(5):
        nb = [Cp[j] - Cp[k] for j in (k - 1, k + 1) if 0 <= j < 5]
        dirs = [v / np.linalg.norm(v) for v in nb]
        if len(dirs) == 1:                                   # chain end: continue the zigzag
            a = dirs[0]
            nxt = Cp[k] + (Cp[k] - (Cp[k - 1] if k else Cp[1])) * np.array([1.0, -1.0, 1.0])
            b = (nxt - Cp[k]) / np.linalg.norm(nxt - Cp[k])
            c, d = _tetra_rest(a, b)
            free = [b, c, d]
        else:
            free = list(_tetra_rest(dirs[0], dirs[1]))
        o_dir = free[0] if k % 2 == 0 else free[1]
        o = add(8, Cp[k] + co * o_dir, k)
        for f in free:
            if f is not o_dir:
                add(1, Cp[k] + ch * f, k)
        # hydroxyl H: 109.5 degrees from the O-C bond, in the plane of the O-C bond and z
        a = -o_dir
        p = np.cross(a, np.array([0.0, 0.0, 1.0]))
        if np.linalg.norm(p) < 1e-6:
            p = np.cross(a, np.array([1.0, 0.0, 0.0]))
        p /= np.linalg.norm(p)
        t = math.radians(109.4712)
        add(1, P[o] + oh * (math.cos(t) * a + math.sin(t) * p), o)
    pos = np.array(P)
    pos -= pos.mean(0)
    return Molecule(np.array(Z, np.int32), pos, bonds)


def polyacene_ribbon(ncell: int, cc: float = 1.40, ch: float = 1.08):
    """A periodic polyacene ribbon along x: ``ncell`` repeats of C4H2 (a rung of two carbons and
    the two apex CH of the next ring), period ``cc * sqrt(3)``.  Returns (Molecule, lattice (3, 3))
    with lattice a = (ncell * period, 0, 0) and b = c = 0 (non-periodic)."""
    per = cc * math.sqrt(3.0)
    Z, P = [], []
    for k in range(ncell):
        x0 = k * per
        Z += [6, 6, 6, 6, 1, 1]
        P += [(x0, 0.5 * cc, 0.0), (x0, -0.5 * cc, 0.0), (x0 + 0.5 * per, cc, 0.0), (x0 + 0.5 * per, -cc, 0.0),
              (x0 + 0.5 * per, cc + ch, 0.0), (x0 + 0.5 * per, -cc - ch, 0.0)]
    P = np.array(P)
    P -= P.mean(0)
    lat = np.zeros((3, 3))
    lat[0, 0] = ncell * per
    return Molecule(np.array(Z, np.int32), P), lat


def charges(rng, n: int, sigma: float = 0.15) -> np.ndarray:
    q = rng.normal(0.0, sigma, n)
    return q - q.mean()


def place(rng, mol: Molecule, xy0, height: float, jitter: float = 0.05, z_top: float = 0.0):
    """Rotate about z (uniform angle), translate to (x0, y0, z_top+height), add clipped Gaussian jitter."""
    th = rng.uniform(0.0, 2.0 * math.pi)
    c, s = math.cos(th), math.sin(th)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    p = mol.pos @ R.T
    p += np.array([xy0[0], xy0[1], z_top + height])
    if jitter > 0:
        p += np.clip(rng.normal(0.0, jitter, p.shape), -JITTER_CLIP, JITTER_CLIP)
    return p


@dataclass
class Slab:
    ions: np.ndarray       # (m,4) x, y, z, q
    Z: np.ndarray          # (m,) int32
    Lx: float
    Ly: float
    z_top: float

    def req(self) -> np.ndarray:
        """(m,4) Morse parameters per ion: (R, sqrt(E), q, 0)."""
        out = np.zeros((self.Z.shape[0], 4))
        for k, z in enumerate(self.Z):
            R, E = ION_RE[int(z)]
            out[k] = (R, math.sqrt(E), self.ions[k, 3], 0.0)
        return out


def rocksalt_slab(ncell: int, nlayers: int, a: float = 5.64, q: float = 0.9, z_top: float = 0.0) -> Slab:
    ions, Zs = [], []
    for L in range(nlayers):
        z = z_top - L * 0.5 * a
        for ix in range(ncell):
            for iy in range(ncell):
                for (fx, fy, cat) in ((0.0, 0.0, True), (0.5, 0.5, True), (0.5, 0.0, False), (0.0, 0.5, False)):
                    na = cat if (L % 2 == 0) else (not cat)
                    ions.append([(ix + fx) * a, (iy + fy) * a, z, q if na else -q])
                    Zs.append(Z_NA if na else Z_CL)
    return Slab(np.array(ions, dtype=np.float64), np.array(Zs, dtype=np.int32), ncell * a, ncell * a, z_top)


@dataclass
class GridSpec:
    nx: int
    ny: int
    nz: int
    p0: tuple
    step: tuple


def grid_for(slab: Slab, nz: int, dz: float = 0.1, z_gap: float = 1.0, h: float = 0.1) -> GridSpec:
    """Periodic x,y grid covering exactly one slab cell at ~h spacing; z from z_top+z_gap upward."""
    nx = int(round(slab.Lx / h))
    ny = int(round(slab.Ly / h))
    return GridSpec(nx, ny, nz, (0.0, 0.0, slab.z_top + z_gap), (slab.Lx / nx, slab.Ly / ny, dz))


@dataclass
class Workload:
    Z: list            # per system (n,) int32
    pos: list          # per system (n,3) float64
    q: list            # per system (n,) float64
    topo_of: np.ndarray  # per system: index of its molecule template (replicas share one)
    slab: Slab
    grid: GridSpec
    seed: int


def config0(seed: int = 0) -> Workload:
    """One 40-atom polyaromatic 3.0 A above a 2-layer 4x4-cell slab; grid 0.1 A, 12 A of z."""
    rng = np.random.default_rng(seed)
    mol = polyaromatic_40(rng)
    q = charges(rng, mol.n)
    slab = rocksalt_slab(4, 2)
    g = grid_for(slab, nz=121)
    p = place(rng, mol, (0.5 * slab.Lx, 0.5 * slab.Ly), 3.0)
    return Workload([mol.Z], [p], [q], np.zeros(1, np.int32), slab, g, seed)


def config1(seed: int = 0, nsys: int = 4096) -> Workload:
    """``nsys`` replicas of the config-0 molecule: random lateral offset, z rotation, height U[2.5,4]."""
    rng = np.random.default_rng(seed)
    mol = polyaromatic_40(rng)
    q = charges(rng, mol.n)
    slab = rocksalt_slab(4, 2)
    g = grid_for(slab, nz=121)
    Zs, Ps, Qs = [], [], []
    for _ in range(nsys):
        xy0 = (rng.uniform(0, slab.Lx), rng.uniform(0, slab.Ly))
        Ps.append(place(rng, mol, xy0, rng.uniform(2.5, 4.0)))
        Zs.append(mol.Z)
        Qs.append(q)
    return Workload(Zs, Ps, Qs, np.zeros(nsys, np.int32), slab, g, seed)


def _ragged_one(args):
    """Molecule i of a ragged workload, from its own generator (seed, i): any subset can be made alone."""
    seed, i, nmin, nmax, Lx, Ly, z_top = args
    rng = np.random.default_rng([seed, i])
    target = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
    mol = ragged_molecule(rng, target)
    q = charges(rng, mol.n)
    xy0 = (rng.uniform(0, Lx), rng.uniform(0, Ly))
    return mol.Z, place(rng, mol, xy0, rng.uniform(2.5, 4.0), z_top=z_top), q


def ragged(seed: int, nsys: int, nmin: int = 20, nmax: int = 400, ncell: int = 8, nlayers: int = 3,
           nz: int = 161, workers: int = 0) -> Workload:
    """Ragged batch: atom counts log-uniform in [nmin, nmax], each molecule distinct; molecule i is
    drawn from its own generator seeded (seed, i).  workers > 1 generates in a spawned process pool
    (call it before any CUDA work in the process)."""
    slab = rocksalt_slab(ncell, nlayers)
    g = grid_for(slab, nz=nz)
    jobs = [(seed, i, nmin, nmax, slab.Lx, slab.Ly, slab.z_top) for i in range(nsys)]
    if workers > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(workers) as pool:
            out = pool.map(_ragged_one, jobs, chunksize=max(1, nsys // (8 * workers)))
    else:
        out = [_ragged_one(j) for j in jobs]
    Zs = [o[0] for o in out]
    Ps = [o[1] for o in out]
    Qs = [o[2] for o in out]
    return Workload(Zs, Ps, Qs, np.arange(nsys, dtype=np.int32), slab, g, seed)


def config3_slab_grid():
    """3-layer 16x16-cell NaCl(100) slab and its 904 x 904 x 160 grid (~0.1 A, z over 16 A)."""
    slab = rocksalt_slab(16, 3)
    nx = ny = 904
    return slab, GridSpec(nx, ny, 160, (0.0, 0.0, slab.z_top + 1.0), (slab.Lx / nx, slab.Ly / ny, 0.1))


def _serve_one(args):
    seed, i, nmin, nmax, Lx, Ly, z_top = args
    r = np.random.default_rng([seed, i])
    target = int(round(math.exp(r.uniform(math.log(nmin), math.log(nmax)))))
    mol = ragged_molecule(r, target)
    q = charges(r, mol.n)
    return mol.Z, place(r, mol, (r.uniform(0, Lx), r.uniform(0, Ly)), r.uniform(2.5, 4.0), z_top=z_top), q


def serve_requests(seed: int, n: int, rate: float, slab: Slab, nmin: int = 20, nmax: int = 2000, workers: int = 0):
    """n requests with Poisson arrivals at `rate` per second: (Z, pos, q, arrival) of molecules with
    log-uniform atom counts in [nmin, nmax]; request i is drawn from its own generator (seed, i).
    workers > 1 generates in a spawned process pool (call it before any CUDA work)."""
    rng = np.random.default_rng([seed, 1 << 20])
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    jobs = [(seed, i, nmin, nmax, slab.Lx, slab.Ly, slab.z_top) for i in range(n)]
    if workers > 1 and n > 8:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(workers) as pool:
            mols = pool.map(_serve_one, jobs, chunksize=max(1, n // (8 * workers)))
    else:
        mols = [_serve_one(j) for j in jobs]
    return [(Z, P, q, float(t[i])) for i, (Z, P, q) in enumerate(mols)]
