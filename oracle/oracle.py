"""ctypes binding of the FP64 parity oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker.  The product library never uses it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)


class OrcFolded(C.Structure):
    _fields_ = [("inv", C.c_double * 4), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("kx", DP), ("ky", DP), ("kz", DP), ("z0", DP), ("cq", DP), ("cp", DP), ("cl", DP),
                ("alpha", C.c_double), ("fmax", C.c_double)]


class OrcGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("p0", C.c_double * 3), ("step", C.c_double * 3),
                ("cf32", C.POINTER(C.c_float)), ("cf64", DP), ("scale", C.c_double * 4),
                ("folded", C.POINTER(OrcFolded))]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_sys_from_molecule.restype = C.c_void_p
        L.orc_sys_from_molecule.argtypes = [C.c_int, IP, DP, DP, C.c_double]
        L.orc_sys_from_molecule_pbc.restype = C.c_void_p
        L.orc_sys_from_molecule_pbc.argtypes = [C.c_int, IP, DP, DP, C.c_double, DP, C.c_char_p, C.c_int]
        L.orc_sys_cells.argtypes = [C.c_void_p, IP]
        L.orc_sys_from_bonds.restype = C.c_void_p
        L.orc_sys_from_bonds.argtypes = [C.c_int, C.c_int, IP, DP, DP]
        L.orc_sys_free.argtypes = [C.c_void_p]
        L.orc_sys_counts.argtypes = [C.c_void_p, IP]
        L.orc_sys_export.argtypes = [C.c_void_p] + [IP, IP, IP, DP, IP, IP, DP, IP, IP, DP, IP, IP, DP, DP, IP]
        L.orc_sys_set_params.argtypes = [C.c_void_p, DP, DP, DP]
        L.orc_type_name.restype = C.c_char_p
        L.orc_type_name.argtypes = [C.c_int]
        L.orc_eval.argtypes = [C.c_void_p, DP, C.POINTER(OrcGrid), DP, DP, DP, DP]
        L.orc_folded_points.argtypes = [C.POINTER(OrcFolded), C.c_int, DP, DP, DP, DP]
        L.orc_relax.restype = C.c_int
        L.orc_relax.argtypes = [C.c_void_p, DP, C.POINTER(OrcGrid), DP, DP, C.c_int, DP, DP, DP, DP, IP]
        L.orc_relax_drive.restype = C.c_int
        L.orc_relax_drive.argtypes = [C.c_void_p, DP, C.POINTER(OrcGrid), DP, DP, C.c_int, DP, DP, DP, DP, DP, DP, IP]
        L.orc_langevin_noise.argtypes = [C.c_int, C.c_float, DP]
        L.orc_relax_batch.argtypes = [C.c_int, C.POINTER(C.c_void_p), C.POINTER(DP), C.POINTER(OrcGrid), DP, DP,
                                      C.c_int, IP, DP, IP, DP, C.c_int]
        L.orc_max_threads.restype = C.c_int
        L.orc_morse_points.argtypes = [C.c_int, DP, C.c_int, DP, DP, DP, C.c_int, C.c_int, C.c_double, DP]
        L.orc_ewald_points.argtypes = [C.c_int, DP, C.c_int, DP, C.c_double, C.c_double, C.c_double, DP]
        L.orc_brute_coulomb_points.argtypes = [C.c_int, DP, C.c_int, DP, C.c_double, C.c_double, C.c_int, DP]
        L.orc_bspline_fit.argtypes = [C.c_int, C.c_int, C.c_int, DP, DP]
        L.orc_bspline_conv.argtypes = [C.c_int, C.c_int, C.c_int, DP, DP]
        L.orc_build_grid.restype = C.c_int
        L.orc_build_grid.argtypes = [C.c_int, DP, DP, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, DP, DP,
                                     C.c_double, C.c_int, C.c_double, DP, DP]
        L.orc_build_grid_fast.restype = C.c_int
        L.orc_build_grid_fast.argtypes = [C.c_int, DP, DP, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, DP, DP,
                                          C.c_double, C.c_int, C.c_double, DP, C.c_double]
        L.orc_substrate_direct.argtypes = [C.c_int, DP, DP, C.c_int, DP, DP, C.c_double, C.c_double, C.c_int,
                                           C.c_double, C.c_double, C.c_double, DP]
        L.orc_ljqh_pairs.argtypes = [C.c_int, DP, DP, C.c_double, DP]
        L.orc_sample_points.argtypes = [C.POINTER(OrcGrid), C.c_int, DP, DP, DP]
        _lib = L
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _dp(a):
    return a.ctypes.data_as(DP) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(IP) if a is not None else None


# Defaults: FireState (crates/libs/molff/src/raff.rs:1053-1055) with dt_max 0.05 as
# the pentacene relaxation uses (crates/libs/surfmol/tests/relax_pentacene_uff.rs:259).
FIRE_DEFAULT = dict(dt0=0.001, dt_max=0.05, alpha0=0.1, f_inc=1.1, f_dec=0.5, f_alpha=0.99, n_min=5,
                    fconv=1e-3, flimit=0.0)
NB_DEFAULT = dict(rdamp=1.0, alpha=1.5, rcut=0.0, excl13=0, lvec=None, npbc=(0, 0, 0))


def fire_vec(**kw):
    p = dict(FIRE_DEFAULT)
    p.update(kw)
    return _d([p["dt0"], p["dt_max"], p["alpha0"], p["f_inc"], p["f_dec"], p["f_alpha"], p["n_min"], p["fconv"],
               p["flimit"]])


def nb_vec(**kw):
    p = dict(NB_DEFAULT)
    p.update(kw)
    lv = np.zeros(9) if p["lvec"] is None else _d(p["lvec"]).reshape(9)
    return _d([p["rdamp"], p["alpha"], p["rcut"], p["excl13"], *lv, *p["npbc"]])


class Grid:
    """Oracle view of a z-fastest float4 coefficient grid (float32 or float64 array (nx,ny,nz,4))."""

    def __init__(self, coef, p0, step, scale=(1.0, 1.0, 1.0, 1.0)):
        self.coef = np.ascontiguousarray(coef)
        nx, ny, nz, _ = self.coef.shape
        self.s = OrcGrid()
        self.s.nx, self.s.ny, self.s.nz = nx, ny, nz
        for k in range(3):
            self.s.p0[k] = float(p0[k])
            self.s.step[k] = float(step[k])
        for k in range(4):
            self.s.scale[k] = float(scale[k])
        if self.coef.dtype == np.float32:
            self.s.cf32 = self.coef.ctypes.data_as(C.POINTER(C.c_float))
            self.s.cf64 = None
        else:
            self.coef = self.coef.astype(np.float64)
            self.s.cf64 = self.coef.ctypes.data_as(DP)
            self.s.cf32 = None

    def ptr(self):
        return C.byref(self.s)


class Folded:
    """Oracle view of a folded surface (SurfaceFolded, crates/libs/surfff/src/lib.rs:126-351):
    lattice (ax, bx, ay, by), harmonics kx, ky, z decays kz, z0, coefficients cq / cp / cl of
    length nx*ny*nz (index ix + nx*(iy + ny*iz)), make_plqs exponent alpha, force clamp fmax.
    Passed where a Grid goes (System.eval / relax / relax_batch)."""

    def __init__(self, ax, bx, ay, by, kx, ky, kz, z0, cq, cp, cl, alpha=2.0, fmax=100.0):
        det = ax * by - bx * ay
        if abs(det) < 1e-12:
            raise ValueError("degenerate 2D lattice")
        self.arrs = [_d(x) for x in (kx, ky, kz, z0, cq, cp, cl)]
        kx, ky, kz, z0, cq, cp, cl = self.arrs
        nb = len(kx) * len(ky) * len(kz)
        if len(z0) != len(kz) or not (len(cq) == len(cp) == len(cl) == nb):
            raise ValueError("folded surface arrays do not match nx*ny*nz")
        self.f = OrcFolded()
        idet = 1.0 / det
        for k, v in enumerate((by * idet, -bx * idet, -ay * idet, ax * idet)):
            self.f.inv[k] = v
        self.f.nx, self.f.ny, self.f.nz = len(kx), len(ky), len(kz)
        for name, a in zip(("kx", "ky", "kz", "z0", "cq", "cp", "cl"), self.arrs):
            setattr(self.f, name, a.ctypes.data_as(DP))
        self.f.alpha, self.f.fmax = float(alpha), float(fmax)
        self.s = OrcGrid()
        self.s.folded = C.pointer(self.f)

    def ptr(self):
        return C.byref(self.s)

    def points(self, pos, req):
        """Energy and clamped force of isolated atoms at pos (n, 3) with req (n, 4) = (R, sqrt E, Q, H)."""
        pos, req = _d(pos).reshape(-1, 3), _d(req).reshape(-1, 4)
        E = np.zeros(len(pos))
        F = np.zeros((len(pos), 3))
        lib().orc_folded_points(C.byref(self.f), len(pos), _dp(pos), _dp(req), _dp(E), _dp(F))
        return E, F


class System:
    """One molecule in the oracle: topology, typing and parameters."""

    def __init__(self, handle):
        self.h = C.c_void_p(handle)
        c = (C.c_int * 5)()
        lib().orc_sys_counts(self.h, c)
        self.n, self.nbonds, self.nang, self.ndih, self.ninv = list(c)

    @classmethod
    def from_molecule(cls, Z, pos, q=None, bond_cut=1.8, lattice=None):
        """lattice: (3, 3) lattice vectors a, b, c (zero rows: non-periodic axes) for a periodic
        molecule whose bonds may cross the cell; None for an isolated molecule."""
        Z = _i(Z)
        pos = _d(pos)
        q = _d(q) if q is not None else None
        if lattice is None:
            return cls(lib().orc_sys_from_molecule(len(Z), _ip(Z), _dp(pos), _dp(q), bond_cut))
        err = C.create_string_buffer(300)
        h = lib().orc_sys_from_molecule_pbc(len(Z), _ip(Z), _dp(pos), _dp(q), bond_cut, _dp(_d(lattice).reshape(9)), err, 300)
        if not h:
            raise ValueError(err.value.decode())
        return cls(h)

    def cells(self):
        """Cell codes of the neighbour slots (n, 4): 4-bit two's-complement lattice offsets x | y << 4 | z << 8."""
        out = np.zeros((self.n, 4), np.int32)
        lib().orc_sys_cells(self.h, _ip(out))
        return out

    @classmethod
    def from_bonds(cls, n, bonds, bparams, req=None):
        bonds = _i(bonds).reshape(-1, 2)
        bp = _d(bparams).reshape(-1, 2)
        req = _d(req) if req is not None else None
        return cls(lib().orc_sys_from_bonds(n, len(bonds), _ip(bonds), _dp(bp), _dp(req)))

    def __del__(self):
        try:
            if self.h:
                lib().orc_sys_free(self.h)
        except Exception:
            pass

    def export(self):
        n, nb, na, nd, ni = self.n, self.nbonds, self.nang, self.ndih, self.ninv
        out = dict(neighs=np.zeros((n, 4), np.int32), neighBs=np.zeros((n, 4), np.int32),
                   bonds=np.zeros((nb, 2), np.int32), bparams=np.zeros((nb, 2)),
                   angs=np.zeros((na, 3), np.int32), ang_ngs=np.zeros((na, 2), np.int32), angp=np.zeros((na, 5)),
                   dihs=np.zeros((nd, 4), np.int32), dih_ngs=np.zeros((nd, 3), np.int32), dihp=np.zeros((nd, 3)),
                   invs=np.zeros((ni, 4), np.int32), inv_ngs=np.zeros((ni, 3), np.int32), invp=np.zeros((ni, 4)),
                   req=np.zeros((n, 4)), type_id=np.zeros(n, np.int32))
        o = out
        lib().orc_sys_export(self.h, _ip(o["neighs"]), _ip(o["neighBs"]), _ip(o["bonds"]), _dp(o["bparams"]),
                             _ip(o["angs"]), _ip(o["ang_ngs"]), _dp(o["angp"]), _ip(o["dihs"]), _ip(o["dih_ngs"]),
                             _dp(o["dihp"]), _ip(o["invs"]), _ip(o["inv_ngs"]), _dp(o["invp"]), _dp(o["req"]),
                             _ip(o["type_id"]))
        out["types"] = [lib().orc_type_name(int(t)).decode() for t in out["type_id"]]
        return out

    def set_params(self, angp=None, dihp=None, invp=None):
        a = _d(angp) if angp is not None else None
        d = _d(dihp) if dihp is not None else None
        v = _d(invp) if invp is not None else None
        lib().orc_sys_set_params(self.h, _dp(a), _dp(d), _dp(v))

    def eval(self, pos, grid: Grid | None = None, **nb):
        pos = _d(pos)
        F = np.zeros((self.n, 3))
        Ea = np.zeros(self.n)
        Ec = np.zeros(8)
        nbp = nb_vec(**nb)
        lib().orc_eval(self.h, _dp(pos), grid.ptr() if grid is not None else None, _dp(nbp), _dp(F), _dp(Ea), _dp(Ec))
        return F, Ea, Ec

    def relax(self, pos, grid: Grid | None = None, max_steps=2000, nb=None, **fire):
        pos = _d(pos).copy()
        F = np.zeros((self.n, 3))
        Ea = np.zeros(self.n)
        Ec = np.zeros(8)
        fmax = C.c_double()
        conv = C.c_int()
        steps = lib().orc_relax(self.h, _dp(pos), grid.ptr() if grid is not None else None, _dp(nb_vec(**(nb or {}))),
                                _dp(fire_vec(**fire)), max_steps, _dp(F), _dp(Ea), _dp(Ec), C.byref(fmax),
                                C.byref(conv))
        return dict(pos=pos, F=F, Ea=Ea, Ec=Ec, steps=steps, fmax=fmax.value, conv=bool(conv.value))

    def relax_drive(self, pos, grid: Grid | None = None, max_steps=2000, nb=None, cons=None, tdrive=None, **fire):
        """relax with the driving terms of updateAtomsMMFFf4: cons = (atoms, target (m, 3), k (m, 3))
        springs, tdrive = (T [K], gamma, seed increment per step, seed) Langevin drive."""
        pos = _d(pos).copy()
        F = np.zeros((self.n, 3))
        Ea = np.zeros(self.n)
        Ec = np.zeros(8)
        fmax = C.c_double()
        conv = C.c_int()
        cv = None
        if cons is not None:
            atoms, target, k = cons
            cv = np.zeros((self.n, 7))
            cv[np.asarray(atoms, int), :3] = np.asarray(target, float).reshape(-1, 3)
            cv[np.asarray(atoms, int), 3] = 1.0
            cv[np.asarray(atoms, int), 4:] = np.broadcast_to(np.asarray(k, float), (len(atoms), 3))
        td = None if tdrive is None else _d(tdrive)
        steps = lib().orc_relax_drive(self.h, _dp(pos), grid.ptr() if grid is not None else None,
                                      _dp(nb_vec(**(nb or {}))), _dp(fire_vec(**fire)), max_steps,
                                      _dp(cv) if cv is not None else None, _dp(td) if td is not None else None,
                                      _dp(F), _dp(Ea), _dp(Ec), C.byref(fmax), C.byref(conv))
        return dict(pos=pos, F=F, Ea=Ea, Ec=Ec, steps=steps, fmax=fmax.value, conv=bool(conv.value))


E_TOT, E_BOND, E_ANG, E_DIH, E_INV, E_NB, E_GRID = range(7)


def relax_batch(systems, positions, grid=None, max_steps=2000, nthreads=0, nb=None, **fire):
    """Relax many systems in parallel (OpenMP, one system per thread). Returns dict of arrays."""
    ns = len(systems)
    hs = (C.c_void_p * ns)(*[s.h.value for s in systems])
    pos = [_d(p).copy() for p in positions]
    pp = (DP * ns)(*[_dp(p) for p in pos])
    steps = np.zeros(ns, np.int32)
    fmax = np.zeros(ns)
    conv = np.zeros(ns, np.int32)
    etot = np.zeros(ns)
    lib().orc_relax_batch(ns, hs, pp, grid.ptr() if grid is not None else None, _dp(nb_vec(**(nb or {}))),
                          _dp(fire_vec(**fire)), max_steps, _ip(steps), _dp(fmax), _ip(conv), _dp(etot), nthreads)
    return dict(pos=pos, steps=steps, fmax=fmax, conv=conv.astype(bool), etot=etot)


def langevin_noise(n, seed):
    """The thermal drive's pseudo-random vectors of atoms 0..n-1 (updateAtomsMMFFf4, UFF.cl:982-991)."""
    out = np.zeros((n, 3))
    lib().orc_langevin_noise(n, C.c_float(seed), _dp(out))
    return out


def max_threads():
    return lib().orc_max_threads()


def ljqh_pairs(dp, reqij, rdamp=1.0):
    """getLJQH (UFF.cl:82-95) in FP64 on pairs: dp (n, 3), mixed REQij (n, 4) -> (n, 4) (f, E)."""
    dp, reqij = _d(dp).reshape(-1, 3), _d(reqij).reshape(-1, 4)
    out = np.zeros((len(dp), 4))
    lib().orc_ljqh_pairs(len(dp), _dp(dp), _dp(reqij), float(rdamp) ** 2, _dp(out))
    return out


def sample_points(grid: Grid, u, plqh):
    """fe3d_pbc_comb (UFF.cl:1459-1511) in FP64: u (n, 3) grid units, PLQH (n, 4) -> (n, 4)
    (dE/du_x, dE/du_y, dE/du_z, E)."""
    u, plqh = _d(u).reshape(-1, 3), _d(plqh).reshape(-1, 4)
    out = np.zeros((len(u), 4))
    lib().orc_sample_points(grid.ptr(), len(u), _dp(u), _dp(plqh), _dp(out))
    return out


def morse_points(pts, ions, ion_req, Lx, Ly, npbc=1, alpha=1.5):
    pts = _d(pts).reshape(-1, 3)
    ions = _d(ions)
    re = _d(ion_req)
    cell = _d([Lx, 0.0, 0.0, Ly])
    out = np.zeros((len(pts), 2))
    lib().orc_morse_points(len(pts), _dp(pts), len(ions), _dp(ions), _dp(re), _dp(cell), npbc, npbc, alpha, _dp(out))
    return out


def ewald_points(pts, ions, Lx, Ly, gcut):
    pts = _d(pts).reshape(-1, 3)
    ions = _d(ions)
    out = np.zeros(len(pts))
    lib().orc_ewald_points(len(pts), _dp(pts), len(ions), _dp(ions), Lx, Ly, gcut, _dp(out))
    return out


def brute_coulomb_points(pts, ions, Lx, Ly, nrep):
    pts = _d(pts).reshape(-1, 3)
    ions = _d(ions)
    out = np.zeros(len(pts))
    lib().orc_brute_coulomb_points(len(pts), _dp(pts), len(ions), _dp(ions), Lx, Ly, nrep, _dp(out))
    return out


def bspline_fit(v):
    v = _d(v)
    nx, ny, nz = v.shape
    c = np.zeros_like(v)
    lib().orc_bspline_fit(nx, ny, nz, _dp(v), _dp(c))
    return c


def bspline_conv(c):
    c = _d(c)
    nx, ny, nz = c.shape
    v = np.zeros_like(c)
    lib().orc_bspline_conv(nx, ny, nz, _dp(c), _dp(v))
    return v


def build_grid(ions, ion_req, Lx, Ly, nx, ny, nz, p0, step, alpha=1.5, npbc=1, gcut=30.0, values=False):
    ions = _d(ions)
    re = _d(ion_req)
    coef = np.zeros((nx, ny, nz, 4))
    val = np.zeros((nx, ny, nz, 4)) if values else None
    lib().orc_build_grid(len(ions), _dp(ions), _dp(re), Lx, Ly, nx, ny, nz, _dp(_d(p0)), _dp(_d(step)), alpha, npbc,
                         gcut, _dp(coef), _dp(val))
    return (coef, val) if values else coef


def substrate_direct(pts, req_atom, ions, ion_req, Lx, Ly, npbc=1, alpha=1.5, gcut=30.0, h=1e-4):
    pts = _d(pts).reshape(-1, 3)
    ra = _d(req_atom).reshape(-1, 4)
    out = np.zeros((len(pts), 4))
    lib().orc_substrate_direct(len(pts), _dp(pts), _dp(ra), len(ions), _dp(_d(ions)), _dp(_d(ion_req)), Lx, Ly, npbc,
                               alpha, gcut, h, _dp(out))
    return out


def build_grid_fast(ions, ion_req, Lx, Ly, nx, ny, nz, p0, step, alpha=1.5, npbc=1, gtol=1e-12, morse_rcut=0.0):
    """orc_build_grid for a slab below the grid, with the separable Ewald evaluation (full-size grids).
    morse_rcut > 0 drops Morse terms of ion images farther than that from a grid column (25 A:
    dropped terms below 1e-15 of the nearest ion's); 0 keeps all, as make_MorseFF does."""
    coef = np.zeros((nx, ny, nz, 4))
    r = lib().orc_build_grid_fast(len(ions), _dp(_d(ions)), _dp(_d(ion_req)), Lx, Ly, nx, ny, nz, _dp(_d(p0)),
                                  _dp(_d(step)), alpha, npbc, gtol, _dp(coef), float(morse_rcut))
    if r != 0:
        raise ValueError("grid must lie above the slab")
    return coef


# ---------------------------------------------------------------------------------------------
# RAFF multi-replica (crates/libs/oclff/src/rrsp3.rs:699-1088, opencl/RRsp3.cl:1774-2048)

def raff_step(pos4, quat4, natoms, nnode, nsteps, topo, dt=0.1, relaxation=0.5, beta=0.0, rot_mass_scale=1.0,
              dmom=None, dqmom=None):
    """FP64 restatement of nsteps multi-replica steps.  pos4 / quat4: (nsys, natoms, 4) with the
    inverse mass in pos4[..., 3]; topo: dict(radius, neighs, excl1, excl2, fixmask, port_local,
    k, bk) in the reference's layouts.  Returns dict(pos, quat, dmom, dqmom, coll, dnode)."""
    L = lib()
    if not getattr(L, "_raff_bound", False):
        L.orc_raff_step.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, DP, C.c_int, DP, IP, IP, IP, IP, DP, DP, IP,
                                    DP, DP, DP, DP, DP, DP]
        L._raff_bound = True
    P = _d(pos4).copy()
    nsys = P.shape[0]
    Q = _d(quat4).copy()
    M = np.zeros_like(P) if dmom is None else _d(dmom).copy()
    MQ = np.zeros_like(P) if dqmom is None else _d(dqmom).copy()
    coll = np.zeros((nsys, natoms, 3))
    dnode = np.zeros((nsys, max(nnode, 1), 3))
    radius = _d(topo["radius"])
    collide = int((radius > 0).any())
    ints = [np.ascontiguousarray(topo[k], dtype=np.int32) for k in ("neighs", "excl1", "excl2", "fixmask", "bk")]
    cfg = _d([dt, relaxation, beta, rot_mass_scale])
    L.orc_raff_step(natoms, nnode, nsys, nsteps, _dp(cfg), collide, _dp(radius), _ip(ints[0]), _ip(ints[1]), _ip(ints[2]),
                    _ip(ints[3]), _dp(_d(topo["port_local"])), _dp(_d(topo["k"])), _ip(ints[4]),
                    _dp(P), _dp(Q), _dp(M), _dp(MQ), _dp(coll), _dp(dnode))
    return dict(pos=P, quat=Q, dmom=M, dqmom=MQ, coll=coll, dnode=dnode[:, :nnode])


def raff_node_order(natoms, bonds):
    """pack_molecules (crates/libs/oclff/src/pack.rs:54-116) for one molecule: nodes (bond degree > 1)
    first, then caps, each in input order.  Returns (perm, nnode)."""
    deg = np.zeros(natoms, int)
    for i, j in bonds:
        if i != j:
            deg[i] += 1
            deg[j] += 1
    nodes = [i for i in range(natoms) if deg[i] > 1]
    return np.array(nodes + [i for i in range(natoms) if deg[i] <= 1], np.int32), len(nodes)


def raff_build_neighs(natoms, bonds):
    """build_neighs_from_bonds (pack.rs:155-172)."""
    ng = -np.ones((natoms, 4), np.int32)
    deg = np.zeros(natoms, int)
    for i, j in bonds:
        if deg[i] >= 4 or deg[j] >= 4:
            raise ValueError(f"atom degree > 4 at bond {i}-{j}")
        ng[i, deg[i]] = j
        ng[j, deg[j]] = i
        deg[i] += 1
        deg[j] += 1
    return ng


def raff_exclusions(neighs):
    """make_exclusions_1st_2nd (pack.rs:176-212)."""
    n = len(neighs)
    e1 = -np.ones((n, 4), np.int32)
    e2 = -np.ones((n, 4), np.int32)
    for i in range(n):
        n1 = [int(j) for j in neighs[i] if j >= 0][:4]
        e1[i, :len(n1)] = n1
        s2 = []
        for j in n1:
            for t in neighs[j]:
                if len(s2) >= 4:
                    break
                t = int(t)
                if t < 0 or t == i or t in n1 or t in s2:
                    continue
                s2.append(t)
        e2[i, :len(s2)] = s2
    return e1, e2


def raff_bk_slots(neighs, nnode):
    """make_bk_slots_clustered (pack.rs:218-246) for one group."""
    n = len(neighs)
    bk = -np.ones((n, 4), np.int32)
    cnt = np.zeros(n, int)
    for il in range(nnode):
        for k in range(4):
            ja = neighs[il, k]
            if ja < 0:
                continue
            if cnt[ja] >= 4:
                raise ValueError(f"atom {ja} has more than 4 back slots")
            bk[ja, cnt[ja]] = 4 * il + k
            cnt[ja] += 1
    return bk


def raff_ports(pos, neighs, k_stiff):
    """make_ports_from_neighs (pack.rs:293-313), float32 as the reference."""
    pos = np.asarray(pos, np.float32)
    n = len(neighs)
    pl = np.zeros((n, 4, 4), np.float32)
    k = np.zeros((n, 4), np.float32)
    for i in range(n):
        for s in range(4):
            j = neighs[i, s]
            if j < 0:
                continue
            pl[i, s, :3] = pos[j] - pos[i]
            k[i, s] = k_stiff
    return pl, k
