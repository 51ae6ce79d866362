"""ctypes binding of oracle/_ref/libsurfref.so: the reference's own OpenCL kernels built for the host.

TEST INFRASTRUCTURE ONLY.  Loaded by tests/ and tests/golden/make_ref_fixtures.py to pin the
FP64 oracle (oracle.py) to the reference's arithmetic; the product never loads it.  The
library is built by `make -C oracle ref` from the reference's opencl/ sources (REF=<root>,
default taken from SURFMOL_REFERENCE); where neither the built library nor the reference
tree is present, available() is False and the tests that need it skip.

All arrays follow the kernels' own layouts and are FP32, as on an OpenCL device.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libsurfref.so")
EXCL_MAX = 16
_lib = None

FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int)


def reference_root():
    return os.environ.get("SURFMOL_REFERENCE", "")


def build():
    """Build from the reference tree named by SURFMOL_REFERENCE (or the Makefile's default)."""
    cmd = ["make", "-s", "-C", _HERE, "ref"]
    if reference_root():
        cmd.append("REF=" + reference_root())
    subprocess.run(cmd, check=True)


def available(build_if_missing=True) -> bool:
    """True if the library is built (building it first where the reference tree is present
    and build_if_missing is set)."""
    if not os.path.exists(LIB_PATH) and build_if_missing:
        try:
            build()
        except Exception:
            return False
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/libsurfref.so is not built and the reference tree is absent")
        L = C.CDLL(LIB_PATH)
        L.ref_mix_req.argtypes = [C.c_int, FP, FP, FP]
        L.ref_ljqh.argtypes = [C.c_int, FP, FP, C.c_float, FP]
        L.ref_sample.argtypes = [C.c_int, FP, FP, C.c_int, C.c_int, C.c_int, FP, FP]
        L.ref_nb_grid.argtypes = [C.c_int, C.c_int, FP, FP, IP, IP, FP, IP, FP, FP, IP, FP, FP, FP, C.c_int]
        L.ref_nb_grid_ex2.argtypes = [C.c_int, C.c_int, FP, FP, IP, FP, IP, FP, FP, IP, FP, FP, FP]
        L.ref_morse.argtypes = [C.c_int, FP, FP, IP, IP, FP, FP, FP, FP, FP, FP, FP]
        L.ref_bspline_conv.argtypes = [C.c_int, C.c_int, C.c_int, FP, FP, FP, C.c_float, C.c_float]
        L.ref_ewald_coefs.argtypes = [C.c_int, FP, C.c_int, FP, FP, C.c_float, FP, FP]
        L.ref_ewald_full.argtypes = [C.c_int, FP, FP, C.c_int, FP, C.c_int, FP, FP, C.c_float, FP]
        L.ref_coulomb_brute.argtypes = [C.c_int, FP, C.c_int, FP, FP, FP, C.c_int, FP]
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _fp(a):
    return None if a is None else a.ctypes.data_as(FP)


def _ip(a):
    return a.ctypes.data_as(IP)


def mix_req(reqi, reqj):
    """mixREQ_arithmetic (UFF.cl:57-65): (n, 4), (n, 4) -> (n, 4)."""
    a, b = _f(reqi).reshape(-1, 4), _f(reqj).reshape(-1, 4)
    out = np.zeros_like(a)
    lib().ref_mix_req(len(a), _fp(a), _fp(b), _fp(out))
    return out


def ljqh(dp, reqij, rdamp=1.0):
    """getLJQH (UFF.cl:82-95): dp (n, 3), mixed REQij (n, 4) -> (n, 4) (fx, fy, fz, E)."""
    dp, r = _f(dp).reshape(-1, 3), _f(reqij).reshape(-1, 4)
    out = np.zeros((len(dp), 4), np.float32)
    lib().ref_ljqh(len(dp), _fp(dp), _fp(r), C.c_float(np.float32(rdamp) * np.float32(rdamp)), _fp(out))
    return out


def sample(grid, u, plqh):
    """fe3d_pbc_comb (UFF.cl:1459-1511) with its make_inds_pbc tables.  grid (nx, ny, nz, 4)
    z fastest; u (n, 3) grid units; PLQH (n, 4) -> (n, 4) (dE/du_x, dE/du_y, dE/du_z, E)."""
    g = _f(grid)
    nx, ny, nz, _ = g.shape
    u, p = _f(u).reshape(-1, 3), _f(plqh).reshape(-1, 4)
    out = np.zeros((len(u), 4), np.float32)
    lib().ref_sample(len(u), _fp(u), _fp(p), nx, ny, nz, _fp(g), _fp(out))
    return out


def _lvecs(lvec, nsys):
    lv = np.zeros((nsys, 3, 4), np.float32)
    if lvec is not None:
        lv[:, :, :3] = np.asarray(lvec, np.float32).reshape(3, 3)
    return lv


def nb_grid(atoms, reqks, neighs, grid, p0, step, rdamp=1.0, alpha=1.5, neighcell=None, lvec=None, npbc=(0, 0, 0),
            nbff=True, forces=None):
    """getNonBond_GridFF_Bspline (UFF.cl:1524-1718) over nsys systems of natoms atoms each.
    atoms / reqks (nsys, natoms, 4), neighs (nsys, natoms, 4) -> forces (nsys, natoms, 4):
    (fx, fy, fz, E) per atom, NB pairs (both atoms' energies) plus the grid.  grid (nx, ny, nz, 4)
    B-spline coefficients z fastest; p0, step its origin and spacing.  GFFParams = (rdamp, alpha)."""
    A = _f(atoms)
    nsys, natoms, _ = A.shape
    R, N = _f(reqks), _i(neighs)
    NC = _i(np.zeros_like(N) if neighcell is None else neighcell)
    g = _f(grid)
    gns = _i([g.shape[0], g.shape[1], g.shape[2], 0])
    F = np.zeros((nsys, natoms, 4), np.float32) if forces is None else _f(forces).copy()
    lib().ref_nb_grid(nsys, natoms, _fp(A), _fp(R), _ip(N), _ip(NC), _fp(_lvecs(lvec, nsys)), _ip(_i(list(npbc) + [0])),
                      _fp(_f([rdamp, alpha, 0, 0])), _fp(g), _ip(gns), _fp(_f([1 / step[0], 1 / step[1], 1 / step[2], 0])),
                      _fp(_f([p0[0], p0[1], p0[2], 0])), _fp(F), 1 if nbff else 0)
    return F


def nb_grid_ex2(atoms, reqks, excl, grid, p0, step, rdamp=1.0, alpha=1.5):
    """getNonBond_GridFF_Bspline_ex2 (UFF.cl:1722-): as nb_grid with the sorted, -1 padded
    exclusion list excl (nsys, natoms, EXCL_MAX) of make_second_neighs (molff/src/nonbonded.rs:112-137)."""
    A = _f(atoms)
    nsys, natoms, _ = A.shape
    R, X = _f(reqks), _i(excl)
    g = _f(grid)
    gns = _i([g.shape[0], g.shape[1], g.shape[2], 0])
    F = np.zeros((nsys, natoms, 4), np.float32)
    lib().ref_nb_grid_ex2(nsys, natoms, _fp(A), _fp(R), _ip(X), _fp(_lvecs(None, nsys)), _ip(_i([0, 0, 0, 0])),
                          _fp(_f([rdamp, alpha, 0, 0])), _fp(g), _ip(gns), _fp(_f([1 / step[0], 1 / step[1], 1 / step[2], 0])),
                          _fp(_f([p0[0], p0[1], p0[2], 0])), _fp(F))
    return F


def second_neighs(neighs):
    """make_second_neighs (molff/src/nonbonded.rs:112-137): per atom the sorted 1-2 and 1-3
    neighbours, -1 padded to EXCL_MAX.  neighs (natoms, 4) -> (natoms, EXCL_MAX)."""
    ng = np.asarray(neighs)
    n = len(ng)
    out = -np.ones((n, EXCL_MAX), np.int32)
    for ia in range(n):
        ex = []

        def add(j):
            if j < 0 or j == ia or j >= n or j in ex:
                return
            if len(ex) >= EXCL_MAX:
                raise ValueError(f"atom {ia}: more than {EXCL_MAX} exclusions")
            ex.append(int(j))
        for j in ng[ia]:
            add(j)
        for j in ng[ia]:
            if 0 <= j < n:
                for k in ng[j]:
                    add(k)
        ex.sort()
        out[ia, :len(ex)] = ex
    return out


def morse(ions, reqs, lvec, ngrid, p0, alpha=1.5, rdamp=1.0, npbc=(1, 1, 0)):
    """make_MorseFF (gridff_build.cl:217-347): ions (n, 4) positions, reqs (n, 4) (R, E, ...),
    lvec (3, 3) cell, ngrid (nx, ny, nz) points over the cell, x fastest -> (Paul, Lond) arrays
    of shape (nz, ny, nx)."""
    A, R = _f(ions), _f(reqs)
    nx, ny, nz = ngrid
    lv = np.zeros((3, 4), np.float32)
    lv[:, :3] = np.asarray(lvec, np.float32)
    P = np.zeros(nx * ny * nz, np.float32)
    Lo = np.zeros_like(P)
    lib().ref_morse(len(A), _fp(A), _fp(R), _ip(_i(list(npbc) + [0])), _ip(_i([nx, ny, nz, 0])), _fp(lv[0]), _fp(lv[1]),
                    _fp(lv[2]), _fp(_f([p0[0], p0[1], p0[2], 0])), _fp(_f([rdamp, alpha, 0, 0])), _fp(P), _fp(Lo))
    return P.reshape(nz, ny, nx), Lo.reshape(nz, ny, nx)


def bspline_conv(Gs, G0=None, cx=1.0, cy=0.0):
    """BsplineConv3D (gridff_build.cl:8-61): Gs (nz, ny, nx) x fastest -> cx*conv(Gs) + cy*G0."""
    g = _f(Gs)
    nz, ny, nx = g.shape
    g0 = None if G0 is None else _f(G0)
    out = np.zeros_like(g)
    lib().ref_bspline_conv(nx, ny, nz, _fp(g), _fp(g0), _fp(out), cx, cy)
    return out


def g_list(Lx, Ly, gcut):
    """The (h, k, |G|, 0) rows of every G != 0 with |G| <= gcut of an orthogonal Lx x Ly cell,
    and the reciprocal vectors b1, b2 (rows)."""
    g1, g2 = 2 * np.pi / Lx, 2 * np.pi / Ly
    H, K = int(np.floor(gcut / g1)), int(np.floor(gcut / g2))
    rows = []
    for h in range(-H, H + 1):
        for k in range(-K, K + 1):
            if h == 0 and k == 0:
                continue
            gn = np.hypot(h * g1, k * g2)
            if gn <= gcut:
                rows.append((h, k, gn, 0.0))
    return np.array(rows, np.float32), np.array([[g1, 0.0], [0.0, g2]], np.float32)


def ewald_full(pts, ions, Lx, Ly, gcut):
    """compute_ewald_coefficients then eval_potential_full (Surface.cl:716-767, 834-906):
    ions (n, 4: x, y, z, q), pts (m, 3) -> phi (m,) in eV/e."""
    I = _f(ions)
    G, b = g_list(Lx, Ly, gcut)
    CG = np.zeros((len(G), 2), np.float32)
    w = np.zeros((len(G), len(I), 2), np.float32)
    lib().ref_ewald_coefs(len(I), _fp(I), len(G), _fp(G), _fp(b), Lx * Ly, _fp(CG), _fp(w))
    P = np.zeros((len(pts), 4), np.float32)
    P[:, :3] = pts
    phi = np.zeros(len(pts), np.float32)
    lib().ref_ewald_full(len(P), _fp(P), _fp(w), len(I), _fp(I), len(G), _fp(G), _fp(b), Lx * Ly, _fp(phi))
    return phi


def coulomb_brute(pts, ions, Lx, Ly, nrep):
    """eval_potential_brute (Surface.cl:911-954): circular image sum of radius nrep cells."""
    I = _f(ions)
    P = np.zeros((len(pts), 4), np.float32)
    P[:, :3] = pts
    phi = np.zeros(len(pts), np.float32)
    lib().ref_coulomb_brute(len(P), _fp(P), len(I), _fp(I), _fp(_f([Lx, 0])), _fp(_f([0, Ly])), nrep, _fp(phi))
    return phi
