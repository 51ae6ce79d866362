"""Python host interface over the C ABI: the multi-system relaxation driver.

``RelaxMulti`` mirrors the shape of the reference's multi-replica GPU harness
(crates/libs/oclff/src/rrsp3.rs:699-1088, RRsp3Multi: new / upload_* /
step_*_multi / download_* / finish) for the UFF + GridFF FIRE path: upload
molecules and systems, set or build the substrate grid, run FIRE steps,
read back positions, forces and energies.  All numerics run in the CUDA
library; this module only marshals arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

GRID_F32, GRID_F16, GRID_BF16 = 0, 1, 2
MODE_BATCHED, MODE_PLAIN = 0, 1
FORM_ROUNDS, FORM_GATHER, FORM_OWNER = 0, 1, 2
ST_RUNNING, ST_CONVERGED, ST_MAXSTEPS, ST_NONFINITE = 0, 1, 2, 3
E_TOTAL, E_BOND, E_ANGLE, E_DIH, E_INV, E_NB, E_GRID = range(7)

# FireState defaults (crates/libs/molff/src/raff.rs:1053-1055), dt_max 0.05 as the
# pentacene relaxation uses (crates/libs/surfmol/tests/relax_pentacene_uff.rs:259).
FIRE_DEFAULT = dict(dt0=0.001, dt_max=0.05, alpha0=0.1, f_inc=1.1, f_dec=0.5, f_alpha=0.99, n_min=5,
                    fconv=1e-3, flimit=0.0)


class SmrError(RuntimeError):
    pass


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def fire_params(**kw) -> N.SmrFireParams:
    p = dict(FIRE_DEFAULT)
    p.update(kw)
    return N.SmrFireParams(p["dt0"], p["dt_max"], p["alpha0"], p["f_inc"], p["f_dec"], p["f_alpha"], int(p["n_min"]),
                           p["fconv"], p["flimit"])


_EXPORT_SHAPES = [("neighs", 4, np.int32), ("neighBs", 4, np.int32), ("bonds", 2, np.int32),
                  ("bparams", 2, np.float64), ("angs", 3, np.int32), ("ang_ngs", 2, np.int32),
                  ("angp", 5, np.float64), ("dihs", 4, np.int32), ("dih_ngs", 3, np.int32),
                  ("dihp", 3, np.float64), ("invs", 4, np.int32), ("inv_ngs", 3, np.int32),
                  ("invp", 4, np.float64), ("req", 4, np.float64), ("type_id", 1, np.int32)]
_COUNT_OF = {"neighs": 0, "neighBs": 0, "bonds": 1, "bparams": 1, "angs": 2, "ang_ngs": 2, "angp": 2, "dihs": 3,
             "dih_ngs": 3, "dihp": 3, "invs": 4, "inv_ngs": 4, "invp": 4, "req": 0, "type_id": 0}


def _export_arrays(counts):
    out = {}
    for name, w, dt in _EXPORT_SHAPES:
        n = counts[_COUNT_OF[name]]
        out[name] = np.zeros((n, w) if w > 1 else n, dtype=dt)
    return out


def _export_ptrs(out):
    ptrs = []
    for name, _, dt in _EXPORT_SHAPES:
        ptrs.append(out[name].ctypes.data_as(N.IP if dt == np.int32 else N.DP))
    return ptrs


def type_name(tid: int) -> str:
    return N.lib().smr_type_name(int(tid)).decode()


class Topology:
    """Host-only molecule preparation (bonds by cutoff, UFF typing, terms, parameters)."""

    def __init__(self, Z, pos, charges=None, bond_cut=1.8):
        L = N.lib()
        Z = _i(Z)
        pos = _d(pos)
        q = _d(charges) if charges is not None else None
        h = N.VP()
        err = C.create_string_buffer(300)
        r = L.smr_topo_build(len(Z), _p(Z, N.IP), _p(pos, N.DP), _p(q, N.DP), bond_cut, C.byref(h), err, 300)
        if r != 0:
            raise SmrError(f"smr_topo_build: {err.value.decode()}")
        self.h = h
        c = (C.c_int * 5)()
        L.smr_topo_counts(self.h, c)
        self.counts = list(c)
        self.n = self.counts[0]

    def __del__(self):
        try:
            if self.h:
                N.lib().smr_topo_free(self.h)
        except Exception:
            pass

    @classmethod
    def from_lists(cls, Z, bonds, angles, dihedrals, inversions, charges=None, types=None):
        """Host topology from explicit bond / term lists (a topology file): lists used as given;
        types: UFF type names (None: typed from Z and the bond graph)."""
        L = N.lib()
        Z = _i(Z)
        b, a, d, v = (_i(np.asarray(x).reshape(-1, w)) for x, w in ((bonds, 2), (angles, 3), (dihedrals, 4), (inversions, 4)))
        tid = None
        if types is not None:
            tid = _i([L.smr_type_id(t.encode()) for t in types])
            if (tid < 0).any():
                raise SmrError(f"unknown UFF type {types[int(np.argmin(tid))]!r}")
        q = _d(charges) if charges is not None else None
        h = N.VP()
        err = C.create_string_buffer(300)
        r_ = L.smr_topo_build_listed(len(Z), _p(Z, N.IP), _p(tid, N.IP), _p(q, N.DP), len(b), _p(b, N.IP), len(a), _p(a, N.IP),
                                     len(d), _p(d, N.IP), len(v), _p(v, N.IP), C.byref(h), err, 300)
        if r_ != 0:
            raise SmrError(f"smr_topo_build_listed: {err.value.decode()}")
        t = cls.__new__(cls)
        t.h = h
        c = (C.c_int * 5)()
        L.smr_topo_counts(t.h, c)
        t.counts = list(c)
        t.n = t.counts[0]
        return t

    def export(self):
        out = _export_arrays(self.counts)
        N.lib().smr_topo_export(self.h, *_export_ptrs(out))
        out["types"] = [type_name(t) for t in out["type_id"]]
        return out

    def prepare(self, team=0):
        """Pack the term records for a team size off any handle (thread-safe; releases the GIL)."""
        r = N.lib().smr_topo_prepare(self.h, int(team))
        if r != 0:
            raise SmrError(f"smr_topo_prepare ({r})")

    def rounds(self, team):
        L = N.lib()
        r = (C.c_int * 3)()
        L.smr_topo_rounds(self.h, team, r, None, None, None)
        arrs = [np.zeros((r[k] * team, 4), np.int16) for k in range(3)]
        L.smr_topo_rounds(self.h, team, r, *[a.ctypes.data_as(N.SP) for a in arrs])
        return list(r), arrs


class RelaxMulti:
    """Many molecules relaxed by FIRE in parallel over one substrate grid, on one GPU."""

    def __init__(self, max_systems: int, max_atoms: int, device: int = 0):
        self.max_systems = int(max_systems)
        self.L = N.lib()
        cfg = N.SmrConfig(device, int(max_systems), int(max_atoms))
        h = N.VP()
        r = self.L.smr_create(C.byref(cfg), C.byref(h))
        if r != 0:
            raise SmrError(f"smr_create failed ({r}): CUDA device {device} unavailable or out of memory")
        self.h = h
        self.natoms_of = {}     # slot -> natoms
        self.topo_n = []        # topology id -> natoms
        self._nat = np.zeros(int(max_systems), np.int64)   # slot -> natoms (0: free), for vectorised checks

    # -- lifecycle
    def finish(self):
        if self.h:
            self.L.smr_destroy(self.h)
            self.h = None

    close = finish

    def __del__(self):
        try:
            self.finish()
        except Exception:
            pass

    def _chk(self, r, what):
        if r != 0:
            raise SmrError(f"{what} ({r}): {self.L.smr_last_error(self.h).decode()}")

    # -- parameters and grid
    def set_nb(self, rdamp=1.0, alpha_morse=1.5, rcut=0.0, excl13=False):
        """GFFParams (rdamp, Morse alpha), intramolecular cutoff (<= 0: none) and the exclusion
        rule: 1-2 pairs (getNonBond_GridFF_Bspline) or, with excl13, 1-2 and 1-3 pairs
        (getNonBond_GridFF_Bspline_ex2)."""
        p = N.SmrNbParams(rdamp, alpha_morse, rcut, 1 if excl13 else 0)
        self._chk(self.L.smr_set_nb_params(self.h, C.byref(p)), "smr_set_nb_params")

    def set_grid(self, coef, p0, step, dtype=GRID_F32, scale=(1, 1, 1, 1), plane_scale=None):
        """coef: (nx, ny, nz, 4) float32 (F32) or uint16 (F16/BF16 bit patterns), z-fastest;
        16-bit grids take per-channel `scale` or an (nz, 4) per-plane `plane_scale`."""
        coef = np.ascontiguousarray(coef)
        nx, ny, nz, _ = coef.shape
        if plane_scale is not None:
            ps = _f(plane_scale)
            self._chk(self.L.smr_set_grid_planes(self.h, coef.ctypes.data_as(N.VP), dtype, _p(ps, N.FP), nx, ny, nz,
                                                 _p(_d(p0), N.DP), _p(_d(step), N.DP)), "smr_set_grid_planes")
            return
        sc = _f(scale)
        self._chk(self.L.smr_set_grid(self.h, coef.ctypes.data_as(N.VP), dtype, _p(sc, N.FP), nx, ny, nz,
                                      _p(_d(p0), N.DP), _p(_d(step), N.DP)), "smr_set_grid")

    def set_grid_device(self, dev_ptr, dims, p0, step, dtype=GRID_F32, scale=(1, 1, 1, 1)):
        """Grid coefficients already on the device (an int address, e.g. a torch tensor's data_ptr();
        dims = (nx, ny, nz), layout as set_grid), copied device to device."""
        sc = _f(scale)
        self._chk(self.L.smr_set_grid_device(self.h, N.VP(int(dev_ptr)), dtype, _p(sc, N.FP), int(dims[0]), int(dims[1]),
                                             int(dims[2]), _p(_d(p0), N.DP), _p(_d(step), N.DP)), "smr_set_grid_device")

    def get_grid(self):
        dt = C.c_int()
        sc = (C.c_float * 4)()
        dims = (C.c_int * 3)()
        p0 = (C.c_double * 3)()
        st = (C.c_double * 3)()
        self._chk(self.L.smr_get_grid(self.h, None, C.byref(dt), sc, dims, p0, st), "smr_get_grid")
        shape = (dims[0], dims[1], dims[2], 4)
        buf = np.zeros(shape, np.float32 if dt.value == GRID_F32 else np.uint16)
        self._chk(self.L.smr_get_grid(self.h, buf.ctypes.data_as(N.VP), None, None, None, None, None), "smr_get_grid")
        ps = np.zeros((dims[2], 4), np.float32)
        self._chk(self.L.smr_get_grid_planes(self.h, _p(ps, N.FP)), "smr_get_grid_planes")
        return dict(coef=buf, dtype=dt.value, scale=np.array(list(sc)), plane_scale=ps, p0=np.array(list(p0)),
                    step=np.array(list(st)))

    def build_grid(self, ions, ion_re, Lx, Ly, nx, ny, nz, p0, step, alpha_morse=1.5, npbc=1, ewald_tol=1e-12,
                   dtype=GRID_F32, morse_rcut=0.0):
        ions = _d(ions)
        re = _d(np.asarray(ion_re)[:, :2])
        p = N.SmrGridBuildParams(alpha_morse, npbc, ewald_tol, dtype, morse_rcut)
        self._chk(self.L.smr_build_grid(self.h, len(ions), _p(ions, N.DP), _p(re, N.DP), Lx, Ly, nx, ny, nz,
                                        _p(_d(p0), N.DP), _p(_d(step), N.DP), C.byref(p)), "smr_build_grid")

    def grid_raw_slab(self, ions, ion_re, Lx, Ly, nx, ny, nz, p0, step, x0, nxs, raw_dev_ptr, alpha_morse=1.5, npbc=1,
                      ewald_tol=1e-12, morse_rcut=0.0):
        """Raw FP64 (Pauli, London, Coulomb) triples of x-planes [x0, x0 + nxs) into the device buffer at
        raw_dev_ptr (an int address, e.g. a torch tensor's data_ptr(); 3 nxs ny nz doubles)."""
        ions = _d(ions)
        re = _d(np.asarray(ion_re)[:, :2])
        p = N.SmrGridBuildParams(alpha_morse, npbc, ewald_tol, GRID_F32, morse_rcut)
        self._chk(self.L.smr_grid_raw_slab(self.h, len(ions), _p(ions, N.DP), _p(re, N.DP), Lx, Ly, nx, ny, nz,
                                           _p(_d(p0), N.DP), _p(_d(step), N.DP), C.byref(p), int(x0), int(nxs),
                                           N.VP(int(raw_dev_ptr))), "smr_grid_raw_slab")

    def grid_from_raw(self, raw_dev_ptr, nx, ny, nz, p0, step, dtype=GRID_F32):
        """Fit and install the grid from 3 nx ny nz raw FP64 values on the device (grid_raw_slab's layout)."""
        self._chk(self.L.smr_grid_from_raw(self.h, N.VP(int(raw_dev_ptr)), nx, ny, nz, _p(_d(p0), N.DP), _p(_d(step), N.DP),
                                           int(dtype)), "smr_grid_from_raw")

    def convert_grid(self, dtype):
        self._chk(self.L.smr_convert_grid(self.h, dtype), "smr_convert_grid")

    def convert_grid_split(self, dtype, zsplit):
        """The FP32 grid becomes a 16-bit grid plus an FP32 copy of its planes [0, zsplit + 3):
        atoms whose stencil starts below plane zsplit read the FP32 copy."""
        self._chk(self.L.smr_convert_grid_split(self.h, dtype, int(zsplit)), "smr_convert_grid_split")

    def get_grid_split(self, planes=False):
        """(zsplit, FP32 planes as an (nx, ny, zsplit + 3, 4) array or None)."""
        zs = C.c_int()
        self._chk(self.L.smr_get_grid_split(self.h, C.byref(zs), None), "smr_get_grid_split")
        if not planes or zs.value == 0:
            return zs.value, None
        g = self.get_grid_dims()
        lo = np.zeros((g[0], g[1], zs.value + 3, 4), np.float32)
        self._chk(self.L.smr_get_grid_split(self.h, C.byref(zs), _p(lo, N.FP)), "smr_get_grid_split")
        return zs.value, lo

    def get_grid_dims(self):
        dims = (C.c_int * 3)()
        self._chk(self.L.smr_get_grid(self.h, None, None, None, dims, None, None), "smr_get_grid")
        return tuple(dims)

    def set_surface_folded(self, surf):
        """Folded-surface substrate in place of the grid (a ``folded.FoldedSurface``, or None to go
        back to the grid): MolWorld's SurfaceFolded with its per-atom force clamp."""
        if surf is None:
            self._chk(self.L.smr_set_surface_folded(self.h, None), "smr_set_surface_folded")
            return
        arrs = [_d(np.ravel(getattr(surf, k))) for k in ("kx", "ky", "kz", "z0", "cq", "cp", "cl")]
        kx, ky, kz, z0, cq, cp, cl = arrs
        if len(z0) != len(kz) or not (len(cq) == len(cp) == len(cl) == len(kx) * len(ky) * len(kz)):
            raise ValueError("folded surface arrays do not match nx*ny*nz")
        f = N.SmrFoldedSurface(surf.ax, surf.bx, surf.ay, surf.by, len(kx), len(ky), len(kz),
                               *[_p(a, N.DP) for a in arrs], surf.alpha, surf.fmax)
        self._chk(self.L.smr_set_surface_folded(self.h, C.byref(f)), "smr_set_surface_folded")

    def set_schedule(self, switch_step=0, latency_team=0, eval_form=0):
        self._chk(self.L.smr_set_schedule(self.h, switch_step, latency_team, eval_form), "smr_set_schedule")

    def get_schedule(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._chk(self.L.smr_get_schedule(self.h, C.byref(a), C.byref(b), C.byref(c)), "smr_get_schedule")
        return a.value, b.value, c.value

    def set_stages(self, starts, forms, teams, eval_form=FORM_ROUNDS):
        """Multi-stage schedule: stage k runs FIRE steps [starts[k], starts[k+1]) in forms[k]
        (FORM_ROUNDS / FORM_GATHER / FORM_OWNER) with teams[k] threads per system (0: by size)."""
        st, fm, tm = _i(starts), _i(forms), _i(teams)
        if not (len(st) == len(fm) == len(tm)):
            raise ValueError("starts, forms and teams differ in length")
        self._chk(self.L.smr_set_stages(self.h, len(st), _p(st, N.IP), _p(fm, N.IP), _p(tm, N.IP), eval_form),
                  "smr_set_stages")

    def get_stages(self):
        n = C.c_int(16)
        st, fm, tm = (np.zeros(16, np.int32) for _ in range(3))
        self._chk(self.L.smr_get_stages(self.h, C.byref(n), _p(st, N.IP), _p(fm, N.IP), _p(tm, N.IP)), "smr_get_stages")
        k = n.value
        return st[:k].tolist(), fm[:k].tolist(), tm[:k].tolist()

    def set_nb_lanes(self, lanes):
        """Lanes per atom in the NB partner loop (0: chosen from system size and team)."""
        self._chk(self.L.smr_set_tuning(self.h, 1, int(lanes)), "smr_set_tuning")

    def set_grid_bricks(self, mode):
        """Grid layout the relax kernel reads: -1 (default) the brick copy for grids larger than
        128 MiB, 0 the z-fastest grid, 1 the brick copy always (results identical bit for bit)."""
        self._chk(self.L.smr_set_tuning(self.h, 6, int(mode)), "smr_set_tuning")

    def set_grid_prefetch(self, on=True):
        """With the brick copy: request each evaluation's stencil lines into L2 at its start."""
        self._chk(self.L.smr_set_tuning(self.h, 8, 1 if on else 0), "smr_set_tuning")

    def set_smem_carveout(self, percent=-1):
        """Block teams' preferred shared-memory share of L1 in percent (-1: driver default)."""
        self._chk(self.L.smr_set_tuning(self.h, 9, int(percent)), "smr_set_tuning")

    def set_occupancy_tiers(self, on=True):
        """Split launch segments by the occupancy each system's size allows (default off)."""
        self._chk(self.L.smr_set_tuning(self.h, 10, 1 if on else 0), "smr_set_tuning")

    def grid_bricks_active(self) -> bool:
        """True if the last relaxation or force evaluation read the brick copy of the grid."""
        v = C.c_int()
        self._chk(self.L.smr_get_tuning(self.h, 7, C.byref(v)), "smr_get_tuning")
        return bool(v.value)

    def set_watchdog(self, ms):
        """Longest wait for device work per call (ms); a call that gives up raises SmrError (-6) and the
        next call waits for the abandoned work first."""
        self._chk(self.L.smr_set_tuning(self.h, 5, int(ms)), "smr_set_tuning")

    def set_nblist(self, min_atoms=None, skin=None, cap=None):
        """NB neighbour lists for systems of >= min_atoms atoms under a cutoff (0: off); skin in A."""
        if min_atoms is not None:
            self._chk(self.L.smr_set_tuning(self.h, 2, int(min_atoms)), "smr_set_tuning")
        if skin is not None:
            self._chk(self.L.smr_set_tuning(self.h, 3, int(round(skin * 1000))), "smr_set_tuning")
        if cap is not None:
            self._chk(self.L.smr_set_tuning(self.h, 4, int(cap)), "smr_set_tuning")

    def get_nb_lanes(self):
        v = C.c_int()
        self._chk(self.L.smr_get_tuning(self.h, 1, C.byref(v)), "smr_get_tuning")
        return v.value

    def set_graph(self, on=True):
        """Replay the batched launch sequence as a CUDA graph when a call repeats the last plan."""
        self._chk(self.L.smr_set_graph(self.h, 1 if on else 0), "smr_set_graph")

    def graph_replays(self):
        v = C.c_longlong()
        self._chk(self.L.smr_graph_stats(self.h, C.byref(v)), "smr_graph_stats")
        return v.value

    def set_team_size(self, max_atoms, threads):
        self._chk(self.L.smr_set_team_size(self.h, max_atoms, threads), "smr_set_team_size")

    # -- molecules
    def add_molecule(self, Z, pos, charges=None, bond_cut=1.8) -> int:
        Z = _i(Z)
        pos = _d(pos)
        q = _d(charges) if charges is not None else None
        tid = C.c_int()
        self._chk(self.L.smr_add_molecule(self.h, len(Z), _p(Z, N.IP), _p(pos, N.DP), _p(q, N.DP), bond_cut,
                                          C.byref(tid)), "smr_add_molecule")
        self.topo_n.append(len(Z))
        return tid.value

    def add_molecule_pbc(self, Z, pos, lattice, charges=None, bond_cut=1.8, npbc=None) -> int:
        """A periodic molecule: ``lattice`` (3, 3) rows a, b, c (zero rows: non-periodic axes); bonds
        may reach a partner's image in the next cell.  ``npbc``: NB images each side per axis for the
        systems made from it (default 1 along the periodic axes)."""
        Z = _i(Z)
        pos = _d(pos)
        q = _d(charges) if charges is not None else None
        lat = _d(np.asarray(lattice, float).reshape(9))
        nimg = _i(npbc) if npbc is not None else None
        tid = C.c_int()
        self._chk(self.L.smr_add_molecule_pbc(self.h, len(Z), _p(Z, N.IP), _p(pos, N.DP), _p(q, N.DP), bond_cut,
                                              _p(lat, N.DP), _p(nimg, N.IP), C.byref(tid)), "smr_add_molecule_pbc")
        self.topo_n.append(len(Z))
        return tid.value

    def set_pbc(self, slots, lattice, npbc):
        """Per-system lattice ((3, 3) or one per slot) and NB images each side ((3,) or one per slot)."""
        slots = _i(slots)
        n = len(slots)
        lat = _d(np.broadcast_to(np.asarray(lattice, float).reshape(-1, 9), (n, 9)))
        nimg = _i(np.broadcast_to(np.asarray(npbc).reshape(-1, 3), (n, 3)))
        self._chk(self.L.smr_set_pbc(self.h, n, _p(slots, N.IP), _p(lat, N.DP), _p(nimg, N.IP)), "smr_set_pbc")

    def get_pbc(self, slot):
        lat = np.zeros(9)
        nimg = np.zeros(3, np.int32)
        self._chk(self.L.smr_get_pbc(self.h, int(slot), _p(lat, N.DP), _p(nimg, N.IP)), "smr_get_pbc")
        return lat.reshape(3, 3), nimg

    def set_constraints(self, slot, atoms=(), target=None, k=None):
        """Harmonic position constraints of one system: atoms (n,), target (n, 3) positions, k (n, 3)
        or (n,) or scalar stiffness per axis (eV/A^2).  No atoms: remove them."""
        atoms = _i(np.ravel(atoms))
        n = len(atoms)
        tgt = _d(np.asarray(target if n else np.zeros((0, 3)), float).reshape(n, 3))
        kk = np.asarray(k if n else 0.0, float)
        kk = _d(np.broadcast_to(kk.reshape(-1, 1) if kk.ndim == 1 else kk, (n, 3)))
        self._chk(self.L.smr_set_constraints(self.h, int(slot), n, _p(atoms, N.IP), _p(tgt, N.DP), _p(kk, N.DP)),
                  "smr_set_constraints")

    def set_thermal_drive(self, slots, T, gamma, seed=0.0, seed_step=0.0):
        """Langevin drive of updateAtomsMMFFf4 on systems: temperature T [K], damping gamma, seed and
        the seed's increment per FIRE step (each a scalar or one value per slot).  gamma <= 0: off."""
        slots = _i(np.ravel(slots))
        n = len(slots)
        td = _d(np.stack([np.broadcast_to(np.asarray(x, float), (n,)) for x in (T, gamma, seed_step, seed)], 1))
        self._chk(self.L.smr_set_thermal_drive(self.h, n, _p(slots, N.IP), _p(td, N.DP)), "smr_set_thermal_drive")

    def topology_counts(self, topo_id):
        """(natoms, nbonds, nang, ndih, ninv, type-rounds) of a topology on the handle."""
        c = (C.c_int * 6)()
        self._chk(self.L.smr_topology_counts(self.h, int(topo_id), c), "smr_topology_counts")
        return list(c)

    def topology_export(self, topo_id):
        """The topology's lists and parameters, as Topology.export."""
        out = _export_arrays(self.topology_counts(topo_id)[:5])
        self._chk(self.L.smr_topology_export(self.h, int(topo_id), *_export_ptrs(out)), "smr_topology_export")
        return out

    def topology_cells(self, topo_id):
        """Cell code of each neighbour slot (natoms, 4)."""
        out = np.zeros((self.topo_n[topo_id], 4), np.int32)
        self._chk(self.L.smr_topology_cells(self.h, int(topo_id), _p(out, N.IP)), "smr_topology_cells")
        return out

    def add_molecules(self, Zs, poss, charges=None, bond_cut=1.8):
        """Many molecules at once (typing and packing on all host cores); returns their topology ids."""
        n = _i([len(z) for z in Zs])
        Z = _i(np.concatenate([np.asarray(z) for z in Zs])) if len(Zs) else _i([])
        P = _d(np.concatenate([np.asarray(p).reshape(-1, 3) for p in poss])) if len(Zs) else _d(np.zeros((0, 3)))
        q = _d(np.concatenate([np.asarray(c) for c in charges])) if charges is not None and len(Zs) else None
        ids = np.zeros(len(Zs), np.int32)
        self._chk(self.L.smr_add_molecules(self.h, len(Zs), _p(n, N.IP), _p(Z, N.IP), _p(P, N.DP), _p(q, N.DP), bond_cut,
                                           _p(ids, N.IP)), "smr_add_molecules")
        self.topo_n.extend(int(k) for k in n)
        return ids

    def add_listed_molecule(self, Z, bonds, angles, dihedrals, inversions, charges=None, types=None) -> int:
        """A molecule from explicit bond / term lists (a topology file); see topo_io."""
        Z = _i(Z)
        b, a, d, v = (_i(np.asarray(x).reshape(-1, w)) for x, w in ((bonds, 2), (angles, 3), (dihedrals, 4), (inversions, 4)))
        tid = None
        if types is not None:
            tid = _i([self.L.smr_type_id(t.encode()) for t in types])
            if (tid < 0).any():
                raise SmrError(f"unknown UFF type {types[int(np.argmin(tid))]!r}")
        q = _d(charges) if charges is not None else None
        out = C.c_int()
        self._chk(self.L.smr_add_listed_molecule(self.h, len(Z), _p(Z, N.IP), _p(tid, N.IP), _p(q, N.DP), len(b), _p(b, N.IP),
                                                 len(a), _p(a, N.IP), len(d), _p(d, N.IP), len(v), _p(v, N.IP), C.byref(out)),
                  "smr_add_listed_molecule")
        self.topo_n.append(len(Z))
        return out.value

    def add_topology_file(self, path, charges=None):
        """Add the molecule of a TopologyData JSON or UFFTOPO file; returns (topology id, positions)."""
        from .topo_io import read
        d = read(path)
        tid = self.add_listed_molecule(d["Z"], d["bonds"], d["angles"], d["dihedrals"], d["inversions"], charges,
                                       d["types"])
        return tid, d["positions"]

    def add_topo(self, topo: Topology) -> int:
        tid = C.c_int()
        self._chk(self.L.smr_add_topo(self.h, topo.h, C.byref(tid)), "smr_add_topo")
        self.topo_n.append(topo.n)
        return tid.value

    def add_topos(self, topos) -> np.ndarray:
        """Attach many host topologies with one device upload; returns their ids."""
        arr = (N.VP * len(topos))(*[t.h.value for t in topos])
        ids = np.zeros(len(topos), np.int32)
        self._chk(self.L.smr_add_topos(self.h, len(topos), arr, _p(ids, N.IP)), "smr_add_topos")
        self.topo_n.extend(t.n for t in topos)
        return ids

    def remove_topologies(self, tids):
        t = _i(tids)
        self._chk(self.L.smr_remove_topologies(self.h, len(t), _p(t, N.IP)), "smr_remove_topologies")

    def remove_topology(self, tid):
        self._chk(self.L.smr_remove_topology(self.h, int(tid)), "smr_remove_topology")

    def add_topology(self, req, neighs, bond_kl, angs=None, angp=None, dihs=None, dihp=None, invs=None, invp=None):
        req = _d(req)
        n = len(req)
        keep = []

        def arr(a, w, f):
            if a is None or len(a) == 0:
                return 0, None
            a = f(a).reshape(-1, w)
            keep.append(a)
            return len(a), a.ctypes.data_as(N.IP if f is _i else N.DP)

        ng = _i(neighs)
        bkl = _d(bond_kl).reshape(n, 8)
        na, pa = arr(angs, 3, _i)
        _, ppa = arr(angp, 5, _d)
        nd, pd = arr(dihs, 4, _i)
        _, ppd = arr(dihp, 3, _d)
        ni, pi = arr(invs, 4, _i)
        _, ppi = arr(invp, 4, _d)
        desc = N.SmrTopologyDesc(n, req.ctypes.data_as(N.DP), ng.ctypes.data_as(N.IP), bkl.ctypes.data_as(N.DP),
                                 na, pa, ppa, nd, pd, ppd, ni, pi, ppi)
        tid = C.c_int()
        self._chk(self.L.smr_add_topology(self.h, C.byref(desc), C.byref(tid)), "smr_add_topology")
        self.topo_n.append(n)
        return tid.value

    def topology(self, tid):
        c = (C.c_int * 6)()
        self._chk(self.L.smr_topology_counts(self.h, tid, c), "smr_topology_counts")
        out = _export_arrays(list(c)[:5])
        self._chk(self.L.smr_topology_export(self.h, tid, *_export_ptrs(out)), "smr_topology_export")
        out["types"] = [type_name(t) for t in out["type_id"]]
        out["rounds"] = c[5]
        return out

    # -- systems
    def add_systems(self, topo_ids, positions) -> np.ndarray:
        topo_ids = _i(topo_ids)
        if len(positions) != len(topo_ids):
            raise ValueError(f"{len(topo_ids)} topology ids but {len(positions)} position arrays")
        for t, p in zip(topo_ids, positions):       # the C call reads natoms x 3 floats per system
            if 0 <= int(t) < len(self.topo_n) and np.asarray(p).size != 3 * self.topo_n[int(t)]:
                raise ValueError(f"topology {int(t)} has {self.topo_n[int(t)]} atoms, positions have {np.asarray(p).size // 3}")
        if len(topo_ids) == 0:
            return np.zeros(0, np.int32)
        pos = _f(np.concatenate([np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in positions]))
        slots = np.zeros(len(topo_ids), np.int32)
        self._chk(self.L.smr_add_systems(self.h, len(topo_ids), _p(topo_ids, N.IP), _p(pos, N.FP), _p(slots, N.IP)),
                  "smr_add_systems")
        for s, t in zip(slots, topo_ids):
            self.natoms_of[int(s)] = self.topo_n[int(t)]
        self._nat[slots] = np.asarray(self.topo_n, np.int64)[topo_ids]
        return slots

    upload_state_multi = add_systems

    def remove_systems(self, slots):
        slots = _i(slots)
        self._chk(self.L.smr_remove_systems(self.h, len(slots), _p(slots, N.IP)), "smr_remove_systems")
        for s in slots:
            self.natoms_of.pop(int(s), None)
        self._nat[slots] = 0

    def _count(self, slots):
        """Total atoms of the slots (0 for slots not active on this handle)."""
        ok = (slots >= 0) & (slots < len(self._nat))
        return int(self._nat[slots[ok]].sum())

    def set_positions(self, slots, positions):
        """positions: one (n, 3) array per slot, or one stacked array ((nsys, n, 3) or (atoms, 3)) in
        slot order."""
        slots = _i(slots)
        if isinstance(positions, np.ndarray) and positions.ndim >= 2 and positions.shape[-1] == 3:
            flat = _f(positions.reshape(-1, 3))
            if flat.shape[0] != self._count(slots):
                raise ValueError(f"{flat.shape[0]} positions for {self._count(slots)} atoms in {len(slots)} slots")
            if len(slots):
                self._chk(self.L.smr_set_positions(self.h, len(slots), _p(slots, N.IP), _p(flat, N.FP)), "smr_set_positions")
            return
        if len(positions) != len(slots):
            raise ValueError(f"{len(slots)} slots but {len(positions)} position arrays")
        for s, p in zip(slots, positions):           # the C call reads natoms x 3 floats per slot
            n = self.natoms_of.get(int(s))
            if n is not None and np.asarray(p).size != 3 * n:
                raise ValueError(f"slot {int(s)} has {n} atoms, positions have {np.asarray(p).size // 3}")
        if len(slots) == 0:
            return
        pos = _f(np.concatenate([np.asarray(p).reshape(-1, 3) for p in positions]))
        self._chk(self.L.smr_set_positions(self.h, len(slots), _p(slots, N.IP), _p(pos, N.FP)), "smr_set_positions")

    def reset_fire(self, slots):
        slots = _i(slots)
        self._chk(self.L.smr_reset_fire(self.h, len(slots), _p(slots, N.IP)), "smr_reset_fire")

    def _split(self, slots, flat, w):
        nat = self._nat[slots] if len(slots) else np.zeros(0, np.int64)
        if len(slots) and (nat == nat[0]).all():      # all systems alike: one (nsys, n, w) array
            return flat.reshape(len(slots), int(nat[0]), w) if w > 1 else flat.reshape(len(slots), int(nat[0]))
        out, k = [], 0
        for s in slots:
            n = self.natoms_of[int(s)]
            out.append(flat[k:k + n].reshape(n, w) if w > 1 else flat[k:k + n])
            k += n
        return out

    def eval_forces(self, slots):
        """One force evaluation: list of (n, 4) float32 arrays (fx, fy, fz, E_atom), energies (nsys, 8)."""
        slots = _i(slots)
        tot = self._count(slots)
        F = np.zeros((tot, 4), np.float32)
        E = np.zeros((len(slots), 8))
        self._chk(self.L.smr_eval_forces(self.h, len(slots), _p(slots, N.IP), _p(F, N.FP), _p(E, N.DP)),
                  "smr_eval_forces")
        return self._split(slots, F, 4), E

    def run_fire(self, max_steps, step_budget=0, mode=MODE_BATCHED, **fire) -> int:
        p = fire_params(**fire)
        nf = C.c_int()
        self._chk(self.L.smr_run_fire(self.h, int(max_steps), int(step_budget), C.byref(p), mode, C.byref(nf)),
                  "smr_run_fire")
        return nf.value

    step_multi = run_fire

    def download(self, slots, pos=True, forces=True):
        slots = _i(slots)
        tot = self._count(slots)
        P = np.zeros((tot, 3), np.float32) if pos else None
        F = np.zeros((tot, 4), np.float32) if forces else None
        E = np.zeros((len(slots), 8))
        steps = np.zeros(len(slots), np.int32)
        status = np.zeros(len(slots), np.int32)
        self._chk(self.L.smr_download(self.h, len(slots), _p(slots, N.IP), _p(P, N.FP), _p(F, N.FP), _p(E, N.DP),
                                      _p(steps, N.IP), _p(status, N.IP)), "smr_download")
        return dict(pos=self._split(slots, P, 3) if pos else None, forces=self._split(slots, F, 4) if forces else None,
                    energy=E[:, 0], steps=steps, status=status)

    def download_pos64(self, slots):
        """Positions at full precision (float + its accumulated rounding error), list of (n, 3) float64."""
        slots = _i(slots)
        tot = self._count(slots)
        P = np.zeros((tot, 3), np.float64)
        self._chk(self.L.smr_download_pos64(self.h, len(slots), _p(slots, N.IP), _p(P, N.DP)), "smr_download_pos64")
        return self._split(slots, P, 3)

    def download_pos_multi(self, slots):
        return self.download(slots, pos=True, forces=False)["pos"]

    def download_pos_replica(self, slot):
        return self.download([slot], pos=True, forces=False)["pos"][0]

    def last_timing(self):
        ms = C.c_double()
        n = C.c_longlong()
        self._chk(self.L.smr_last_timing(self.h, C.byref(ms), C.byref(n)), "smr_last_timing")
        return ms.value, n.value

    def active_slots(self):
        n = C.c_int()
        self.L.smr_active_slots(self.h, C.byref(n), None)
        ids = np.zeros(n.value, np.int32)
        self.L.smr_active_slots(self.h, C.byref(n), _p(ids, N.IP))
        return ids
