"""Multi-replica rigid-atom relaxation (RAFF / RRsp3) over the C ABI of include/surfmol_raff.h.

``RaffMulti`` mirrors the reference's RRsp3Multi harness (crates/libs/oclff/src/rrsp3.rs:699-1088):
the same method names, argument layouts and step configuration, so a caller of the OpenCL harness
switches by changing the constructor.  ``prepare`` does the host preparation of
crates/libs/oclff/src/pack.rs for one molecule (nodes-first order, neighbours, exclusions,
back-slots, ports, masses) through the library's native builders.  All numerics run in the CUDA
library; this module marshals arrays.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N

# StepConfig defaults (rrsp3.rs:67-73)
STEP_DEFAULT = dict(dt=0.1, k_coll=50.0, relaxation=0.5, momentum_beta=0.0, rot_mass_scale=1.0)


class RaffError(RuntimeError):
    pass


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


@dataclass
class Prepared:
    """One molecule laid out for the multi-replica harness (pack.rs layout, one group)."""
    perm: np.ndarray          # packed atom k = input atom perm[k]
    nnode: int
    Z: np.ndarray             # packed order
    pos: np.ndarray           # (natoms, 3) float32, packed order
    bonds: np.ndarray         # (nbonds, 2) packed indices
    neighs: np.ndarray        # (natoms, 4)
    excl1: np.ndarray
    excl2: np.ndarray
    bk_slots: np.ndarray      # (natoms, 4)
    port_local: np.ndarray    # (natoms, 4, 4)
    k: np.ndarray             # (natoms, 4)
    inv_mass: np.ndarray      # (natoms,)

    @property
    def natoms(self):
        return len(self.Z)


def _chk(r, what):
    if r < 0:
        raise RaffError(f"{what} failed ({r})")
    return r


def prepare(Z, pos, bonds, k_stiff=200.0) -> Prepared:
    """Host preparation of one molecule as raff_ocl_benchmark does it (pack.rs): nodes (bond degree
    > 1) first, neighbours from the bonds, 1st / 2nd exclusions, ports along the initial bond
    vectors with stiffness k_stiff, back-slots, inverse masses from the elements."""
    L = N.lib()
    Z = _i(Z)
    n = len(Z)
    pos = _f(np.asarray(pos).reshape(n, 3))
    b = _i(np.asarray(bonds).reshape(-1, 2))
    perm = np.zeros(n, np.int32)
    nnode = _chk(L.smr_raff_node_order(n, len(b), _p(b, N.IP), _p(perm, N.IP)), "smr_raff_node_order")
    inv = np.empty(n, np.int32)
    inv[perm] = np.arange(n, dtype=np.int32)
    bp = _i(inv[b]) if len(b) else _i(np.zeros((0, 2)))
    Zp, Pp = _i(Z[perm]), _f(pos[perm])
    neighs = np.zeros((n, 4), np.int32)
    _chk(L.smr_raff_build_neighs(n, len(bp), _p(bp, N.IP), _p(neighs, N.IP)), "smr_raff_build_neighs (degree > 4?)")
    e1 = np.zeros((n, 4), np.int32)
    e2 = np.zeros((n, 4), np.int32)
    _chk(L.smr_raff_exclusions(n, _p(neighs, N.IP), _p(e1, N.IP), _p(e2, N.IP)), "smr_raff_exclusions")
    bk = np.zeros((n, 4), np.int32)
    _chk(L.smr_raff_bk_slots(n, nnode, _p(neighs, N.IP), _p(bk, N.IP)), "smr_raff_bk_slots")
    pl = np.zeros((n, 4, 4), np.float32)
    kk = np.zeros((n, 4), np.float32)
    _chk(L.smr_raff_ports(n, _p(Pp, N.FP), _p(neighs, N.IP), float(k_stiff), _p(pl, N.FP), _p(kk, N.FP)), "smr_raff_ports")
    inv_mass = np.array([1.0 / L.smr_raff_element_mass(int(z)) for z in Zp], np.float32)
    return Prepared(perm, nnode, Zp, Pp, bp, neighs, e1, e2, bk, pl, kk, inv_mass)


class RaffMulti:
    """nsys replicas of one molecule (natoms atoms each), relaxed on one GPU (RRsp3Multi)."""

    def __init__(self, natoms: int, nsys: int, device: int = 0):
        self.L = N.lib()
        cfg = N.SmrRaffConfig(device, int(natoms), int(nsys))
        h = N.VP()
        r = self.L.smr_raff_create(C.byref(cfg), C.byref(h))
        if r != 0:
            raise RaffError(f"smr_raff_create failed ({r}): CUDA device {device} unavailable, or natoms outside [1, 1024]")
        self.h = h
        self.natoms, self.nsys = int(natoms), int(nsys)
        self.nnode = 0

    def finish(self):
        if self.h:
            self.L.smr_raff_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.finish()
        except Exception:
            pass

    def _chk(self, r, what):
        if r != 0:
            raise RaffError(f"{what} ({r}): {self.L.smr_raff_last_error(self.h).decode()}")

    # -- uploads (RRsp3Multi names)
    def upload_radius(self, radius):
        self._chk(self.L.smr_raff_upload_radius(self.h, _p(_f(radius), N.FP)), "upload_radius")

    def upload_neighs_and_exclusions(self, neighs, excl1, excl2):
        a, b, c = (_i(np.asarray(x).reshape(-1)) for x in (neighs, excl1, excl2))
        self._chk(self.L.smr_raff_upload_neighs_and_exclusions(self.h, _p(a, N.IP), _p(b, N.IP), _p(c, N.IP)),
                  "upload_neighs_and_exclusions")

    def upload_fixmask(self, fixmask):
        self._chk(self.L.smr_raff_upload_fixmask(self.h, _p(_i(fixmask), N.IP)), "upload_fixmask")

    def upload_cluster_ports_multi(self, port_local, k, nnode):
        pl, kk = _f(np.asarray(port_local).reshape(-1)), _f(np.asarray(k).reshape(-1))
        self._chk(self.L.smr_raff_upload_cluster_ports(self.h, _p(pl, N.FP), _p(kk, N.FP), int(nnode)),
                  "upload_cluster_ports_multi")
        self.nnode = int(nnode)

    def upload_bk_slots_multi(self, bk_slots):
        self._chk(self.L.smr_raff_upload_bk_slots(self.h, _p(_i(np.asarray(bk_slots).reshape(-1)), N.IP)),
                  "upload_bk_slots_multi")

    def upload_state_multi(self, pos3, inv_mass, quat=None):
        p = _f(np.asarray(pos3).reshape(-1))
        q = None if quat is None else _f(np.asarray(quat).reshape(-1))
        self._chk(self.L.smr_raff_upload_state(self.h, _p(p, N.FP), _p(_f(inv_mass), N.FP), _p(q, N.FP)),
                  "upload_state_multi")

    def upload_prepared(self, prep: Prepared, pos3, radius=None, fixmask=None, quat=None):
        """Everything raff_ocl_benchmark uploads, from ``prepare``'s output; pos3 (nsys, natoms, 3)
        in packed order."""
        self.upload_radius(np.zeros(prep.natoms) if radius is None else radius)
        self.upload_neighs_and_exclusions(prep.neighs, prep.excl1, prep.excl2)
        self.upload_cluster_ports_multi(prep.port_local[:prep.nnode], prep.k[:prep.nnode], prep.nnode)
        self.upload_bk_slots_multi(prep.bk_slots)
        if fixmask is not None:
            self.upload_fixmask(fixmask)
        self.upload_state_multi(pos3, prep.inv_mass, quat)

    # -- stepping
    def step_cluster_multi(self, nsteps=1, **cfg):
        """nsteps steps (the reference's step_cluster_multi repeated), all in one launch."""
        p = dict(STEP_DEFAULT)
        p.update(cfg)
        c = N.SmrRaffStepConfig(p["dt"], p["k_coll"], p["relaxation"], p["momentum_beta"], p["rot_mass_scale"])
        self._chk(self.L.smr_raff_step(self.h, int(nsteps), C.byref(c)), "step_cluster_multi")

    def last_ms(self):
        v = C.c_float()
        self._chk(self.L.smr_raff_last_ms(self.h, C.byref(v)), "smr_raff_last_ms")
        return v.value

    # -- downloads
    def _rows(self, fn, isys, rows, w):
        out = np.zeros(((self.nsys if isys < 0 else 1) * rows, w), np.float32)
        self._chk(getattr(self.L, fn)(self.h, int(isys), _p(out, N.FP)), fn)
        return out.reshape(-1, rows, w) if isys < 0 else out

    def download_pos_multi(self):
        return self._rows("smr_raff_download_pos", -1, self.natoms, 3)

    def download_pos_replica(self, isys):
        return self._rows("smr_raff_download_pos", isys, self.natoms, 3)

    def download_quat_replica(self, isys):
        return self._rows("smr_raff_download_quat", isys, self.natoms, 4)

    def download_quat_multi(self):
        return self._rows("smr_raff_download_quat", -1, self.natoms, 4)

    def download_dpos_coll_replica(self, isys):
        return self._rows("smr_raff_download_dpos_coll", isys, self.natoms, 3)

    def download_dpos_node_replica(self, isys):
        return self._rows("smr_raff_download_dpos_node", isys, self.nnode, 3)
