"""Folded-surface substrate: the reference's SurfaceFolded model (crates/libs/surfff/src/lib.rs:
126-351), a drop-in alternative to the B-spline grid.

The potential of one atom is a separable sum over basis functions
``cos(2 pi kx[ix] u) * cos(2 pi ky[iy] v) * exp(-kz[iz] (z - z0[iz]))`` with ``(u, v)`` the atom's
fractional coordinates in the 2D lattice, weighted per basis function by ``cq * Q + cp * P + cl * L``
(the atom's charge and its Pauli / London prefactors, NonBondedFF::make_plqs,
crates/libs/molff/src/nonbonded.rs:98-108).  The force on an atom is clamped to ``fmax`` as
MolWorld::eval_forces does (crates/libs/surfmol/src/mol_world.rs:80-83, 100 eV/A).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class FoldedSurface:
    ax: float
    bx: float
    ay: float
    by: float
    kx: np.ndarray
    ky: np.ndarray
    kz: np.ndarray
    z0: np.ndarray
    cq: np.ndarray = field(default=None)
    cp: np.ndarray = field(default=None)
    cl: np.ndarray = field(default=None)
    alpha: float = 2.0          # make_plqs exponent (molengine: 2.0)
    fmax: float = 100.0         # per-atom force clamp (eV/A)

    def __post_init__(self):
        self.kx, self.ky, self.kz, self.z0 = (np.asarray(x, np.float64) for x in (self.kx, self.ky, self.kz, self.z0))
        nb = self.nbasis
        for name in ("cq", "cp", "cl"):
            v = getattr(self, name)
            setattr(self, name, np.zeros(nb) if v is None else np.asarray(v, np.float64).reshape(nb))

    @property
    def nbasis(self):
        return len(self.kx) * len(self.ky) * len(self.kz)

    def set_coeffs(self, ib, q, p, l):
        self.cq[ib], self.cp[ib], self.cl[ib] = q, p, l

    def as_dict(self):
        return dict(ax=self.ax, bx=self.bx, ay=self.ay, by=self.by, kx=self.kx, ky=self.ky, kz=self.kz, z0=self.z0,
                    cq=self.cq, cp=self.cp, cl=self.cl, alpha=self.alpha, fmax=self.fmax)


def nacl(a=5.66, z0=0.0, beta_charge=0.3, beta_morse_ratio=2.0, q_amp=1.0, plq_amp=1.0) -> FoldedSurface:
    """The NaCl-like folded surface of setup_nacl_surface (crates/libs/surfff/src/lib.rs:364-412):
    z decays 2 b_m (Pauli), b_m (London), b_q (charge) with b_m = ratio * b_q; harmonics 0 and 1 in x
    and y; a constant Pauli term (x40, giving a minimum ~1.5 A above the plane), a constant London
    term and a checkerboard charge term.  Defaults: the editor's constants (apps/editor/src/main.rs:52-57)."""
    bm = beta_charge * beta_morse_ratio
    s = FoldedSurface(a, 0.0, 0.0, a, [0.0, 1.0], [0.0, 1.0], [2.0 * bm, bm, beta_charge], [z0, z0, z0])
    nx, ny = 2, 2
    for iz in range(3):
        const, check = iz * nx * ny + 0, iz * nx * ny + 1 + nx * 1
        if iz == 0:
            s.set_coeffs(const, 0.0, plq_amp * 40.0, 0.0)
        elif iz == 1:
            s.set_coeffs(const, 0.0, 0.0, -plq_amp)
        else:
            s.set_coeffs(check, q_amp, 0.0, 0.0)
    return s
