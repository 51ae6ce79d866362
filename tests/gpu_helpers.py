"""Shared set-up for the GPU parity tests."""
import numpy as np

from surfmol_b200 import synth

# per-atom force parity bar: |dF| <= 1e-4 eV/A relative to max(1, max|F|)
F_RTOL = 1e-4


def small_slab_grid(ncell=1, nlayers=2, nxy=28, nz=48, dz=0.2, z_gap=1.0):
    slab = synth.rocksalt_slab(ncell, nlayers)
    step = (slab.Lx / nxy, slab.Ly / nxy, dz)
    p0 = (0.0, 0.0, slab.z_top + z_gap)
    return slab, (nxy, nxy, nz), p0, step


def build_device_grid(R, slab, dims, p0, step, alpha=1.5, dtype=0):
    R.build_grid(slab.ions, slab.req()[:, :2], slab.Lx, slab.Ly, dims[0], dims[1], dims[2], p0, step,
                 alpha_morse=alpha, npbc=1, ewald_tol=1e-12, dtype=dtype)
    return R.get_grid()


def decode(g):
    """Host decode of a downloaded grid to float64 values (stored * scale)."""
    c = g["coef"]
    if g["dtype"] == 0:
        return c.astype(np.float64)
    if g["dtype"] == 1:
        v = c.view(np.float16).astype(np.float64)
    else:
        v = (c.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    ps = g.get("plane_scale")
    if ps is not None:
        return v * ps.astype(np.float64)[None, None, :, :]
    return v * g["scale"][None, None, None, :]


def force_err(Fg, Fo):
    return np.abs(np.asarray(Fg, float)[:, :3] - Fo).max() / max(1.0, np.abs(Fo).max())


def molecule_on_slab(rng, n, slab, height=3.0):
    m = synth.ragged_molecule(rng, n) if n != 40 else synth.polyaromatic_40(rng)
    p = synth.place(rng, m, (rng.uniform(0, slab.Lx), rng.uniform(0, slab.Ly)), height, z_top=slab.z_top)
    return m.Z, p, synth.charges(rng, m.n)
