"""Generate tests/golden/ref_kernels.json: seeded inputs and the outputs of the reference's own
OpenCL kernels, compiled for the host as oracle/_ref (oracle/ref_gen.py + oracle/ref_cl.h).

Run where the reference tree is present:
    SURFMOL_REFERENCE=<reference root> python tests/golden/make_ref_fixtures.py
The JSON is committed, so tests/test_oracle_ref_pin.py checks the FP64 oracle against these
reference outputs without the reference tree.  Cases (reference file:line):
  ljqh       getLJQH + mixREQ_arithmetic            opencl/UFF.cl:57-95
  sample     fe3d_pbc_comb and its PBC index tables  opencl/UFF.cl:1384-1511
  nb_grid    getNonBond_GridFF_Bspline              opencl/UFF.cl:1524-1718
  nb_ex2     getNonBond_GridFF_Bspline_ex2          opencl/UFF.cl:1722-
  morse      make_MorseFF                           opencl/gridff_build.cl:217-347
  conv       BsplineConv3D                          opencl/gridff_build.cl:8-61
  ewald      eval_potential_full                    opencl/Surface.cl:716-767, 834-906
  brute      eval_potential_brute                   opencl/Surface.cl:911-954
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def _short(x):
    """The shortest decimal that reads back as the same float32."""
    return float(np.format_float_scientific(np.float32(x), unique=True))


def L(a):
    """float32 values as JSON lists; each reads back as exactly the same float32."""
    a = np.asarray(a)
    if a.dtype.kind == "f":
        return np.vectorize(_short, otypes=[float])(a).tolist()
    return a.tolist()


def main():
    from oracle import ref as R
    from surfmol_b200 import synth
    if not R.available():
        print("oracle/_ref is not built and the reference tree is absent", file=sys.stderr)
        return 2
    rng = np.random.default_rng(20261204)
    out = {"source": "outputs of the reference's OpenCL kernels built for the host (oracle/_ref), FP32"}
    # getLJQH on mixed parameters
    n = 48
    reqi = np.c_[rng.uniform(1.4, 2.0, n), np.sqrt(rng.uniform(1e-3, 1e-2, n)), rng.normal(0, 0.3, n), rng.uniform(-.9, .9, n)]
    reqj = np.c_[rng.uniform(1.4, 2.0, n), np.sqrt(rng.uniform(1e-3, 1e-2, n)), rng.normal(0, 0.3, n), rng.uniform(-.9, .9, n)]
    mix = R.mix_req(reqi, reqj)
    dp = rng.normal(0, 3.0, (n, 3)).astype(np.float32)
    out["ljqh"] = {"reqi": L(reqi), "reqj": L(reqj), "mixed": L(mix), "dp": L(dp), "rdamp": 1.0,
                   "out": L(R.ljqh(dp, mix, 1.0))}
    # the sampler, with points across the periodic x / y wraps and both z bounds
    g = rng.normal(size=(6, 5, 9, 4)).astype(np.float32)
    u = np.c_[rng.uniform(-2, 8, 64), rng.uniform(-2, 7, 64), rng.uniform(-0.5, 9.5, 64)].astype(np.float32)
    plqh = rng.normal(size=(64, 4)).astype(np.float32)
    out["sample"] = {"grid": L(g), "u": L(u), "plqh": L(plqh), "out": L(R.sample(g, u, plqh))}
    # NB + grid on a built substrate grid, two placements of the 40-atom molecule
    from oracle import oracle as O
    slab = synth.rocksalt_slab(1, 2)
    dims, p0 = (14, 14, 24), (0.0, 0.0, slab.z_top + 1.0)
    step = (slab.Lx / 14, slab.Ly / 14, 0.25)
    coef = O.build_grid_fast(slab.ions, slab.req(), slab.Lx, slab.Ly, *dims, p0, step).astype(np.float32)
    m = synth.polyaromatic_40(np.random.default_rng(1))
    q = synth.charges(rng, m.n)
    P = [synth.place(rng, m, (rng.uniform(0, slab.Lx), rng.uniform(0, slab.Ly)), h) for h in (2.4, 3.6)]
    S = O.System.from_molecule(m.Z, P[0], q)
    e = S.export()
    A = np.zeros((2, m.n, 4), np.float32)
    A[:, :, :3] = np.array(P)
    Rq = np.tile(e["req"].astype(np.float32), (2, 1, 1))
    Ng = np.tile(e["neighs"].astype(np.int32), (2, 1, 1))
    X = np.tile(R.second_neighs(e["neighs"]), (2, 1, 1))
    common = {"grid": L(coef), "p0": list(p0), "step": [float(s) for s in step], "atoms": L(A), "req": L(e["req"]),
              "neighs": L(e["neighs"]), "bonds": L(e["bonds"]), "rdamp": 1.0, "alpha": 1.5}
    out["nb_grid"] = dict(common, out=L(R.nb_grid(A, Rq, Ng, coef, p0, step)))
    out["nb_ex2"] = {"excl": L(X[0]), "out": L(R.nb_grid_ex2(A, Rq, X, coef, p0, step))}
    # Morse over a 2x2-cell slab, 16 x 16 x 8 points of a 2.4 A high cell
    s2 = synth.rocksalt_slab(2, 2)
    lvec = np.diag([s2.Lx, s2.Ly, 2.4])
    Pm, Lm = R.morse(np.c_[s2.ions[:, :3], np.zeros(len(s2.ions))], s2.req(), lvec, (16, 16, 8), (0.0, 0.0, 1.0))
    out["morse"] = {"ions": L(s2.ions), "req": L(s2.req()), "Lx": s2.Lx, "Ly": s2.Ly, "ngrid": [16, 16, 8], "p0": [0, 0, 1.0],
                    "cz": 2.4, "npbc": 1, "alpha": 1.5, "paul": L(Pm), "lond": L(Lm)}
    # BsplineConv3D (x fastest)
    c = rng.normal(size=(5, 6, 7)).astype(np.float32)
    out["conv"] = {"coef_xfast": L(c), "out": L(R.bspline_conv(c))}
    # Ewald-2D and the direct image sum
    pts = np.c_[rng.uniform(0, s2.Lx, 12), rng.uniform(0, s2.Ly, 12), rng.uniform(1.0, 6.0, 12)]
    out["ewald"] = {"pts": L(pts), "ions": L(s2.ions), "Lx": s2.Lx, "Ly": s2.Ly, "gcut": 6.0,
                    "phi": L(R.ewald_full(pts, s2.ions, s2.Lx, s2.Ly, 6.0))}
    out["brute"] = {"nrep": 10, "phi": L(R.coulomb_brute(pts, s2.ions, s2.Lx, s2.Ly, 10))}
    with open(os.path.join(HERE, "ref_kernels.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    return 0


if __name__ == "__main__":
    sys.exit(main())
