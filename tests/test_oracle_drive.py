"""The driving terms of the MD update in the FP64 oracle (updateAtomsMMFFf4, opencl/UFF.cl:974-991):
the Langevin drive's hashed noise against an independent restatement, bit for bit; the driven
relaxation with no drive is the plain one; constraint springs and a fixed-seed drive end in
force balance."""
import math

import numpy as np
import pytest

from surfmol_b200 import synth

KB = 8.617333262145e-5


def noise_restated(ia, seed):
    """UFF.cl:982-989 with Python integers for the 64-bit hash and numpy float32 for the kernel's FP32
    sum and product; the sine in FP64."""
    f = np.float32
    seed = f(seed)
    out = []
    for c, m in ((136, 1000.0), (778, 1013.0), (4578, 998.0)):
        x = ia + c + int(f(m) * seed)                   # (int) truncates toward zero
        r = f((x * 2654435761) >> 16 & 0xFF) * f(0.00390625)
        out.append(math.sin(float((r + seed) * f(124.4565))))
    return out


@pytest.mark.parametrize("seed", [0.0, 2.5, -7.3, 123.456, 1000.0])
def test_noise_matches_restatement(oracle, seed):
    got = oracle.langevin_noise(600, seed)
    ref = np.array([noise_restated(i, seed) for i in range(600)])
    assert np.array_equal(got, ref)
    assert np.abs(got).max() <= 1.0 and got.std() > 0.3


def test_undriven_is_plain_relaxation(oracle):
    rng = np.random.default_rng(2)
    m = synth.polyaromatic_40(rng)
    P = m.pos + rng.normal(0, 0.05, m.pos.shape)
    S = oracle.System.from_molecule(m.Z, P, synth.charges(rng, m.n))
    a = S.relax(P, None, max_steps=80, fconv=1e-9)
    b = S.relax_drive(P, None, max_steps=80, tdrive=(100.0, 0.0, 0.0, 3.0), fconv=1e-9)
    assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["F"], b["F"])


def test_springs_and_fixed_seed_drive_balance(oracle):
    """At convergence the velocity is ~0, so the physical force balances the springs plus the constant
    noise pattern times one amplitude, sqrt(2 kB T gamma / dt) at the final FIRE dt: the fitted
    amplitude implies a dt within [dt0, dt_max] and leaves a residual of the size the last move
    makes (positions advance once more on the converging step, main.rs:270-275), well below the
    load itself."""
    rng = np.random.default_rng(3)
    m = synth.polyaromatic_40(rng)
    P = m.pos + rng.normal(0, 0.05, m.pos.shape)
    S = oracle.System.from_molecule(m.Z, P, synth.charges(rng, m.n))
    atoms = np.array([0, 11, 27])
    target = P[atoms] + [[0.3, 0.0, 0.1], [0.0, 0.2, -0.1], [-0.2, 0.0, 0.2]]
    k = np.array([[3.0, 3.0, 3.0], [0.0, 5.0, 2.0], [4.0, -1.0, 4.0]])
    T, gamma, seed = 20.0, 0.05, 1.75
    r = S.relax_drive(P, None, max_steps=20000, cons=(atoms, target, k), tdrive=(T, gamma, 0.0, seed),
                      fconv=1e-4, dt0=1e-3, dt_max=0.05)
    assert r["conv"]
    F, _, _ = S.eval(r["pos"])
    springs = np.zeros_like(F)
    springs[atoms] = (target - r["pos"][atoms]) * np.maximum(k, 0.0)
    noise = oracle.langevin_noise(m.n, seed)
    amp = -np.sum(noise * (F + springs)) / np.sum(noise * noise)
    assert np.abs(F + springs + amp * noise).max() < 3e-3
    assert np.abs(F + springs).max() > 2e-2                           # without the load no balance
    dt = 2 * KB * float(np.float32(T)) * float(np.float32(gamma)) / amp ** 2
    assert 1e-3 <= dt <= 0.05 * 1.01, dt                               # the fit carries the residual
    assert np.abs(springs).max() > 1e-2 and amp * np.abs(noise).max() > 2e-2
