"""The oracle's folded surface against the reference's own known answers
(crates/libs/surfff/src/lib.rs:437-511) and against finite differences."""
import math

import numpy as np
import pytest

from surfmol_b200.folded import FoldedSurface, nacl

REQ = [3.0, 0.1, 0.5, 0.0]           # the reference tests' REQ (R=3, req[1]=0.1, Q=0.5)


def one_basis(kx, ky, kz, z0, q=0.0, p=0.0, l=0.0):
    s = FoldedSurface(10.0, 0.0, 0.0, 10.0, [kx], [ky], [kz], [z0])
    s.set_coeffs(0, q, p, l)
    return s


def test_constant_basis(oracle):          # lib.rs:437-456
    f = oracle.Folded(**one_basis(0.0, 0.0, 0.0, 0.0, q=1.0).as_dict())
    E, F = f.points([[3.0, 4.0, 1.0]], [REQ])
    assert abs(E[0] - 0.5) < 1e-10 and np.abs(F).max() < 1e-10


def test_cos_x(oracle):                   # lib.rs:459-482
    f = oracle.Folded(**one_basis(1.0, 0.0, 0.0, 0.0, q=1.0).as_dict())
    req = [[3.0, 0.1, 1.0, 0.0]] * 3
    E, _ = f.points([[0.0, 0.0, 0.0], [5.0, 0.0, 0.0], [2.5, 0.0, 0.0]], req)
    assert abs(E[0] - 1.0) < 1e-10 and abs(E[1] + 1.0) < 1e-10 and abs(E[2]) < 1e-10


def test_z_decay(oracle):                 # lib.rs:485-501
    f = oracle.Folded(**one_basis(0.0, 0.0, 1.0, 0.0, q=1.0).as_dict())
    E, _ = f.points([[0.0, 0.0, 1.0]], [[3.0, 0.1, 1.0, 0.0]])
    assert abs(E[0] - math.exp(-1.0)) < 1e-10


def test_req2plq(oracle):                 # lib.rs:504-511: P = e^2 sqrt(req1), L = e sqrt(req1), e = exp(-2 R)
    e = math.exp(-6.0)
    for c, want in (("p", e * e * math.sqrt(0.1)), ("l", e * math.sqrt(0.1))):
        f = oracle.Folded(**one_basis(0.0, 0.0, 0.0, 0.0, **{c: 1.0}).as_dict(), )
        E, _ = f.points([[1.0, 1.0, 1.0]], [REQ])
        assert abs(E[0] - want) < 1e-15


@pytest.mark.parametrize("alpha", [2.0, 1.5])
def test_forces_are_gradients(oracle, alpha):
    s = nacl()
    s.alpha = alpha
    f = oracle.Folded(**s.as_dict())
    rng = np.random.default_rng(3)
    pos = np.column_stack([rng.uniform(0, 11, 20), rng.uniform(0, 11, 20), rng.uniform(1.2, 6.0, 20)])
    req = np.column_stack([rng.uniform(1.4, 2.0, 20), rng.uniform(0.03, 0.08, 20), rng.normal(0, 0.2, 20), np.zeros(20)])
    E, F = f.points(pos, req)
    h = 1e-6
    for k in range(3):
        d = np.zeros(3); d[k] = h
        Ep, _ = f.points(pos + d, req)
        Em, _ = f.points(pos - d, req)
        assert np.abs(-(Ep - Em) / (2 * h) - F[:, k]).max() < 1e-6


def test_force_clamp(oracle):
    s = nacl()
    E, F0 = oracle.Folded(**s.as_dict()).points([[0.3, 0.2, 0.4]], [[1.9, 0.07, 0.1, 0.0]])
    s.fmax = 0.5 * np.linalg.norm(F0[0])
    E, F = oracle.Folded(**s.as_dict()).points([[0.3, 0.2, 0.4]], [[1.9, 0.07, 0.1, 0.0]])
    assert abs(np.linalg.norm(F[0]) - s.fmax) < 1e-12
    assert np.abs(F[0] / np.linalg.norm(F[0]) - F0[0] / np.linalg.norm(F0[0])).max() < 1e-12
