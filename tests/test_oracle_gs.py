"""Known-answer and property tests of the oracle's ground-state pieces
(CG eigensolver, preconditioner, Gram-Schmidt, subspace diagonalisation)."""
import functools

import numpy as np

from oracle import Oracle
from salmon2_b200 import synth


@functools.lru_cache(maxsize=None)
def real_system():
    return synth.isolated_system(num=20, no=6, natom=2, seed=21, real=True, name="gs20")


def inner(s, a, b):
    sl = s.grid.interior_slices()
    return np.sum(a[sl] * b[sl]) * s.grid.hvol


def test_gram_schmidt_real_orthonormal():
    s = real_system()
    O = Oracle(s)
    rng = np.random.default_rng(0)
    psi = s.psi + 0.3 * rng.standard_normal(s.psi.shape) * (s.psi != 0)
    out = O.gram_schmidt_real(psi)
    for i in range(s.no):
        for j in range(s.no):
            v = inner(s, out[..., 0, i, 0], out[..., 0, j, 0])
            assert abs(v - (1.0 if i == j else 0.0)) < 1e-12


def test_gram_schmidt_complex_orthonormal():
    s = synth.periodic_system(a=10.26, num=12, nkgrid=1, no=4, seed=22)
    O = Oracle(s)
    rng = np.random.default_rng(1)
    psi = s.psi + 0.2 * (rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape))
    out = O.gram_schmidt_complex(psi)
    sl = s.grid.interior_slices()
    for i in range(s.no):
        for j in range(s.no):
            v = np.vdot(out[sl + (0, i, 0)], out[sl + (0, j, 0)]) * s.grid.hvol
            assert abs(v - (1.0 if i == j else 0.0)) < 1e-12


def test_subspace_diag_matches_eigh():
    s = real_system()
    O = Oracle(s)
    h = O.hpsi_real(s.psi)
    no = s.no
    M = np.array([[inner(s, s.psi[..., 0, i, 0], h[..., 0, j, 0]) for j in range(no)] for i in range(no)])
    M = 0.5 * (M + M.T)
    w = np.linalg.eigvalsh(M)
    out, ev = O.subspace_diag_real(s.psi)
    np.testing.assert_allclose(ev, w, rtol=1e-10, atol=1e-10)
    # rotated orbitals are orthonormal and diagonalise H in the subspace
    h2 = O.hpsi_real(out)
    for i in range(no):
        assert abs(inner(s, out[..., 0, i, 0], h2[..., 0, i, 0]) - w[i]) < 1e-9


def test_precond_plane_wave_symbol():
    s = synth.periodic_system(a=10.26, num=12, nkgrid=1, no=1, seed=23)
    g = s.grid
    L = g.num * g.hgs
    m = np.array([1, -2, 3])
    q = 2 * np.pi * m / L
    X, Y, Z = np.meshgrid(g.coordinate(0), g.coordinate(1), g.coordinate(2), indexing="ij")
    f = np.cos(q[0] * X + q[1] * Y + q[2] * Z)
    psi = np.zeros(g.shape_array + (1, 1, 1), order="F")
    psi[g.interior_slices() + (0, 0, 0)] = f
    O = Oracle(s)
    out = O.precond_real(psi, alpha=0.6)
    omega = 2 * (1 - 0.6)
    d = -0.5 * np.sum(-2.0 / g.hgs ** 2)
    lam = np.sum((2 * np.cos(q * g.hgs) - 2) / g.hgs ** 2)
    factor = omega / d * (2 - omega / d * (-0.5 * lam))
    np.testing.assert_allclose(out[g.interior_slices() + (0, 0, 0)], factor * f, rtol=1e-12, atol=1e-13)


def test_cg_lowers_rayleigh_quotients():
    s = real_system()
    O = Oracle(s)
    psi = O.gram_schmidt_real(s.psi)
    h = O.hpsi_real(psi)
    e0 = np.array([inner(s, psi[..., 0, i, 0], h[..., 0, i, 0]) for i in range(s.no)])
    for pre in (False, True):
        out, esp = O.gscg(psi, ncg=4, precondition=pre)
        assert np.all(esp <= e0 + 1e-12)
        assert np.sum(esp) < np.sum(e0)
        for i in range(s.no):
            assert abs(inner(s, out[..., 0, i, 0], out[..., 0, i, 0]) - 1.0) < 1e-12
