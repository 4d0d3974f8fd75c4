"""GPU parity of the ground-state path (real orbitals) against the oracle:
real hpsi, the CG eigensolver (with and without the low-pass
preconditioner), classical Gram-Schmidt (real, and complex as the RT path
calls it) and the subspace diagonalisation."""
import functools

import numpy as np
import pytest

import _systems as S
from oracle import Oracle
from salmon2_b200 import synth

pytestmark = pytest.mark.gpu


@functools.lru_cache(maxsize=None)
def gs_system():
    return synth.isolated_system(num=24, no=6, natom=2, seed=41, real=True, name="gs24")


def _ctx(s):
    from salmon2_b200.rt import Context
    return Context(s)


def test_hpsi_real_parity():
    s = gs_system()
    O = Oracle(s)
    ref = O.hpsi_real(s.psi)
    ctx = _ctx(s)
    t = ctx.gs_upload(s.psi)
    h = ctx.gs_empty()
    ctx.hpsi_real(t, h)
    assert S.rel_err(ctx.gs_download(h), ref) < 1e-12


def test_gs_relayout_round_trip():
    s = gs_system()
    ctx = _ctx(s)
    assert np.array_equal(ctx.gs_download(ctx.gs_upload(s.psi)), s.psi)


@pytest.mark.parametrize("pre", ["none", "lowpass"])
def test_gscg_parity(pre):
    s = gs_system()
    O = Oracle(s)
    psi0 = O.gram_schmidt_real(s.psi)
    ref, esp_ref = O.gscg(psi0, ncg=4, precondition=(pre == "lowpass"))
    ctx = _ctx(s)
    psi = ctx.gs_upload(psi0)
    esp = ctx.gscg(psi, ncg=4, precondition=pre)
    np.testing.assert_allclose(esp, esp_ref, rtol=1e-10, atol=1e-12)
    assert S.rel_err(ctx.gs_download(psi), ref) < 1e-9


def test_gram_schmidt_real_parity():
    s = gs_system()
    rng = np.random.default_rng(5)
    psi0 = s.psi + 0.3 * rng.standard_normal(s.psi.shape) * (s.psi != 0)
    O = Oracle(s)
    ref = O.gram_schmidt_real(psi0)
    ctx = _ctx(s)
    psi = ctx.gs_upload(psi0)
    ctx.gram_schmidt_real(psi)
    assert S.rel_err(ctx.gs_download(psi), ref) < 1e-11


def test_subspace_diag_parity():
    s = gs_system()
    O = Oracle(s)
    psi0 = O.gram_schmidt_real(s.psi)
    ref, ev_ref = O.subspace_diag_real(psi0)
    ctx = _ctx(s)
    psi = ctx.gs_upload(psi0)
    ev = ctx.subspace_diag_real(psi)
    np.testing.assert_allclose(ev, ev_ref, rtol=1e-10, atol=1e-12)
    got = ctx.gs_download(psi)
    # eigenvectors are defined up to sign; both sides fix the largest component positive
    assert S.rel_err(got, ref) < 1e-8


@pytest.mark.parametrize("make", [S.periodic_small, S.isolated_odd], ids=lambda f: f.__name__)
def test_gram_schmidt_complex_parity(make):
    """Complex column Gram-Schmidt (RT path, every (k, spin) group) against the
    oracle's gram_schmidt_col_complex8, on orbitals mixed to be far from
    orthonormal; the result is orthonormal in the hvol metric."""
    s = make()
    rng = np.random.default_rng(5)
    psi = s.psi.copy(order="F")
    no = s.no
    mix = np.eye(no) + 0.3 * (rng.standard_normal((no, no)) + 1j * rng.standard_normal((no, no)))
    psi = np.asfortranarray(np.einsum("xyzsok,op->xyzspk", psi, mix))
    ref = Oracle(s).gram_schmidt_complex(psi)
    ctx = _ctx(s)
    d = ctx.upload(psi)
    ctx.gram_schmidt_complex(d)
    out = ctx.download(d)
    assert S.rel_err(out, ref) < 1e-12
    sl = s.grid.interior_slices()
    for ik in range(s.nk):
        for isp in range(s.nspin):
            X = out[sl + (isp, slice(None), ik)].reshape(-1, no, order="F")
            np.testing.assert_allclose(X.conj().T @ X * s.grid.hvol, np.eye(no), atol=1e-12)


@pytest.mark.parametrize("no", [1, 2, 3, 37, 160], ids=lambda n: f"no{n}")
def test_subspace_diag_gpu_eigensolver(no):
    """The subspace Hamiltonian is diagonalised on the GPU (Householder
    reduction, accumulated reflections, implicit-shift QL).  Against numpy's
    eigvalsh of the same matrix built from the oracle's H: eigenvalues to
    1e-10, and the rotated orbitals are orthonormal and diagonalise H in the
    subspace (the residual ||H V - V Lambda|| checks of a dsyev result)."""
    s = synth.isolated_system(num=20, no=no, natom=2, seed=52 + no, real=True, name=f"gs20n{no}")
    O = Oracle(s)
    psi0 = O.gram_schmidt_real(s.psi)
    sl = s.grid.interior_slices()
    X = np.stack([psi0[sl + (0, i, 0)].ravel(order="F") for i in range(no)], axis=1)
    h = O.hpsi_real(psi0)
    HX = np.stack([h[sl + (0, i, 0)].ravel(order="F") for i in range(no)], axis=1)
    M = X.T @ HX * s.grid.hvol
    w_ref = np.linalg.eigvalsh(np.triu(M) + np.triu(M, 1).T)
    ctx = _ctx(s)
    psi = ctx.gs_upload(psi0)
    ev = ctx.subspace_diag_real(psi)
    np.testing.assert_allclose(ev, w_ref, rtol=1e-10, atol=1e-10 * np.max(np.abs(w_ref)))
    out = ctx.gs_download(psi)
    Y = np.stack([out[sl + (0, i, 0)].ravel(order="F") for i in range(no)], axis=1)
    h2 = O.hpsi_real(out)
    HY = np.stack([h2[sl + (0, i, 0)].ravel(order="F") for i in range(no)], axis=1)
    np.testing.assert_allclose(Y.T @ Y * s.grid.hvol, np.eye(no), atol=1e-11)
    D = Y.T @ HY * s.grid.hvol
    assert np.max(np.abs(D - np.diag(w_ref))) <= 1e-9 * max(1.0, np.max(np.abs(w_ref)))
