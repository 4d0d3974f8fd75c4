"""The non-orthogonal-lattice hpsi on the GPU (sb200_set_lattice; the
reference's zstencil_nonorthogonal, stencil.f90:120-214, with B (k+A) and the
mixed second derivatives, and the B^T of calc_current) against the oracle,
through the C ABI: H psi with and without the KB term, the Taylor step, the
time loop with J(t) ('tr' and 'lo'), on an fcc primitive cell and a triclinic
cell with unequal grid extents.

Tolerances as for the orthogonal path: 1e-12 relative per H psi and Taylor
step, 1e-10 on J(t) over the loop.
"""
import functools

import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_H = 1e-12
TOL_OBS = 1e-10


def _fcc(a=10.26):
    h = a / 2.0
    return np.array([[0.0, h, h], [h, 0.0, h], [h, h, 0.0]]).T


def _triclinic():
    return np.array([[7.2, 0.0, 0.0], [1.9, 6.8, 0.0], [-1.1, 2.3, 7.9]]).T


@functools.lru_cache(maxsize=None)
def _fcc12():
    from salmon2_b200 import synth
    return synth.nonorthogonal_system(_fcc(), 12, nkgrid=2, no=2, seed=71, natom=2, name="fcc12")


@functools.lru_cache(maxsize=None)
def _tric():
    from salmon2_b200 import synth
    return synth.nonorthogonal_system(_triclinic(), (10, 12, 14), nkgrid=1, no=3, seed=72, natom=3, nspin=2,
                                      name="tric")


def _ctx(system):
    from salmon2_b200.rt import Context
    return Context(system, device=0)


@pytest.mark.parametrize("make", [_fcc12, _tric], ids=["fcc12", "triclinic"])
@pytest.mark.parametrize("with_pp", [True, False])
def test_hpsi_nonorthogonal_against_oracle(make, with_pp):
    s = make() if with_pp else S.no_pp(make())
    O = Oracle(s)
    ctx = _ctx(s)
    for ac in ((0.0, 0.0, 0.0), (0.013, -0.021, 0.034)):
        O.set_vec_Ac(ac)
        ctx.set_vec_Ac(ac)
        h = ctx.zeros()
        ctx.hpsi(ctx.upload(s.psi), h)
        assert S.rel_err(ctx.download(h), O.hpsi(s.psi)) < TOL_H
    ctx.close()


def test_cubic_cell_through_the_nonorthogonal_branch_equals_the_orthogonal_kernels():
    """A cubic cell set as a lattice (F = (1, 1, 1, 0, 0, 0), B = 1) takes the
    two-pass kernels; the orthogonal path takes the tiled sweep: same H psi."""
    import dataclasses
    from salmon2_b200 import synth
    s = synth.nonorthogonal_system(np.diag([8.0, 8.0, 8.0]), 12, nkgrid=2, no=2, seed=73)
    a, b = _ctx(s), _ctx(dataclasses.replace(s, lattice=None))
    for ctx in (a, b):
        ctx.set_vec_Ac((0.02, 0.01, -0.03))
    ha, hb = a.zeros(), b.zeros()
    a.hpsi(a.upload(s.psi), ha)
    b.hpsi(b.upload(s.psi), hb)
    assert S.rel_err(a.download(ha), b.download(hb)) < TOL_H
    a.close()
    b.close()


def test_taylor_nonorthogonal_against_oracle():
    from salmon2_b200 import synth
    s = _fcc12()
    zc = synth.taylor_zc(0.08)
    O = Oracle(s)
    ctx = _ctx(s)
    ac = (0.01, 0.02, -0.005)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    out, work = ctx.zeros(), ctx.zeros()
    ctx.taylor(ctx.upload(s.psi), out, work, zc)
    assert S.rel_err(ctx.download(out), O.taylor(s.psi, zc)) < TOL_H
    ctx.close()


@pytest.mark.parametrize("make,trans", [(_fcc12, "tr"), (_fcc12, "lo"), (_tric, "tr")],
                         ids=["fcc12_tr", "fcc12_lo", "triclinic_tr"])
def test_rt_propagate_nonorthogonal_against_oracle(make, trans):
    """The time loop on a non-orthogonal cell: J(t) with the B^T of
    calc_current, the induced field ('lo') and the orbitals after 12 steps.
    dt = 0.02 au: the white-noise orbitals reach the top of the grid's
    spectrum, where dt = 0.08 puts dt E above the 4-term Taylor step's
    stability limit (the 'lo' feedback then diverges in the oracle too)."""
    from salmon2_b200 import synth
    s = make()
    nt, dt = 12, 0.02
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    ref = Oracle(s).rt_run(s.psi, nt, dt, zc, Ac_ext=Ac, trans_longi=1 if trans == "lo" else 0)
    ctx = _ctx(s)
    a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac, trans_longi=trans)
    jmax = np.max(np.abs(ref["curr"]))
    assert np.isfinite(jmax) and jmax > 0
    assert np.max(np.abs(res["curr"] - ref["curr"])) <= TOL_OBS * jmax
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-11
    if trans == "lo":
        assert np.max(np.abs(res["Ac_tot"] - ref["Ac_tot"])) <= TOL_OBS * np.max(np.abs(ref["Ac_tot"]))
    ctx.close()


def test_nonorthogonal_refuses_the_mixed_form_and_isolated_grids():
    from salmon2_b200 import _lib, synth
    from salmon2_b200.rt import Context
    s = _fcc12()
    ctx = Context(s, precision="mixed")
    out, work = ctx.zeros(), ctx.zeros()
    with pytest.raises(_lib.SB200Error):
        ctx.taylor(ctx.upload(s.psi), out, work, synth.taylor_zc(0.08))
    ctx.close()
    iso = Context(S.isolated_small())
    rB = np.eye(3)
    F = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])
    rc = _lib.lib().sb200_set_lattice(iso.h, rB.ctypes.data_as(_lib._dp), F.ctypes.data_as(_lib._dp))
    assert rc == 3  # SB200_ERR_UNSUPPORTED
    iso.close()
