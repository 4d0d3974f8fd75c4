"""The absorbing boundary along z on the GPU (sb200_set_absorbing_boundary;
add_imaginary_potential_for_absorbing_boundary_z of hamiltonian.f90, -i w(z)
psi on the planes within imagnary_potential_dr of the cell's z faces) against
the oracle, through the C ABI: H psi with and without the KB term, two spins,
with the single-scale stencil, ttpsi, the Taylor step and the time loop (whose
norm it absorbs).  Tolerances as for the other H psi forms: 1e-12 per call,
1e-10 over the loop."""
import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu

W0, DR = 0.3, 2.0


def _pair(s):
    from salmon2_b200.rt import Context
    O, ctx = Oracle(s), Context(s)
    O.set_absorbing_boundary(W0, DR)
    ctx.set_absorbing_boundary(W0, DR)
    return O, ctx


@pytest.mark.parametrize("make", [S.periodic_small, lambda: S.no_pp(S.periodic_small()),
                                  lambda: S.periodic_small(nspin=2), S.isolated_small],
                         ids=["pp", "no_pp", "two_spins", "isolated"])
def test_hpsi_absorbing_boundary_against_oracle(make):
    s = make()
    O, ctx = _pair(s)
    ac = (0.01, -0.02, 0.005)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(s.psi), h)
    assert S.rel_err(ctx.download(h), O.hpsi(s.psi)) < 1e-12
    ctx.close()


def test_absorbing_boundary_with_the_single_scale_stencil_and_ttpsi():
    from test_gpu_microac import _field
    s = S.periodic_small()
    O, ctx = _pair(s)
    acm, div = _field(s.grid, 7)
    O.set_micro_ac(acm, div)
    ctx.set_micro_ac(acm, div)
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(s.psi), h)
    assert S.rel_err(ctx.download(h), O.hpsi(s.psi)) < 1e-12
    O.set_micro_ac(None)
    ctx.set_micro_ac(None)
    h, tt = ctx.zeros(), ctx.zeros()
    ctx.hpsi_tt(ctx.upload(s.psi), h, tt)
    h_ref, tt_ref = O.hpsi_tt(s.psi)
    assert S.rel_err(ctx.download(h), h_ref) < 1e-12
    assert S.rel_err(ctx.download(tt), tt_ref) < 1e-12
    ctx.close()


def test_time_loop_with_absorbing_boundary_against_oracle():
    from salmon2_b200 import synth
    s = S.periodic_small()
    O, ctx = _pair(s)
    nt, dt = 12, 0.02
    zc = synth.taylor_zc(dt)
    out, work = ctx.zeros(), ctx.zeros()
    ctx.taylor(ctx.upload(s.psi), out, work, zc)
    assert S.rel_err(ctx.download(out), O.taylor(s.psi, zc)) < 1e-12
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    ref = O.rt_run(s.psi, nt, dt, zc, Ac_ext=Ac)
    res = ctx.rt_propagate(ctx.upload(s.psi), ctx.zeros(), ctx.zeros(), nt, dt, zc, Ac_ext=Ac)
    jmax = np.max(np.abs(ref["curr"]))
    assert np.max(np.abs(res["curr"] - ref["curr"])) <= 1e-10 * jmax
    got = ctx.download(res["psi"])
    assert S.rel_err(got, ref["psi"]) < 1e-10
    sl = s.grid.interior_slices()
    assert np.linalg.norm(got[sl]) < np.linalg.norm(s.psi[sl])  # the boundary absorbs
    ctx.close()


def test_absorbing_boundary_refuses_the_mixed_form_and_lattices():
    from salmon2_b200 import _lib, synth
    from salmon2_b200.rt import Context
    s = S.periodic_small()
    ctx = Context(s, precision="mixed")
    ctx.set_absorbing_boundary(W0, DR)
    out, work = ctx.zeros(), ctx.zeros()
    with pytest.raises(_lib.SB200Error):
        ctx.taylor(ctx.upload(s.psi), out, work, synth.taylor_zc(0.05))
    ctx.close()
    rB = np.eye(3)
    F = np.array([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])
    ctx = Context(s)
    ctx.set_absorbing_boundary(W0, DR)
    rc = _lib.lib().sb200_set_lattice(ctx.h, rB.ctypes.data_as(_lib._dp), F.ctypes.data_as(_lib._dp))
    assert rc == 3  # SB200_ERR_UNSUPPORTED
    ctx.close()
