"""An isolated molecule driven by a pulse in the length gauge
(sb200_set_length_gauge; calcVbox and V_local + Vbox of the reference's time
step, E_ext(itt) = -(Ac_ext(itt+1) - Ac_ext(itt)) / dt) against the oracle's
loop: the dipole every step and the final orbitals, with the fixed potential
and with the self-consistent CG potential, odd and even grid extents (the two
forms of lg%coordinate).  The same pulse without the length gauge leaves an
isolated system untouched (no A(t) on isolated grids).  Tolerance 1e-10, as
for the other loops."""
import dataclasses as dc

import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _pulse(nt, dt, f0=0.05):
    from salmon2_b200 import synth
    return synth.asin2cos(nt, dt, omega=0.2, f0=f0, tw=nt * dt, epdir=(0.3, -0.2, 0.93))


@pytest.mark.parametrize("make", [S.isolated_small, S.isolated_odd], ids=["even", "odd"])
def test_length_gauge_loop_against_oracle(make):
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s = make()
    nt, dt = 12, 0.05
    zc = synth.taylor_zc(dt)
    Ac = _pulse(nt, dt)
    O = Oracle(s)
    O.set_length_gauge(True)
    ref = O.rt_run(s.psi, nt, dt, zc, Ac_ext=Ac)
    free = Oracle(s).rt_run(s.psi, nt, dt, zc, Ac_ext=Ac)
    ctx = Context(s)
    ctx.set_length_gauge(True)
    res = ctx.rt_propagate(ctx.upload(s.psi), ctx.zeros(), ctx.zeros(), nt, dt, zc, Ac_ext=Ac)
    d_ref = ref["rbox"][:3] - free["rbox"][:3]
    assert np.max(np.abs(d_ref)) > 1e-6 * np.max(np.abs(ref["rbox"][:3]))  # the field acts
    assert np.max(np.abs(res["rbox"][:3] - ref["rbox"][:3])) <= 1e-10 * np.max(np.abs(d_ref))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-10
    # the field-free potential is back after the loop: H psi as without the gauge
    h = ctx.zeros()
    ctx.hpsi(res["psi"], h)
    assert S.rel_err(ctx.download(h), Oracle(s).hpsi(ref["psi"])) < 1e-12
    ctx.close()


def test_length_gauge_with_the_self_consistent_cg_loop():
    import oracle as OR
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    from test_gpu_scf import _brl, _oracle
    s = S.isolated_small()
    nt, dt = 6, 0.05
    zc = synth.taylor_zc(dt)
    Ac = _pulse(nt, dt)
    vpsl = np.array(s.V_local[..., 0])
    O = _oracle(s)
    O.set_length_gauge(True)
    rho0 = O.density(s.psi)[..., 0]
    vh0, _ = O.poisson_isolated_cg(rho0)
    vxc0 = OR.exc_cor_pz(rho0, s.grid.hvol)[0]
    v0 = OR.update_vlocal(vpsl, vh0, vxc0[..., None])[..., 0]
    ref = O.rt_run_scf(s.psi, nt, dt, zc, vpsl, None, v0, Ac_ext=Ac, cg=dict(vh0=vh0))
    ctx = Context(s)
    ctx.update_vlocal(vpsl, vh0, vxc0)
    ctx.set_hartree_cg(vh0)
    ctx.set_self_consistent(True, vpsl, _brl(s))
    ctx.set_length_gauge(True)
    res = ctx.rt_propagate(ctx.upload(s.psi), ctx.zeros(), ctx.zeros(), nt, dt, zc, Ac_ext=Ac)
    d_ref = ref["rbox"][:3] - ref["rbox"][:3, :1]
    d_got = res["rbox"][:3] - res["rbox"][:3, :1]
    assert np.max(np.abs(d_got - d_ref)) <= 1e-8 * np.max(np.abs(d_ref))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-10
    ctx.close()


def test_length_gauge_is_refused_on_periodic_grids():
    from salmon2_b200 import _lib
    from salmon2_b200.rt import Context
    ctx = Context(S.periodic_small())
    with pytest.raises(_lib.SB200Error):
        ctx.set_length_gauge(True)
    ctx.close()
