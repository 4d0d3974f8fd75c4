"""yn_predictor_corrector = 'y' on the GPU (sb200_set_predictor_corrector;
time_evolution_step's predictor_corrector: a predicted step, the potential of
its density, V_local = (V_step + V_predicted) / 2, the step again) against the
oracle's loop: periodic self-consistent (J(t), orbitals), isolated with the
Hartree potential by CG, and an isolated molecule in the length gauge with a
fixed potential.  Tolerance 1e-10 over the loop (the CG loop: the dipole
response to 1e-8, as for the plain CG loop)."""
import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu


def test_predictor_corrector_periodic_self_consistent():
    import oracle as OR
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    from test_gpu_scf import _brl, _oracle
    s = S.periodic_small()
    nt, dt = 6, 0.08
    zc = synth.taylor_zc(dt)
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    brl = _brl(s)
    vpsl = np.array(s.V_local[..., 0])
    O = _oracle(s)
    O.set_predictor_corrector(True)
    rho0 = O.density(s.psi)[..., 0]
    vh0 = OR.poisson_ft(rho0, brl)
    vxc0 = OR.exc_cor_pz(rho0, s.grid.hvol)[0]
    v0 = OR.update_vlocal(vpsl, vh0, vxc0[..., None])[..., 0]
    ref = O.rt_run_scf(s.psi, nt, dt, zc, vpsl, brl, v0, Ac_ext=Ac)
    ctx = Context(s)
    ctx.update_vlocal(vpsl, vh0, vxc0)
    ctx.set_self_consistent(True, vpsl, brl)
    ctx.set_predictor_corrector(True)
    res = ctx.rt_propagate(ctx.upload(s.psi), ctx.zeros(), ctx.zeros(), nt, dt, zc, Ac_ext=Ac)
    jmax = np.max(np.abs(ref["curr"]))
    assert jmax > 0 and np.max(np.abs(res["curr"] - ref["curr"])) <= 1e-10 * jmax
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-10
    ctx.close()


def test_predictor_corrector_isolated_cg():
    import dataclasses as dc
    import oracle as OR
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    from test_gpu_scf import _brl, _oracle
    s0 = S.isolated_small()
    s = dc.replace(s0, psi=synth.impulse_kick(s0.grid, s0.psi, 1e-3))
    nt, dt = 5, 0.05
    zc = synth.taylor_zc(dt)
    vpsl = np.array(s.V_local[..., 0])
    O = _oracle(s)
    O.set_predictor_corrector(True)
    rho0 = O.density(s.psi)[..., 0]
    vh0, _ = O.poisson_isolated_cg(rho0)
    vxc0 = OR.exc_cor_pz(rho0, s.grid.hvol)[0]
    v0 = OR.update_vlocal(vpsl, vh0, vxc0[..., None])[..., 0]
    ref = O.rt_run_scf(s.psi, nt, dt, zc, vpsl, None, v0, cg=dict(vh0=vh0))
    ctx = Context(s)
    ctx.update_vlocal(vpsl, vh0, vxc0)
    ctx.set_hartree_cg(vh0)
    ctx.set_self_consistent(True, vpsl, _brl(s))
    ctx.set_predictor_corrector(True)
    res = ctx.rt_propagate(ctx.upload(s.psi), ctx.zeros(), ctx.zeros(), nt, dt, zc)
    d_ref = ref["rbox"][:3] - ref["rbox"][:3, :1]
    d_got = res["rbox"][:3] - res["rbox"][:3, :1]
    assert np.max(np.abs(d_got - d_ref)) <= 1e-8 * np.max(np.abs(d_ref))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-10
    ctx.close()


def test_predictor_corrector_length_gauge_fixed_potential():
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s = S.isolated_odd()
    nt, dt = 6, 0.05
    zc = synth.taylor_zc(dt)
    Ac = synth.asin2cos(nt, dt, omega=0.2, f0=0.05, tw=nt * dt, epdir=(0.3, -0.2, 0.93))
    O = Oracle(s)
    O.set_length_gauge(True)
    O.set_predictor_corrector(True)
    ref = O.rt_run(s.psi, nt, dt, zc, Ac_ext=Ac)
    ctx = Context(s)
    ctx.set_length_gauge(True)
    ctx.set_predictor_corrector(True)
    res = ctx.rt_propagate(ctx.upload(s.psi), ctx.zeros(), ctx.zeros(), nt, dt, zc, Ac_ext=Ac)
    assert np.max(np.abs(res["rbox"] - ref["rbox"])) <= 1e-10 * np.max(np.abs(ref["rbox"]))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-10
    ctx.close()
