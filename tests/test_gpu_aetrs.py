"""propagator = 'aetrs' on the GPU (sb200_set_propagator; the two half steps
of time_evolution_step with the extrapolated potential 3 V - 3 V_old1 +
V_old2 and the predicted A(itt+1)) against the oracle's loop: periodic 'tr'
and 'lo' (J(t), A(t), orbitals), the fused 16^3 Taylor-step kernel, the
self-consistent loop (where the extrapolation acts) and an isolated molecule
in the length gauge.  Tolerance 1e-10 over the loop."""
import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _fields(nt, dt):
    from salmon2_b200 import synth
    return synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)


@pytest.mark.parametrize("make,trans,nt", [(S.periodic_small, "tr", 8), (S.periodic_small, "lo", 7),
                                           (S.periodic_c2_like, "tr", 6)], ids=["p12_tr", "p12_lo", "p16_fused"])
def test_aetrs_loop_against_oracle(make, trans, nt):
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s = make()
    dt = 0.04
    zh = synth.taylor_zc(dt, aetrs=True)
    Ac = _fields(nt, dt)
    O = Oracle(s)
    O.set_propagator("aetrs")
    ref = O.rt_run(s.psi, nt, dt, zh, Ac_ext=Ac, trans_longi=1 if trans == "lo" else 0)
    ctx = Context(s)
    ctx.set_propagator("aetrs")
    res = ctx.rt_propagate(ctx.upload(s.psi), ctx.zeros(), ctx.zeros(), nt, dt, zh, Ac_ext=Ac, trans_longi=trans)
    jmax = np.max(np.abs(ref["curr"]))
    assert jmax > 0 and np.max(np.abs(res["curr"] - ref["curr"])) <= TOL * jmax
    assert np.max(np.abs(res["Ac_tot"] - ref["Ac_tot"])) <= TOL * np.max(np.abs(ref["Ac_tot"]))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < TOL
    ctx.close()


def test_aetrs_self_consistent_loop_against_oracle():
    import oracle as OR
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    from test_gpu_scf import _brl, _oracle
    s = S.periodic_small()
    nt, dt = 6, 0.04
    zh = synth.taylor_zc(dt, aetrs=True)
    Ac = _fields(nt, dt)
    brl = _brl(s)
    vpsl = np.array(s.V_local[..., 0])
    O = _oracle(s)
    O.set_propagator("aetrs")
    rho0 = O.density(s.psi)[..., 0]
    vh0 = OR.poisson_ft(rho0, brl)
    vxc0 = OR.exc_cor_pz(rho0, s.grid.hvol)[0]
    v0 = OR.update_vlocal(vpsl, vh0, vxc0[..., None])[..., 0]
    ref = O.rt_run_scf(s.psi, nt, dt, zh, vpsl, brl, v0, Ac_ext=Ac)
    ctx = Context(s)
    ctx.update_vlocal(vpsl, vh0, vxc0)
    ctx.set_self_consistent(True, vpsl, brl)
    ctx.set_propagator("aetrs")
    res = ctx.rt_propagate(ctx.upload(s.psi), ctx.zeros(), ctx.zeros(), nt, dt, zh, Ac_ext=Ac)
    jmax = np.max(np.abs(ref["curr"]))
    assert np.max(np.abs(res["curr"] - ref["curr"])) <= TOL * jmax
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < TOL
    ctx.close()


def test_aetrs_isolated_length_gauge_against_oracle():
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s = S.isolated_small()
    nt, dt = 7, 0.05
    zh = synth.taylor_zc(dt, aetrs=True)
    Ac = synth.asin2cos(nt, dt, omega=0.2, f0=0.05, tw=nt * dt, epdir=(0.3, -0.2, 0.93))
    O = Oracle(s)
    O.set_propagator("aetrs")
    O.set_length_gauge(True)
    ref = O.rt_run(s.psi, nt, dt, zh, Ac_ext=Ac)
    ctx = Context(s)
    ctx.set_propagator("aetrs")
    ctx.set_length_gauge(True)
    res = ctx.rt_propagate(ctx.upload(s.psi), ctx.zeros(), ctx.zeros(), nt, dt, zh, Ac_ext=Ac)
    assert np.max(np.abs(res["rbox"] - ref["rbox"])) <= TOL * np.max(np.abs(ref["rbox"]))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < TOL
    ctx.close()
