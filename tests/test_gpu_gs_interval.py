"""gram_schmidt_interval inside the time loop on the GPU
(sb200_set_gram_schmidt_interval: gram_schmidt of psi(t+dt) every N steps,
before its density and current, as a conditional node of the loop's CUDA
graph) against the oracle's loop: periodic 'tr' with N = 2 and 3 (odd and
even step counts), the fused 16^3 kernel (its observables then taken after
the Gram-Schmidt step), and AETRS.  Tolerance 1e-10 over the loop."""
import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.mark.parametrize("make,n,nt,prop", [(S.periodic_small, 2, 7, "middlepoint"),
                                            (S.periodic_small, 3, 6, "middlepoint"),
                                            (S.periodic_c2_like, 2, 6, "middlepoint"),
                                            (S.periodic_small, 2, 6, "aetrs")],
                         ids=["p12_n2", "p12_n3", "p16_fused_n2", "p12_aetrs"])
def test_loop_with_gram_schmidt_against_oracle(make, n, nt, prop):
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s = make()
    dt = 0.02
    zc = synth.taylor_zc(dt, aetrs=prop == "aetrs")
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    psi0 = s.psi * 1.3
    O = Oracle(s)
    O.set_gram_schmidt_interval(n)
    O.set_propagator(prop)
    ref = O.rt_run(psi0, nt, dt, zc, Ac_ext=Ac)
    ctx = Context(s)
    ctx.set_gram_schmidt_interval(n)
    ctx.set_propagator(prop)
    res = ctx.rt_propagate(ctx.upload(psi0), ctx.zeros(), ctx.zeros(), nt, dt, zc, Ac_ext=Ac)
    jmax = np.max(np.abs(ref["curr"]))
    assert jmax > 0 and np.max(np.abs(res["curr"] - ref["curr"])) <= TOL * jmax
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < TOL
    # back to the plain loop
    ctx.set_gram_schmidt_interval(-1)
    res2 = ctx.rt_propagate(ctx.upload(psi0), ctx.zeros(), ctx.zeros(), 2, dt, zc, Ac_ext=Ac[:, :4])
    O2 = Oracle(s)
    O2.set_propagator(prop)
    ref2 = O2.rt_run(psi0, 2, dt, zc, Ac_ext=Ac[:, :4])
    assert S.rel_err(ctx.download(res2["psi"]), ref2["psi"]) < TOL
    ctx.close()
