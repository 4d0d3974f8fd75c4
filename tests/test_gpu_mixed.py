"""Mixed-precision form (FP32 Taylor terms n >= 2, FP64 first term and psi
accumulation) against the FP64 oracle.  The error budget of the mixed form is
a relative error of J(t) <= 1e-6; the tests state the error they measure."""
import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_J_MIXED = 1e-6


def _ctx(system, precision):
    from salmon2_b200.rt import Context
    return Context(system, device=0, precision=precision)


@pytest.mark.parametrize("make", [S.periodic_small, S.periodic_c2_like, S.isolated_small], ids=lambda f: f.__name__)
def test_mixed_taylor_step_close_to_fp64(make):
    from salmon2_b200 import synth
    s = make()
    O = Oracle(s)
    ac = (0.0, 0.0, 0.02)
    O.set_vec_Ac(ac)
    zc = synth.taylor_zc(0.05)
    ref = O.taylor(s.psi, zc)
    ctx = _ctx(s, "mixed")
    ctx.set_vec_Ac(ac)
    a = ctx.upload(s.psi)
    out, work = ctx.zeros(), ctx.zeros()
    ctx.taylor(a, out, work, zc)
    err = S.rel_err(ctx.download(out), ref)
    # FP32 rounding of terms n >= 2, damped by dt^n / n!
    assert err < 1e-6, err
    assert err > 1e-14  # the FP32 path really ran


def test_mixed_current_over_time_loop():
    from salmon2_b200 import synth
    s = S.periodic_small()
    nt, dt = 200, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    ref = Oracle(s).rt_run(s.psi, nt, dt, zc, Ac_ext=Ac)
    ctx = _ctx(s, "mixed")
    a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)
    jmax = np.max(np.abs(ref["curr"]))
    err_j = np.max(np.abs(res["curr"] - ref["curr"])) / jmax
    norm_ref = ref["rbox"][3]
    norm_mix = res["rbox"][3]
    assert err_j <= TOL_J_MIXED, err_j
    assert np.max(np.abs(norm_mix - norm_ref)) / norm_ref[0] < 1e-6


def test_mixed_taylor_step_with_tensor_core_projections(monkeypatch):
    """The mixed form's FP32 Taylor terms feed the tensor-core projections
    through their FP32-input path (SB200_PROJECT=dmma): a Taylor step stays
    within the mixed form's error of the FP64 oracle."""
    from salmon2_b200 import synth
    monkeypatch.setenv("SB200_PROJECT", "dmma")
    s = synth.periodic_system(a=10.26, num=12, nkgrid=1, no=20, seed=45, name="p12n20")
    O = Oracle(s)
    ac = (0.0, 0.0, 0.02)
    O.set_vec_Ac(ac)
    zc = synth.taylor_zc(0.05)
    ref = O.taylor(s.psi, zc)
    ctx = _ctx(s, "mixed")
    ctx.set_vec_Ac(ac)
    out, work = ctx.zeros(), ctx.zeros()
    ctx.taylor(ctx.upload(s.psi), out, work, zc)
    err = S.rel_err(ctx.download(out), ref)
    assert 1e-14 < err < 1e-6, err
