"""The FP64 time loop over 1000 steps against the oracle's loop, on the
configuration shapes.

* Isolated molecule: 64^3 Dirichlet grid, h = 0.25 A, 5 complex orbitals,
  4 atoms x 4 Gaussian KB projectors (rc = 1.2 A), 1e-3 au impulse kick along
  z, dt = 0.05 au, 1000 steps (main_tddft.f90:89-130 with taylor.f90:21-121);
  the tensor-copy sweep.
* Periodic bulk: the 16^3 diamond cell (a = 10.26 bohr, 8 atoms) with 32
  orbitals per k, Asin2cos A(t) (omega = 1.55 eV, peak A/c = 1e-3 au),
  dt = 0.08 au, 1000 steps; the fused Taylor-step kernel.  The k-mesh is cut
  to 2^3 ('tr') and 1 k-point ('lo', induced field on) so that the oracle
  finishes in seconds; every orbital takes the same kernel as in the full
  64-k run.

Both with the configurations' white-noise orbitals and with band-limited
orbitals (|k+G|^2/2 <= 2 Ha, a stand-in for occupied states).  The 4-term
Taylor step is not unitary: components with dt*E above about 2.8 grow and
those below decay as 1 - (dt E)^6/72, so white noise up to the grid cutoff
loses most of its norm over 1000 steps in the oracle and on the GPU alike,
while band-limited orbitals keep it.

Bar (FP64 form): 1e-10 relative on J(t) and on the dipole over the whole
loop.  The electron-count (norm) drift of both runs is printed on a line
starting with LONGLOOP, with the errors.
"""
import json

import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_OBS = 1e-10
NT = 1000


def _ctx(system):
    from salmon2_b200.rt import Context
    return Context(system, device=0)


def _report(name, **kw):
    print("LONGLOOP " + json.dumps(dict(case=name, **{k: float(v) for k, v in kw.items()})))


@pytest.mark.parametrize("ecut", [None, 2.0], ids=["white", "band_limited"])
def test_isolated_molecule_1000_steps(ecut):
    from salmon2_b200 import synth
    sysm = synth.isolated_system(num=64, h_aa=0.25, no=5, natom=4, seed=1, name="isolated_molecule", ecut=ecut)
    psi0 = synth.impulse_kick(sysm.grid, sysm.psi, 1e-3)
    dt = 0.05
    zc = synth.taylor_zc(dt)
    ref = Oracle(sysm).rt_run(psi0, NT, dt, zc)
    ctx = _ctx(sysm)
    a, b, w = ctx.upload(psi0), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, NT, dt, zc)
    d_ref = ref["rbox"][:3]
    d_got = res["rbox"][:3]
    resp_ref = d_ref - d_ref[:, :1]
    resp_got = d_got - d_got[:, :1]
    err_dip = np.max(np.abs(d_got - d_ref)) / np.max(np.abs(d_ref))
    err_resp = np.max(np.abs(resp_got - resp_ref)) / np.max(np.abs(resp_ref))
    n_ref, n_got = ref["rbox"][3], res["rbox"][3]
    err_psi = S.rel_err(ctx.download(res["psi"]), ref["psi"])
    _report("isolated_molecule_64cubed_5orb_" + ("white" if ecut is None else "band_limited"), dipole_rel=err_dip,
            dipole_response_rel=err_resp, psi_rel=err_psi, norm_drift_gpu=(n_got[-1] - n_got[0]) / n_got[0],
            norm_drift_oracle=(n_ref[-1] - n_ref[0]) / n_ref[0],
            norm_gpu_vs_oracle=np.max(np.abs(n_got - n_ref)) / n_ref[0])
    assert err_dip <= TOL_OBS
    assert err_resp <= 1e-8  # the kicked response is 1e-3 of the static dipole
    assert np.max(np.abs(n_got - n_ref)) <= 1e-12 * n_ref[0]
    ctx.close()


@pytest.mark.parametrize("trans,nkgrid,ecut", [("tr", 2, None), ("lo", 1, None), ("tr", 2, 2.0)],
                         ids=["tr_white", "lo_white", "tr_band_limited"])
def test_periodic_bulk_1000_steps_fused(trans, nkgrid, ecut):
    from salmon2_b200 import synth
    sysm = synth.periodic_system(a=10.26, num=16, nkgrid=nkgrid, no=32, seed=2, name="periodic_bulk", ecut=ecut)
    dt, omega = 0.08, 0.05696
    Ac = synth.asin2cos(NT, dt, omega=omega, f0=omega * 1e-3, tw=NT * dt)
    zc = synth.taylor_zc(dt)
    ref = Oracle(sysm).rt_run(sysm.psi, NT, dt, zc, Ac_ext=Ac, trans_longi=1 if trans == "lo" else 0)
    ctx = _ctx(sysm)
    a, b, w = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, NT, dt, zc, Ac_ext=Ac, trans_longi=trans)
    jmax = np.max(np.abs(ref["curr"]))
    err_j = np.max(np.abs(res["curr"] - ref["curr"])) / jmax
    err_rbox = S.rel_err(res["rbox"][:3], ref["rbox"][:3])
    n_ref, n_got = ref["rbox"][3], res["rbox"][3]
    err_psi = S.rel_err(ctx.download(res["psi"]), ref["psi"])
    extra = {}
    if trans == "lo":
        extra["Ac_tot_rel"] = np.max(np.abs(res["Ac_tot"] - ref["Ac_tot"])) / np.max(np.abs(ref["Ac_tot"]))
    _report(f"periodic_bulk_16cubed_{nkgrid ** 3}k_32orb_{trans}_" + ("white" if ecut is None else "band_limited"),
            current_rel=err_j, dipole_rel=err_rbox,
            psi_rel=err_psi, norm_drift_gpu=(n_got[-1] - n_got[0]) / n_got[0],
            norm_drift_oracle=(n_ref[-1] - n_ref[0]) / n_ref[0],
            norm_gpu_vs_oracle=np.max(np.abs(n_got - n_ref)) / n_ref[0], **extra)
    assert jmax > 0
    assert err_j <= TOL_OBS
    assert err_rbox <= TOL_OBS
    assert np.max(np.abs(n_got - n_ref)) <= 1e-12 * n_ref[0]
    if trans == "lo":
        assert extra["Ac_tot_rel"] <= TOL_OBS
    ctx.close()
