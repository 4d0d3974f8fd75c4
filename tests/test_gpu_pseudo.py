"""H psi and a short time loop on the GPU with the Kleinman-Bylander tables and
the local potential built from pseudopotential files by the library's
host-side set-up (sb200_init_ps_ky for Yabana-Bertsch files; sb200_init_ps
for ABINIT and FHI files), against the oracle on the same tables: the
set-up's output drives the propagation path unchanged."""
import dataclasses

import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _ky_molecule(tmp_path):
    from salmon2_b200 import pseudo, synth
    fa = S.write_ky_file(str(tmp_path / "A_rps.dat"), zps=4.0, mlps=2, seed=11)
    fb = S.write_ky_file(str(tmp_path / "B_rps.dat"), zps=1.0, mlps=1, rc=0.9, seed=12)
    base = synth.isolated_system(num=28, h_aa=0.25, no=4, natom=3, seed=21, name="ky28")
    rion = np.array([[0.4, -0.3, 1.2], [-1.5, 0.6, -0.8], [1.9, 1.1, 0.2]]).T
    pp, vpsl = pseudo.init_ps_ky([fa, fb], [2, 0], base.grid, rion, [1, 2, 1])
    return dataclasses.replace(base, pp=pp, rion=rion, V_local=np.asfortranarray(vpsl[..., None]))


def test_hpsi_with_tables_from_pseudopotential_files(tmp_path):
    from salmon2_b200.rt import Context
    s = _ky_molecule(tmp_path)
    assert s.pp.nlma == 11
    ctx = Context(s)
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(s.psi), h)
    assert S.rel_err(ctx.download(h), Oracle(s).hpsi(s.psi)) < 1e-12
    ctx.close()


def test_time_loop_with_tables_from_pseudopotential_files(tmp_path):
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s0 = _ky_molecule(tmp_path)
    s = dataclasses.replace(s0, psi=synth.impulse_kick(s0.grid, s0.psi, 1e-3))
    nt, dt = 20, 0.05
    zc = synth.taylor_zc(dt)
    ref = Oracle(s).rt_run(s.psi, nt, dt, zc)
    ctx = Context(s)
    a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc)
    d_ref = ref["rbox"][:3] - ref["rbox"][:3, :1]
    d_got = res["rbox"][:3] - res["rbox"][:3, :1]
    assert np.max(np.abs(d_got - d_ref)) <= 1e-10 * np.max(np.abs(ref["rbox"][:3]))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-11
    ctx.close()


@pytest.mark.parametrize("fmt", ["pspnc", "fhi"])
def test_hpsi_with_tables_from_abinit_and_fhi_files(tmp_path, fmt):
    from salmon2_b200 import pseudo, synth
    from salmon2_b200.rt import Context
    if fmt == "pspnc":
        f = S.write_abinit_file(str(tmp_path / "A.pspnc"), zps=4.0, mlps=2, seed=13)
    else:
        f = S.write_fhi_file(str(tmp_path / "A.fhi"), zps=4.0, mlps=2, seed=13)
    base = synth.isolated_system(num=28, h_aa=0.25, no=4, natom=2, seed=22, name="fmt28")
    rion = np.array([[0.4, -0.3, 1.2], [-1.5, 0.6, -0.8]]).T
    pp, vpsl = pseudo.init_ps([f], [2], base.grid, rion, [1, 1])
    s = dataclasses.replace(base, pp=pp, rion=rion, V_local=np.asfortranarray(vpsl[..., None]))
    assert s.pp.nlma == 8
    ctx = Context(s)
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(s.psi), h)
    assert S.rel_err(ctx.download(h), Oracle(s).hpsi(s.psi)) < 1e-12
    ctx.close()
