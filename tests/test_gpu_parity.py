"""GPU parity of the FP64 path against the CPU oracle, through the C ABI.

Tolerances (FP64 form): 1e-12 relative (max-norm) per H psi and per Taylor
step; 1e-10 relative on the current J(t) and the dipole over the time loop.
"""
import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_H = 1e-12
TOL_OBS = 1e-10


def _ctx(system, precision="fp64"):
    from salmon2_b200.rt import Context
    return Context(system, device=0, precision=precision)


SYSTEMS = [S.periodic_small, S.periodic_c2_like, S.isolated_small, S.isolated_odd]


@pytest.mark.parametrize("make", SYSTEMS, ids=lambda f: f.__name__)
def test_relayout_round_trip(make):
    sysm = make()
    ctx = _ctx(sysm)
    psi = ctx.upload(sysm.psi)
    back = ctx.download(psi)
    assert np.array_equal(back, sysm.psi)


@pytest.mark.parametrize("make", SYSTEMS, ids=lambda f: f.__name__)
@pytest.mark.parametrize("with_pp", [True, False])
def test_hpsi_parity(make, with_pp):
    sysm = make() if with_pp else S.no_pp(make())
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    ac = (0.013, -0.021, 0.034)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    ref = O.hpsi(sysm.psi)
    t = ctx.upload(sysm.psi)
    h = ctx.zeros()
    ctx.hpsi(t, h)
    got = ctx.download(h)
    assert S.rel_err(got, ref) < TOL_H


def test_hpsi_parity_two_spins():
    sysm = S.periodic_small(nspin=2)
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    ref = O.hpsi(sysm.psi)
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(sysm.psi), h)
    assert S.rel_err(ctx.download(h), ref) < TOL_H


@pytest.mark.parametrize("make", SYSTEMS, ids=lambda f: f.__name__)
def test_hpsi_tt_and_eigen_energy(make):
    """hpsi's optional kinetic output ttpsi and calc_eigen_energy (esp,
    E_kin, E_ion_nloc) against the oracle."""
    sysm = make()
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    ac = (0.013, -0.004, 0.02)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    t = ctx.upload(sysm.psi)
    h, tt = ctx.zeros(), ctx.zeros()
    ctx.hpsi_tt(t, h, tt)
    ref_h, ref_tt = O.hpsi_tt(sysm.psi)
    assert S.rel_err(ctx.download(h), ref_h) < TOL_H
    assert S.rel_err(ctx.download(tt), ref_tt) < TOL_H
    esp, ek, en = ctx.calc_eigen_energy(t, h, tt)
    ref_esp, ref_ek, ref_en = O.calc_eigen_energy(sysm.psi)
    scale = np.max(np.abs(ref_esp))
    assert np.max(np.abs(esp - ref_esp)) <= TOL_H * scale
    assert abs(ek - ref_ek) <= TOL_H * abs(ref_ek)
    assert abs(en - ref_en) <= TOL_H * max(abs(ref_en), scale)


@pytest.mark.parametrize("make", SYSTEMS, ids=lambda f: f.__name__)
def test_taylor_parity(make):
    from salmon2_b200 import synth
    sysm = make()
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    ac = (0.0, 0.0, 0.02)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    zc = synth.taylor_zc(0.05)
    ref = O.taylor(sysm.psi, zc)
    a = ctx.upload(sysm.psi)
    out, work = ctx.zeros(), ctx.zeros()
    ctx.taylor(a, out, work, zc)
    assert S.rel_err(ctx.download(out), ref) < TOL_H


@pytest.mark.parametrize("make", SYSTEMS, ids=lambda f: f.__name__)
def test_density_and_dip(make):
    sysm = make()
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    psi = ctx.upload(sysm.psi)
    rho = ctx.calc_density(psi)
    rho_ref = O.density(sysm.psi)
    assert S.rel_err(rho, rho_ref) < TOL_H
    rb = ctx.calc_dip(rho_ref)
    rb_ref = O.dip(rho_ref)
    assert np.max(np.abs(rb - rb_ref)) <= 1e-11 * np.max(np.abs(rb_ref))


@pytest.mark.parametrize("make", [S.periodic_small, S.periodic_c2_like], ids=lambda f: f.__name__)
def test_current(make):
    sysm = make()
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    a_mid, a_cur = (0.01, 0.02, -0.03), (0.011, 0.019, -0.029)
    O.set_vec_Ac(a_mid)
    ctx.set_vec_Ac(a_mid)
    O.set_vec_Ac_local_only(a_cur)
    ref = O.current(sysm.psi)
    got = ctx.calc_current(ctx.upload(sysm.psi), a_cur)
    assert np.max(np.abs(got - ref)) <= TOL_OBS * max(np.max(np.abs(ref)), 1e-30)


@pytest.mark.parametrize("trans", ["tr", "lo"])
def test_rt_propagate_periodic(trans):
    from salmon2_b200 import synth
    sysm = S.periodic_small()
    nt, dt = 40, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    O = Oracle(sysm)
    ref = O.rt_run(sysm.psi, nt, dt, zc, Ac_ext=Ac, trans_longi=1 if trans == "lo" else 0)
    ctx = _ctx(sysm)
    a, b, w = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac, trans_longi=trans)
    jmax = np.max(np.abs(ref["curr"]))
    assert jmax > 0
    assert np.max(np.abs(res["curr"] - ref["curr"])) <= TOL_OBS * jmax
    assert S.rel_err(res["rbox"], ref["rbox"]) < TOL_OBS
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-11
    if trans == "lo":
        assert np.max(np.abs(res["Ac_tot"] - ref["Ac_tot"])) <= 1e-10 * np.max(np.abs(ref["Ac_tot"]))


def test_rt_propagate_isolated_kick():
    from salmon2_b200 import synth
    sysm = S.isolated_small()
    psi0 = synth.impulse_kick(sysm.grid, sysm.psi, 1e-3)
    nt, dt = 30, 0.05
    zc = synth.taylor_zc(dt)
    O = Oracle(sysm)
    ref = O.rt_run(psi0, nt, dt, zc)
    ctx = _ctx(sysm)
    a, b, w = ctx.upload(psi0), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc)
    # dipole response relative to the static dipole (dDp_e of dip.f90:62-63)
    d_ref = ref["rbox"][:3] - ref["rbox"][:3, :1]
    d_got = res["rbox"][:3] - res["rbox"][:3, :1]
    assert np.max(np.abs(d_got - d_ref)) <= TOL_OBS * np.max(np.abs(ref["rbox"][:3]))
    assert np.max(np.abs(res["rbox"][3] - ref["rbox"][3])) <= 1e-12 * ref["rbox"][3, 0]


def test_error_codes():
    from salmon2_b200.rt import SB200Error
    sysm = S.periodic_small()
    ctx = _ctx(sysm)
    a = ctx.upload(sysm.psi)
    with pytest.raises(SB200Error) as e:
        ctx.hpsi(a, a)  # aliased input / output
    assert e.value.code == 1


@pytest.mark.parametrize("trans", ["tr", "lo"])
def test_rt_propagate_periodic16_orbital_kernel(trans):
    """16^3 periodic grids take the orbital-resident kernel with the
    observables fused into the last Taylor term."""
    from salmon2_b200 import synth
    sysm = synth.periodic_system(a=10.26, num=16, nkgrid=2, no=2, seed=31, name="periodic16k8")
    nt, dt = 24, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    O = Oracle(sysm)
    ref = O.rt_run(sysm.psi, nt, dt, zc, Ac_ext=Ac, trans_longi=1 if trans == "lo" else 0)
    ctx = _ctx(sysm)
    a, b, w = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac, trans_longi=trans)
    jmax = np.max(np.abs(ref["curr"]))
    assert np.max(np.abs(res["curr"] - ref["curr"])) <= TOL_OBS * jmax
    assert S.rel_err(res["rbox"], ref["rbox"]) < TOL_OBS
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-11


@pytest.mark.parametrize("variant", ["fused", "fused_nosplit", "unstaged", "persistent", "terms"])
def test_rt_propagate_periodic16_many_orbitals(variant, monkeypatch):
    """More orbitals than SMs: the fused-step kernel (all Taylor terms in one
    launch; its default form with the KB projections split over two warps per
    atom, and the form with one warp per atom) with its KB tables staged in
    shared memory and without, the persistent per-term form that walks several
    orbitals per CTA through double-buffered bulk copies (buffer reuse, barrier
    phase flips) and the one-launch-per-term form, each against the oracle on
    the same input."""
    from salmon2_b200 import synth
    monkeypatch.setenv("SB200_ORBITAL", variant.split("_")[0])
    monkeypatch.setenv("SB200_BLK_SPLIT", "0" if variant.endswith("nosplit") else "1")
    sysm = synth.periodic_system(a=10.26, num=16, nkgrid=4, no=5, seed=32, name="periodic16k64")
    nt, dt = 6, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    ref = Oracle(sysm).rt_run(sysm.psi, nt, dt, zc, Ac_ext=Ac, trans_longi=1)
    ctx = _ctx(sysm)
    a, b, w = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac, trans_longi="lo")
    jmax = np.max(np.abs(ref["curr"]))
    assert np.max(np.abs(res["curr"] - ref["curr"])) <= TOL_OBS * jmax
    assert S.rel_err(res["rbox"], ref["rbox"]) < TOL_OBS
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-11


def _p16_two_spins():
    from salmon2_b200 import synth
    return synth.periodic_system(a=10.26, num=16, nkgrid=1, no=2, seed=35, nspin=2, name="p16s2")


def _p16_wide_spheres():
    # rc = 2.0 A: about 860 sphere points per atom, pair tables too large for
    # shared memory -> the fused step reads the KB tables from global memory
    from salmon2_b200 import synth
    return synth.periodic_system(a=10.26, num=16, nkgrid=1, no=2, seed=36, rc_aa=2.0, name="p16wide")


def _p16_no_pp():
    from salmon2_b200 import synth
    return S.no_pp(synth.periodic_system(a=10.26, num=16, nkgrid=2, no=2, seed=37, name="p16nopp"))


def _p16_twelve_atoms():
    # 12 atoms (more than half the warps of the fused step: the split
    # projections take two rounds, and no TMEM cache), smaller spheres
    import dataclasses
    from salmon2_b200 import synth
    s = synth.periodic_system(a=10.26, num=16, nkgrid=1, no=3, seed=39, rc_aa=0.9, name="p16twelve")
    rng = np.random.default_rng(39)
    rion = np.asfortranarray(np.concatenate([s.rion, rng.uniform(0.0, 10.26, size=(3, 4))], axis=1))
    pp = synth.make_pp(s.grid, rion, 0.9 / synth.AU_LENGTH_AA, sigma=rng.uniform(0.5, 0.8, 12),
                       amp=rng.uniform(0.3, 0.6, 12), inorm=rng.choice([-1, 1], size=(12, 2)),
                       cell=np.full(3, 10.26))
    return dataclasses.replace(s, pp=pp, rion=rion)


@pytest.mark.parametrize("make", [_p16_two_spins, _p16_wide_spheres, _p16_no_pp, _p16_twelve_atoms],
                         ids=lambda f: f.__name__)
def test_fused_step_variants_against_oracle(make):
    """The fused 16^3 step on two spins, on projector spheres whose tables do
    not fit in shared memory (fallback to global tables), without projectors
    and with more atoms than warp pairs: J(t), the dipole and psi against the
    oracle's time loop."""
    from salmon2_b200 import synth
    sysm = make()
    nt, dt = 6, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    ref = Oracle(sysm).rt_run(sysm.psi, nt, dt, zc, Ac_ext=Ac, trans_longi=0)
    ctx = _ctx(sysm)
    a, b, w = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac, trans_longi="tr")
    jmax = np.max(np.abs(ref["curr"]))
    assert np.max(np.abs(res["curr"] - ref["curr"])) <= TOL_OBS * max(jmax, 1e-30)
    assert S.rel_err(res["rbox"], ref["rbox"]) < TOL_OBS
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-11


def _iso_no_pp():
    return S.no_pp(S.isolated_small())


def _p32_no_pp():
    return S.no_pp(_periodic32())


def _p12_two_spins():
    return S.periodic_small(nspin=2)


@pytest.mark.parametrize("make", [_iso_no_pp, _p32_no_pp, _p12_two_spins], ids=lambda f: f.__name__)
def test_rt_propagate_edge_systems(make):
    """The time loop on the tiled / tensor-copy kernels and the separate
    observables kernels without projectors and with two spins."""
    from salmon2_b200 import synth
    sysm = make()
    nt, dt = 6, 0.05
    zc = synth.taylor_zc(dt)
    if sysm.grid.periodic:
        Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
        ref = Oracle(sysm).rt_run(sysm.psi, nt, dt, zc, Ac_ext=Ac, trans_longi=0)
    else:
        Ac = None
        ref = Oracle(sysm).rt_run(sysm.psi, nt, dt, zc)
    ctx = _ctx(sysm)
    a, b, w = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac, trans_longi="tr") if Ac is not None else \
        ctx.rt_propagate(a, b, w, nt, dt, zc)
    if sysm.grid.periodic:
        jmax = np.max(np.abs(ref["curr"]))
        assert np.max(np.abs(res["curr"] - ref["curr"])) <= TOL_OBS * jmax
    assert S.rel_err(res["rbox"], ref["rbox"]) < TOL_OBS
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-11


@pytest.mark.parametrize("num,a", [(12, 6.0), (16, 6.0)])
def test_spheres_reaching_a_point_twice(num, a):
    """Projector spheres wider than half the cell reach some grid points through
    two periodic images: the (point, atom) pair form does not apply and the
    kernels take the per-entry scatter (12^3: tiled sweep; 16^3: fused step)."""
    from salmon2_b200 import synth
    sysm = synth.periodic_system(a=a, num=num, nkgrid=1, no=2, seed=38, rc_aa=1.8, name="wrap")
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    ac = (0.01, 0.0, -0.02)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    t = ctx.upload(sysm.psi)
    h = ctx.zeros()
    ctx.hpsi(t, h)
    assert S.rel_err(ctx.download(h), O.hpsi(sysm.psi)) < TOL_H
    zc = synth.taylor_zc(0.05)
    out, work = ctx.zeros(), ctx.zeros()
    ctx.taylor(ctx.upload(sysm.psi), out, work, zc)
    assert S.rel_err(ctx.download(out), O.taylor(sysm.psi, zc)) < TOL_H


@pytest.mark.parametrize("n_hamil", [4, 1, 3])
def test_fused_step_equals_term_launches(n_hamil, monkeypatch):
    """The fused Taylor step with the global KB tables and the per-term
    launches do the same arithmetic per point and term: Taylor steps, J(t),
    the dipole and the orbitals agree bit for bit.  (The default fused form
    stages the tables in shared memory and sums the scatter by (point, atom)
    pair; it is checked against the oracle.)"""
    from salmon2_b200 import synth
    sysm = synth.periodic_system(a=10.26, num=16, nkgrid=2, no=3, seed=34, name="periodic16k8")
    zc = synth.taylor_zc(0.08)[:n_hamil]
    nt, dt = 5, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    outs, runs = [], []
    for variant in ("unstaged", "terms"):
        monkeypatch.setenv("SB200_ORBITAL", variant)
        ctx = _ctx(sysm)
        ctx.set_vec_Ac((0.01, -0.02, 0.03))
        a, out, work = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
        ctx.taylor(a, out, work, zc)
        outs.append(ctx.download(out))
        if n_hamil == 4:
            a, b, w = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
            res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac, trans_longi="tr")
            runs.append((res["curr"].copy(), res["rbox"].copy(), ctx.download(res["psi"])))
        ctx.close()
    assert np.array_equal(outs[0], outs[1])
    if runs:
        for x, y in zip(runs[0], runs[1]):
            assert np.array_equal(x, y)


def _periodic32():
    from salmon2_b200 import synth
    # 2x2x2 supercell of the diamond cell: a periodic 32^3 grid, one k-point
    return synth.periodic_system(a=10.26, num=16, nkgrid=1, no=2, supercell=2, seed=33, name="periodic32")


def test_taylor_parity_periodic32():
    """Periodic grid with nx = 32: the tensor-copy kernel wraps y and z by
    coordinates and x inside the tile."""
    from salmon2_b200 import synth
    sysm = _periodic32()
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    ac = (0.011, -0.007, 0.02)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(sysm.psi), h)
    assert S.rel_err(ctx.download(h), O.hpsi(sysm.psi)) < TOL_H
    zc = synth.taylor_zc(0.08)
    a, out, work = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
    ctx.taylor(a, out, work, zc)
    assert S.rel_err(ctx.download(out), O.taylor(sysm.psi, zc)) < TOL_H


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("make", [S.isolated_small, S.isolated_odd, _periodic32], ids=lambda f: f.__name__)
def test_tensor_copy_kernel_equals_register_sweep(make, precision, monkeypatch):
    """The tensor-copy-fed tiled kernel and the register-prefetch sweep do the
    same arithmetic in the same order: their Taylor steps agree bit for bit."""
    from salmon2_b200 import synth
    sysm = make()
    zc = synth.taylor_zc(0.05)
    outs = []
    for flag in ("on", "off"):
        monkeypatch.setenv("SB200_TMA", flag)
        ctx = _ctx(sysm, precision)
        ctx.set_vec_Ac((0.0, 0.0, 0.02))
        a, out, work = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
        ctx.taylor(a, out, work, zc)
        outs.append(ctx.download(out))
        ctx.close()
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("trans", ["tr", "lo"])
def test_rt_propagate_periodic32_current(trans):
    """32^3 periodic grid: the tensor-copy sweep for H psi and the observables
    z sweep (shared-memory plane + register window) for J(t) and the dipole."""
    from salmon2_b200 import synth
    sysm = _periodic32()
    nt, dt = 8, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    ref = Oracle(sysm).rt_run(sysm.psi, nt, dt, zc, Ac_ext=Ac, trans_longi=1 if trans == "lo" else 0)
    ctx = _ctx(sysm)
    a, b, w = ctx.upload(sysm.psi), ctx.zeros(), ctx.zeros()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac, trans_longi=trans)
    jmax = np.max(np.abs(ref["curr"]))
    assert np.max(np.abs(res["curr"] - ref["curr"])) <= TOL_OBS * jmax
    assert S.rel_err(res["rbox"], ref["rbox"]) < TOL_OBS
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < 1e-11


def test_current_periodic32():
    sysm = _periodic32()
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    a_mid, a_cur = (0.01, 0.02, -0.03), (0.011, 0.019, -0.029)
    O.set_vec_Ac(a_mid)
    ctx.set_vec_Ac(a_mid)
    O.set_vec_Ac_local_only(a_cur)
    ref = O.current(sysm.psi)
    got = ctx.calc_current(ctx.upload(sysm.psi), a_cur)
    assert np.max(np.abs(got - ref)) <= TOL_OBS * max(np.max(np.abs(ref)), 1e-30)


def _p12_twenty_orbitals():
    # 20 orbitals per k-point: one full 16-orbital tile of the tensor-core
    # projection and a partial one
    from salmon2_b200 import synth
    return synth.periodic_system(a=10.26, num=12, nkgrid=1, no=20, seed=45, name="p12n20")


def _p12_two_spins_ten():
    from salmon2_b200 import synth
    return synth.periodic_system(a=10.26, num=12, nkgrid=2, no=10, seed=46, nspin=2, name="p12s2n10")


def _iso_eighteen():
    from salmon2_b200 import synth
    return synth.isolated_system(num=(20, 24, 22), no=18, natom=3, seed=47, name="iso18")


@pytest.mark.parametrize("variant", ["dmma", "warp", "split"])
@pytest.mark.parametrize("make", [_p12_twenty_orbitals, _p12_two_spins_ten, _iso_eighteen, S.periodic_small],
                         ids=lambda f: f.__name__)
def test_projection_forms_against_oracle(make, variant, monkeypatch):
    """The KB projections on the FP64 tensor cores (mma.sync m8n8k4 over
    16-orbital tiles, SB200_PROJECT=dmma), in the warp-per-(orbital, atom)
    form and in the CTA-per-(orbital, atom) form (SB200_PROJECT=split), under
    H psi and a Taylor step, against the oracle: full and partial tiles, two
    spins, isolated grids, fewer orbitals than a tile."""
    from salmon2_b200 import synth
    monkeypatch.setenv("SB200_PROJECT", variant)
    sysm = make()
    O = Oracle(sysm)
    ctx = _ctx(sysm)
    ac = (0.02, -0.01, 0.015) if sysm.grid.periodic else (0.0, 0.0, 0.0)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    t = ctx.upload(sysm.psi)
    h = ctx.zeros()
    ctx.hpsi(t, h)
    assert S.rel_err(ctx.download(h), O.hpsi(sysm.psi)) < TOL_H
    zc = synth.taylor_zc(0.05)
    out, work = ctx.zeros(), ctx.zeros()
    ctx.taylor(ctx.upload(sysm.psi), out, work, zc)
    assert S.rel_err(ctx.download(out), O.taylor(sysm.psi, zc)) < TOL_H


@pytest.mark.parametrize("make,epdir", [(S.isolated_small, (0.0, 0.0, 1.0)), (S.isolated_odd, (0.6, 0.0, 0.8)),
                                        (S.periodic_small, (1.0, 0.0, 0.0))], ids=["iso24_z", "iso_odd", "p12_x"])
def test_impulse_kick_against_oracle(make, epdir):
    """sb200_impulse_kick on the resident block against the oracle's
    restatement of initialization_rt.f90:382-423 (odd and even grid sizes,
    the coordinate conventions of set_gridcoordinate)."""
    sysm = make()
    ctx = _ctx(sysm)
    psi = ctx.upload(sysm.psi)
    ctx.impulse_kick(psi, 1e-3, epdir)
    ref = Oracle(sysm).impulse_kick(sysm.psi, 1e-3, epdir)
    assert S.rel_err(ctx.download(psi), ref) < 1e-15 * 10
