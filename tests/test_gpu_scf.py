"""Per-step potential update on the GPU against the oracle: PZ-LDA
exchange-correlation, the periodic Hartree potential (separable transforms)
and update_vlocal, each through the C ABI with host and device arrays, and a
self-consistent time loop (Taylor step, density, Hartree, XC, V_local every
step) against the same loop run by the oracle."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import _systems as S
import oracle as OR
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12        # relative (max-norm) per call, FP64
TOL_LOOP = 1e-10   # relative on the density and orbitals after the loop


def _brl(system):
    g = system.grid
    return OR.primitive_b_orthogonal([n * h for n, h in zip(g.shape, g.hgs)])


def _periodic_box(num, h=0.6, no=2):
    """A periodic system on an arbitrary (non-cubic) grid, without projectors;
    only its grid is used."""
    from salmon2_b200 import synth
    base = S.no_pp(S.periodic_small())
    g = synth.make_grid(list(num), h, periodic=True)
    shp = g.shape_array
    return dataclasses.replace(base, grid=g, no=no, nk=1, vec_k=np.zeros((3, 1), order="F"),
                               rocc=np.asfortranarray(np.full((no, 1, 1), 2.0)), wtk=np.ones(1),
                               V_local=np.zeros(tuple(num) + (1,), order="F"),
                               psi=np.zeros(shp + (1, no, 1), dtype=np.complex128, order="F"),
                               ngrid=int(np.prod(num)))


def _oracle(system):
    """An oracle with its own copy of V_local (the tests rewrite it in place)."""
    return Oracle(dataclasses.replace(system, V_local=np.array(system.V_local, order="F")))


def test_exc_cor_pz_against_oracle():
    import torch
    from salmon2_b200 import _lib
    from salmon2_b200.rt import Context

    s = S.periodic_small()
    ctx = Context(s)
    rho = Oracle(s).density(s.psi)[..., 0]
    rng = np.random.default_rng(7)
    wide = np.exp(rng.uniform(np.log(1e-5), np.log(50.0), rho.shape))  # rs from 0.17 to 29
    for f in (rho, wide):
        v, e = ctx.exc_cor_pz(f)
        vr, er = OR.exc_cor_pz(f, s.grid.hvol)
        assert S.rel_err(v, vr) < TOL
        assert abs(e - er) <= TOL * abs(er)
    # device input and output
    fd = torch.from_numpy(np.ascontiguousarray(wide.ravel(order="F"))).cuda()
    vd = torch.empty_like(fd)
    e = C.c_double(0.0)
    _lib.check(_lib.lib().sb200_exc_cor_pz(ctx.h, C.c_void_p(fd.data_ptr()), C.c_void_p(vd.data_ptr()),
                                           C.byref(e)))
    vr, er = OR.exc_cor_pz(wide, s.grid.hvol)
    assert S.rel_err(vd.cpu().numpy(), vr.ravel(order="F")) < TOL
    assert abs(e.value - er) <= TOL * abs(er)
    ctx.close()


@pytest.mark.parametrize("num", [(12, 12, 12), (16, 16, 16), (12, 16, 20), (15, 9, 10)])
def test_hartree_periodic_against_oracle(num):
    import torch
    from salmon2_b200 import _lib
    from salmon2_b200.rt import Context

    s = S.periodic_small() if num == (12, 12, 12) else _periodic_box(num)
    ctx = Context(s)
    brl = _brl(s)
    rng = np.random.default_rng(sum(num))
    rho = rng.uniform(0.0, 0.2, tuple(num))
    vh = ctx.hartree_periodic(rho, brl)
    ref = OR.poisson_ft(rho, brl)
    assert S.rel_err(vh, ref) < TOL
    # a second call with another cell reuses the transform tables and rebuilds 4 pi / |G|^2
    brl2 = 1.1 * brl
    assert S.rel_err(ctx.hartree_periodic(rho, brl2), OR.poisson_ft(rho, brl2)) < TOL
    # device arrays
    rd = torch.from_numpy(np.ascontiguousarray(rho.ravel(order="F"))).cuda()
    vd = torch.empty_like(rd)
    b = np.asfortranarray(brl)
    _lib.check(_lib.lib().sb200_hartree_periodic(ctx.h, b.ctypes.data_as(C.POINTER(C.c_double)),
                                                 C.c_void_p(rd.data_ptr()), C.c_void_p(vd.data_ptr())))
    assert S.rel_err(vd.cpu().numpy(), ref.ravel(order="F")) < TOL
    ctx.close()


def test_hartree_needs_a_periodic_grid():
    from salmon2_b200.rt import Context, SB200Error

    s = S.isolated_small()
    ctx = Context(s)
    with pytest.raises(SB200Error):
        ctx.hartree_periodic(np.zeros(s.grid.shape), np.eye(3))
    ctx.close()


def test_update_vlocal_feeds_hpsi():
    """After update_vlocal the context's H uses the new potential: H psi
    matches the oracle's H psi with V_local = Vpsl + Vh + Vxc."""
    from salmon2_b200.rt import Context

    s = S.periodic_c2_like()
    O = _oracle(s)
    ctx = Context(s)
    rng = np.random.default_rng(8)
    shp = s.grid.shape
    vpsl = s.V_local[..., 0]
    vh, vxc = rng.standard_normal(shp), rng.standard_normal(shp)
    ctx.update_vlocal(vpsl, vh, vxc)
    O.V[...] = OR.update_vlocal(vpsl, vh, vxc[..., None])
    psi = ctx.upload(s.psi)
    h = ctx.zeros()
    ctx.hpsi(psi, h)
    assert S.rel_err(ctx.download(h), O.hpsi(s.psi)) < TOL
    ctx.close()


def test_self_consistent_time_loop_against_oracle():
    """Four steps of the self-consistent loop of time_evolution_step
    (taylor, calc_density, hartree, exchange_correlation, update_vlocal), with
    the fixed Gaussian local potential standing in for Vpsl: on the GPU through
    Context.update_potential (device arrays only), on the CPU by the oracle."""
    import torch
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context

    s = S.periodic_small()
    O = _oracle(s)
    ctx = Context(s)
    brl = _brl(s)
    zc = synth.taylor_zc(0.05)
    vpsl = np.array(s.V_local[..., 0])
    vpsl_dev = torch.from_numpy(np.ascontiguousarray(vpsl.ravel(order="F"))).cuda()
    a = ctx.upload(s.psi)
    out, work = ctx.zeros(), ctx.zeros()
    psi_ref = s.psi
    for step in range(4):
        ctx.taylor(a, out, work, zc)
        a, out = out, a
        exc = ctx.update_potential(a, vpsl_dev, brl)
        rho = ctx._pot_buf[0].cpu().numpy().reshape(s.grid.shape, order="F")

        psi_ref = O.taylor(psi_ref, zc)
        rho_ref = O.density(psi_ref)[..., 0]
        vh_ref = OR.poisson_ft(rho_ref, brl)
        vxc_ref, exc_ref = OR.exc_cor_pz(rho_ref, s.grid.hvol)
        O.V[...] = OR.update_vlocal(vpsl, vh_ref, vxc_ref[..., None])

        assert S.rel_err(rho, rho_ref) < TOL_LOOP, step
        assert abs(exc - exc_ref) <= TOL_LOOP * abs(exc_ref), step
    assert S.rel_err(ctx.download(a), psi_ref) < TOL_LOOP
    # the potential the next step would use, through the host path of each call
    rho_h = ctx.calc_density(a)[..., 0]
    vh_h = ctx.hartree_periodic(rho_h, brl)
    vxc_h, _ = ctx.exc_cor_pz(rho_h)
    assert S.rel_err(vh_h, OR.poisson_ft(rho_ref, brl)) < TOL_LOOP
    assert S.rel_err(vxc_h, vxc_ref) < TOL_LOOP
    ctx.close()


@pytest.mark.parametrize("make,nt", [(S.periodic_small, 6), (S.periodic_small, 5), (S.periodic_c2_like, 6)],
                         ids=["p12_even", "p12_odd", "p16_fused"])
def test_rt_propagate_self_consistent(make, nt):
    """sb200_rt_propagate with the potential update inside its CUDA graph
    against the oracle's self-consistent loop, under a sin^2-envelope field:
    J(t) and the dipole every step, the final orbitals and V_local.  The
    16^3 system runs the fused Taylor-step kernel, the 12^3 one the sweep."""
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context

    s = make()
    dt = 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    brl = _brl(s)
    vpsl = np.array(s.V_local[..., 0])
    O = _oracle(s)
    rho0 = O.density(s.psi)[..., 0]
    v0 = OR.update_vlocal(vpsl, OR.poisson_ft(rho0, brl), OR.exc_cor_pz(rho0, s.grid.hvol)[0][..., None])[..., 0]
    ref = O.rt_run_scf(s.psi, nt, dt, zc, vpsl, brl, v0, Ac_ext=Ac)

    ctx = Context(s)
    a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
    rho = ctx.calc_density(a)[..., 0]
    vxc, _ = ctx.exc_cor_pz(rho)
    ctx.update_vlocal(vpsl, ctx.hartree_periodic(rho, brl), vxc)
    ctx.set_self_consistent(True, vpsl, brl)
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)
    jmax = np.max(np.abs(ref["curr"]))
    assert jmax > 0
    assert np.max(np.abs(res["curr"] - ref["curr"])) <= TOL_LOOP * jmax
    assert S.rel_err(res["rbox"], ref["rbox"]) < TOL_LOOP
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < TOL_LOOP
    # the potential the loop left behind: H psi with it matches the oracle's
    # (both at A = 0: the oracle's loop leaves its last A(t) set)
    O.V[..., 0] = ref["V_local"]
    O.set_vec_Ac((0.0, 0.0, 0.0))
    ctx.set_vec_Ac((0.0, 0.0, 0.0))
    h = ctx.zeros()
    ctx.hpsi(res["psi"], h)
    assert S.rel_err(ctx.download(h), O.hpsi(ref["psi"])) < TOL_LOOP
    # the fixed-potential loop again after switching the update off
    ctx.set_self_consistent(False)
    ctx.update_vlocal(vpsl, np.zeros_like(vpsl), np.zeros_like(vpsl))
    a2, b2, w2 = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
    res2 = ctx.rt_propagate(a2, b2, w2, 2, dt, zc, Ac_ext=Ac[:, :4])
    ref2 = _oracle(s).rt_run(s.psi, 2, dt, zc, Ac_ext=Ac[:, :4])
    assert S.rel_err(ctx.download(res2["psi"]), ref2["psi"]) < TOL_LOOP
    ctx.close()


def test_rt_propagate_self_consistent_mixed():
    """The mixed form (FP32 terms n >= 2) in the self-consistent loop: the
    update also refreshes the FP32 copy of V_local; J(t) stays within the
    mixed form's budget (1e-6 relative) of the FP64 self-consistent loop."""
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context

    s = S.periodic_small()
    nt, dt = 20, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    brl = _brl(s)
    vpsl = np.array(s.V_local[..., 0])
    out = {}
    for prec in ("fp64", "mixed"):
        ctx = Context(s, precision=prec)
        a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
        ctx.update_potential(a, vpsl, brl)
        ctx.set_self_consistent(True, vpsl, brl)
        out[prec] = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)["curr"]
        ctx.close()
    jmax = np.max(np.abs(out["fp64"]))
    err = np.max(np.abs(out["mixed"] - out["fp64"])) / jmax
    print("self-consistent loop, mixed vs FP64: J(t) rel err %.2e over %d steps" % (err, nt))
    assert 0 < err <= 1e-6


def test_density_comm_single_rank():
    """A one-rank NCCL communicator: calc_density and the self-consistent loop
    with the density all-reduce (inside the loop's CUDA graph) give exactly the
    numbers of the same calls without it."""
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context, nccl_unique_id

    s = S.periodic_small()
    nt, dt = 4, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    brl = _brl(s)
    vpsl = np.array(s.V_local[..., 0])
    got = {}
    for comm in (False, True):
        ctx = Context(s)
        if comm:
            ctx.set_density_comm(1, 0, nccl_unique_id())
        a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
        rho = ctx.calc_density(a)
        ctx.update_potential(a, vpsl, brl)
        ctx.set_self_consistent(True, vpsl, brl)
        r = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)
        got[comm] = (rho, r["curr"], ctx.download(r["psi"]))
        ctx.set_density_comm(0, 0, None)
        ctx.close()
    for x, y in zip(got[False], got[True]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("num", [12, 16], ids=["tiled", "fused16"])
def test_shard_current_sum_single_rank_lo(num):
    """With a shard communicator the loop's finalize runs in two stages around
    an NCCL all-reduce of J(t) and the dipole sums (inside the CUDA graph);
    with one rank that all-reduce is the identity, so J(t), A_tot, the dipole
    and the orbitals of the induced-field ('lo') loop equal those without a
    communicator bit for bit."""
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context, nccl_unique_id

    s = synth.periodic_system(a=10.26, num=num, nkgrid=1, no=3, seed=44, name=f"lo{num}")
    nt, dt = 6, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    got = {}
    for comm in (False, True):
        ctx = Context(s)
        if comm:
            ctx.set_density_comm(1, 0, nccl_unique_id())
        a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
        r = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac, trans_longi="lo")
        got[comm] = (r["curr"], r["Ac_tot"], r["rbox"], ctx.download(r["psi"]))
        ctx.set_density_comm(0, 0, None)
        ctx.close()
    for x, y in zip(got[False], got[True]):
        assert np.array_equal(x, y)
    assert np.max(np.abs(got[True][0])) > 0


@pytest.mark.parametrize("make", [S.isolated_small, S.isolated_odd], ids=["iso24", "iso_odd"])
def test_hartree_isolated_ft_against_oracle(make):
    import torch
    from salmon2_b200 import _lib
    from salmon2_b200.rt import Context

    s = make()
    ctx = Context(s)
    brl = _brl(s)
    rho = Oracle(s).density(s.psi)[..., 0]
    vh = ctx.hartree_isolated_ft(rho, brl)
    ref = OR.poisson_isolated_ft(rho, brl)
    assert S.rel_err(vh, ref) < TOL
    rd = torch.from_numpy(np.ascontiguousarray(rho.ravel(order="F"))).cuda()
    vd = torch.empty_like(rd)
    b = np.asfortranarray(brl)
    _lib.check(_lib.lib().sb200_hartree_isolated_ft(ctx.h, b.ctypes.data_as(C.POINTER(C.c_double)),
                                                    C.c_void_p(rd.data_ptr()), C.c_void_p(vd.data_ptr())))
    assert S.rel_err(vd.cpu().numpy(), ref.ravel(order="F")) < TOL
    ctx.close()


def test_rt_propagate_self_consistent_isolated():
    """The self-consistent loop on an isolated grid after an impulse kick (the
    doubled-box Hartree solve inside the graph) against the oracle's loop:
    dipole every step, final orbitals."""
    import dataclasses as dc
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context

    s0 = S.isolated_small()
    s = dc.replace(s0, psi=synth.impulse_kick(s0.grid, s0.psi, 1e-3))
    nt, dt = 6, 0.05
    zc = synth.taylor_zc(dt)
    brl = _brl(s)
    vpsl = np.array(s.V_local[..., 0])
    O = _oracle(s)
    rho0 = O.density(s.psi)[..., 0]
    v0 = OR.update_vlocal(vpsl, OR.poisson_isolated_ft(rho0, brl),
                          OR.exc_cor_pz(rho0, s.grid.hvol)[0][..., None])[..., 0]
    ref = O.rt_run_scf(s.psi, nt, dt, zc, vpsl, brl, v0)
    ctx = Context(s)
    a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
    ctx.update_potential(a, vpsl, brl)
    ctx.set_self_consistent(True, vpsl, brl)
    res = ctx.rt_propagate(a, b, w, nt, dt, zc)
    d_ref = ref["rbox"][:3] - ref["rbox"][:3, :1]
    d_got = res["rbox"][:3] - res["rbox"][:3, :1]
    assert np.max(np.abs(d_got - d_ref)) <= TOL_LOOP * np.max(np.abs(ref["rbox"][:3]))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < TOL_LOOP
    ctx.close()


def _gaussian_rho(system, centre=(0.7, -0.4, 0.3), sigma=1.0):
    g = system.grid
    x = [((np.arange(g.is_[d], g.ie[d] + 1) - (0.5 if g.num[d] % 2 == 0 else 0.0)) * g.hgs[d]) for d in range(3)]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    r = np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2)
    return np.exp(-r ** 2 / (2 * sigma * sigma)) / (2 * np.pi * sigma * sigma) ** 1.5, r


@pytest.mark.parametrize("make", [S.isolated_small, S.isolated_odd], ids=["iso24", "iso_odd"])
@pytest.mark.parametrize("layout", [1, 2, 3])
def test_hartree_isolated_cg_fixed_iterations_against_oracle(make, layout):
    """25 CG iterations with the threshold at zero (no early exit) from the
    multipole boundary of each layout, on the orbitals' density: the same
    iterate as the oracle's within 1e-10 relative (the per-block sums of the
    dot products are ordered differently from the oracle's serial sums, and
    CG carries those roundings forward)."""
    from salmon2_b200.rt import Context

    s = make()
    ctx = Context(s)
    rho = Oracle(s).density(s.psi)[..., 0]
    npx = (2, 2, 1) if layout == 3 else None
    ref, it_ref = Oracle(s).poisson_isolated_cg(rho, layout=layout, npole_xyz=npx, threshold=0.0, maxiter=25)
    got, it = ctx.hartree_isolated_cg(rho, layout=layout, npole_xyz=npx, threshold=0.0, maxiter=25)
    print(f"CG fixed {s.name} layout {layout}: rel {S.rel_err(got, ref):.3e}")
    assert it == it_ref == 26
    assert S.rel_err(got, ref) < 1e-10
    ctx.close()


@pytest.mark.parametrize("layout", [1, 2, 3])
def test_hartree_isolated_cg_converged_against_oracle(layout):
    """The default threshold (1e-15 per grid point): the same iteration count
    as the oracle (within one) and the same potential within 1e-9 relative;
    device arrays in and out; a second solve started from the first solution
    stops after fewer iterations, as the oracle's does."""
    import torch
    from salmon2_b200 import _lib
    from salmon2_b200.rt import Context

    s = S.isolated_small()
    ctx = Context(s)
    rho = Oracle(s).density(s.psi)[..., 0]
    ref, it_ref = Oracle(s).poisson_isolated_cg(rho, layout=layout)
    got, it = ctx.hartree_isolated_cg(rho, layout=layout)
    print(f"CG converged layout {layout}: iterations {it} (oracle {it_ref}), rel {S.rel_err(got, ref):.3e}")
    assert it_ref <= 1000 and abs(it - it_ref) <= 1
    assert S.rel_err(got, ref) < 1e-9
    rd = torch.from_numpy(np.ascontiguousarray(rho.ravel(order="F"))).cuda()
    vd = torch.zeros_like(rd)
    ri = np.ascontiguousarray(np.asarray(s.rion, dtype=np.float64).reshape(3, -1, order="F").T)
    itc = C.c_int(0)
    _lib.check(_lib.lib().sb200_hartree_isolated_cg(
        ctx.h, C.c_void_p(rd.data_ptr()), C.c_void_p(vd.data_ptr()), layout, 4,
        ri.ctypes.data_as(C.POINTER(C.c_double)), ri.shape[0], None, 1e-15, 1000, C.byref(itc)))
    assert itc.value == it
    assert np.array_equal(vd.cpu().numpy(), got.ravel(order="F"))
    again, it2 = ctx.hartree_isolated_cg(rho, vh0=got, layout=layout)
    again_ref, it2_ref = Oracle(s).poisson_isolated_cg(rho, vh0=ref, layout=layout)
    assert it2 < it and abs(it2 - it2_ref) <= 1
    assert S.rel_err(again, again_ref) < 1e-9 and S.rel_err(again, got) < 1e-7
    ctx.close()


def test_hartree_isolated_cg_gaussian_charge():
    """A unit Gaussian charge off the box centre: the solution equals
    erf(r / (sqrt(2) s)) / r within 5e-5 of its peak (the finite-difference
    Laplacian and the l <= 4 boundary), and the default cells of layout 3 for a
    16 A box (2 per axis) agree with the oracle's rule."""
    from math import erf
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context

    s = S.no_pp(synth.isolated_system(num=32, h_aa=0.25, no=1, natom=2, seed=5, name="gauss32"))
    rho, r = _gaussian_rho(s)
    exact = np.vectorize(lambda q: erf(q / np.sqrt(2.0)) / q)(r)
    ctx = Context(s)
    for layout in (1, 3):
        v, it = ctx.hartree_isolated_cg(rho, layout=layout)
        assert it < 1000
        assert np.max(np.abs(v - exact)) < 5e-5 * np.max(exact)
    assert OR.multipole_cells([64] * 3, [0.25 / 0.52917721067] * 3) == [2, 2, 2]
    ctx.close()


def test_hartree_isolated_cg_refuses_periodic_and_bad_layout():
    from salmon2_b200 import _lib
    from salmon2_b200.rt import Context

    ctx = Context(S.periodic_small())
    rho = np.zeros(S.periodic_small().grid.shape)
    with pytest.raises(_lib.SB200Error):
        ctx.hartree_isolated_cg(rho)
    ctx.close()
    s = S.isolated_small()
    ctx = Context(s)
    with pytest.raises(_lib.SB200Error):
        ctx.hartree_isolated_cg(np.zeros(s.grid.shape), layout=4)
    assert b"layout_multipole" in _lib.lib().sb200_last_error()
    ctx.close()


@pytest.mark.parametrize("nt", [5, 6])
def test_rt_propagate_self_consistent_isolated_cg(nt):
    """The isolated self-consistent loop with method_poisson = 'cg' (the
    reference's default): each step's Hartree potential by CG from the
    extrapolated potential (time_evolution_step.f90:186-198), the solve
    inside the loop's CUDA graph (the odd last step of
    nt = 5 runs outside the graph; the iterations in one cooperative launch
    by default), against the oracle's loop: dipole every step, final
    orbitals."""
    import dataclasses as dc
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context

    s0 = S.isolated_small()
    s = dc.replace(s0, psi=synth.impulse_kick(s0.grid, s0.psi, 1e-3))
    dt = 0.05
    zc = synth.taylor_zc(dt)
    vpsl = np.array(s.V_local[..., 0])
    O = _oracle(s)
    rho0 = O.density(s.psi)[..., 0]
    vh0, _ = O.poisson_isolated_cg(rho0)
    v0 = OR.update_vlocal(vpsl, vh0, OR.exc_cor_pz(rho0, s.grid.hvol)[0][..., None])[..., 0]
    ref = O.rt_run_scf(s.psi, nt, dt, zc, vpsl, None, v0, cg=dict(vh0=vh0))
    assert max(ref["cg_iters"]) < 1000
    ctx = Context(s)
    a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
    ctx.update_vlocal(vpsl, vh0, OR.exc_cor_pz(rho0, s.grid.hvol)[0])
    ctx.set_hartree_cg(vh0)
    ctx.set_self_consistent(True, vpsl, _brl(s))
    res = ctx.rt_propagate(a, b, w, nt, dt, zc)
    d_ref = ref["rbox"][:3] - ref["rbox"][:3, :1]
    d_got = res["rbox"][:3] - res["rbox"][:3, :1]
    print(f"CG loop nt={nt}: iterations {list(ref['cg_iters'])}, dipole response err "
          f"{np.max(np.abs(d_got - d_ref)) / np.max(np.abs(d_ref)):.3e}")
    assert np.max(np.abs(d_got - d_ref)) <= TOL_LOOP * np.max(np.abs(ref["rbox"][:3]))
    assert np.max(np.abs(d_got - d_ref)) <= 1e-8 * np.max(np.abs(d_ref))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < TOL_LOOP
    ctx.close()


@pytest.mark.parametrize("layout", [1, 3])
def test_hartree_isolated_cg_one_launch_equals_two_launch_form(layout, monkeypatch):
    """The CG solve in one cooperative launch (default, grid barriers between
    the two halves of each iteration) against the two-launch form
    (SB200_PCG_PERSISTENT=0) on a 64^3 grid, where the one-launch form runs
    on two blocks per SM: the same iteration count within one and the same
    potential within 1e-10 relative (the per-block partial sums are cut
    differently); then a short isolated self-consistent loop with CG under
    each form: the same orbitals within 1e-10."""
    import dataclasses as dc
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context

    s0 = synth.isolated_system(num=64, h_aa=0.25, no=2, natom=2, seed=9, name="iso64cg")
    s = dc.replace(s0, psi=synth.impulse_kick(s0.grid, s0.psi, 1e-3))
    rho = Oracle(s).density(s.psi)[..., 0]
    out = {}
    for form in ("1", "0"):
        monkeypatch.setenv("SB200_PCG_PERSISTENT", form)
        ctx = Context(s)
        v, it = ctx.hartree_isolated_cg(rho, layout=layout)
        a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
        vpsl = np.array(s.V_local[..., 0])
        ctx.update_vlocal(vpsl, v, OR.exc_cor_pz(rho, s.grid.hvol)[0])
        ctx.set_hartree_cg(v, layout=layout)
        ctx.set_self_consistent(True, vpsl, _brl(s))
        res = ctx.rt_propagate(a, b, w, 4, 0.05, synth.taylor_zc(0.05))
        out[form] = (v, it, ctx.download(res["psi"]))
        ctx.close()
    (v1, it1, p1), (v0, it0, p0) = out["1"], out["0"]
    print(f"CG one launch / two launches, layout {layout}: iterations {it1} / {it0}, "
          f"potential rel {S.rel_err(v1, v0):.3e}, orbitals rel {S.rel_err(p1, p0):.3e}")
    assert it1 < 1000 and abs(it1 - it0) <= 1
    assert S.rel_err(v1, v0) < 1e-10
    assert S.rel_err(p1, p0) < 1e-10


def test_cg_grid_barrier_wait_expires_with_an_error():
    """The one-launch CG solve's grid barrier is a bounded wait: when one block
    of the cooperative grid never arrives (sb200_check_grid_barrier with
    withhold), the others give up after about a second and the call returns
    SB200_ERR_TIMEOUT; the context stays usable: the check then passes and a
    CG solve gives the same potential as before."""
    from salmon2_b200 import _lib
    from salmon2_b200.rt import Context

    s = S.isolated_small()
    ctx = Context(s)
    rho = Oracle(s).density(s.psi)[..., 0]
    v0, it0 = ctx.hartree_isolated_cg(rho)
    assert _lib.lib().sb200_check_grid_barrier(ctx.h, 0) == 0
    rc = _lib.lib().sb200_check_grid_barrier(ctx.h, 1)
    assert rc == 6  # SB200_ERR_TIMEOUT
    assert b"grid barrier" in _lib.lib().sb200_last_error()
    assert _lib.lib().sb200_check_grid_barrier(ctx.h, 0) == 0
    v1, it1 = ctx.hartree_isolated_cg(rho)
    assert it1 == it0 and np.array_equal(v1, v0)
    ctx.close()


def test_exc_cor_pz_spin_polarised_against_oracle():
    """exc_cor_pz_sp on the GPU (nspin = 2: spin densities in, Vxc per spin out)
    against the oracle's restatement, on the orbitals' spin densities and on
    random spin densities over rs 0.17 .. 29 and all polarisations."""
    from salmon2_b200.rt import Context
    s = S.periodic_small(nspin=2)
    ctx = Context(s)
    rho_s = Oracle(s).density(s.psi)
    rng = np.random.default_rng(9)
    wide = np.exp(rng.uniform(np.log(1e-5), np.log(50.0), rho_s.shape))
    wide[..., 1] *= rng.uniform(0.0, 1.0, wide.shape[:3])  # zeta over (0, 1)
    for f in (rho_s, wide):
        v, e = ctx.exc_cor_pz(f)
        vr, er = OR.exc_cor_pz_sp(f, s.grid.hvol)
        assert v.shape == f.shape
        assert S.rel_err(v, vr) < TOL
        assert abs(e - er) <= TOL * abs(er)
    ctx.close()


@pytest.mark.parametrize("kind", ["periodic", "isolated_cg"])
def test_rt_propagate_self_consistent_spin_polarised(kind):
    """The self-consistent loop with nspin = 2 (Hartree of rho_up + rho_dn, the
    spin-polarised PZ, V_local per spin) inside the loop's CUDA graph against
    the oracle's loop: J(t) (periodic) and the dipole every step, the final
    orbitals and the potential left behind."""
    import dataclasses as dc
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    nt = 6
    if kind == "periodic":
        s = S.periodic_small(nspin=2)
        dt = 0.08
        Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)
    else:
        s0 = synth.isolated_system(num=24, no=3, natom=2, seed=15, nspin=2, name="isolated24_sp")
        s = dc.replace(s0, psi=synth.impulse_kick(s0.grid, s0.psi, 1e-3))
        dt, Ac = 0.05, None
    zc = synth.taylor_zc(dt)
    brl = _brl(s)
    vpsl = np.array(s.V_local[..., 0])
    O = _oracle(s)
    rho0_s = O.density(s.psi)
    rho0 = rho0_s[..., 0] + rho0_s[..., 1]
    vxc0 = OR.exc_cor_pz_sp(rho0_s, s.grid.hvol)[0]
    cg = None
    if kind == "periodic":
        vh0 = OR.poisson_ft(rho0, brl)
    else:
        vh0, _ = O.poisson_isolated_cg(rho0)
        cg = dict(vh0=vh0)
    v0 = OR.update_vlocal(vpsl, vh0, vxc0)
    ref = O.rt_run_scf(s.psi, nt, dt, zc, vpsl, brl, v0, Ac_ext=Ac, cg=cg)
    ctx = Context(s)
    a, b, w = ctx.upload(s.psi), ctx.zeros(), ctx.zeros()
    ctx.update_vlocal(vpsl, vh0, vxc0)
    if cg is not None:
        ctx.set_hartree_cg(vh0)
    ctx.set_self_consistent(True, vpsl, brl)
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)
    if kind == "periodic":
        jmax = np.max(np.abs(ref["curr"]))
        assert jmax > 0 and np.max(np.abs(res["curr"] - ref["curr"])) <= TOL_LOOP * jmax
        assert S.rel_err(res["rbox"], ref["rbox"]) < TOL_LOOP
    else:
        d_ref = ref["rbox"][:3] - ref["rbox"][:3, :1]
        d_got = res["rbox"][:3] - res["rbox"][:3, :1]
        assert np.max(np.abs(d_got - d_ref)) <= 1e-8 * np.max(np.abs(d_ref))
    assert S.rel_err(ctx.download(res["psi"]), ref["psi"]) < TOL_LOOP
    O.V[...] = ref["V_local"]
    O.set_vec_Ac((0.0, 0.0, 0.0))
    ctx.set_vec_Ac((0.0, 0.0, 0.0))
    h = ctx.zeros()
    ctx.hpsi(res["psi"], h)
    assert S.rel_err(ctx.download(h), O.hpsi(ref["psi"])) < TOL_LOOP
    ctx.close()
