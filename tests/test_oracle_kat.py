"""Known-answer and property tests of the CPU oracle (CPU only).

These pin the restated arithmetic where the reference's own tests hold no
vectors at the hpsi / taylor boundary: plane-wave eigenvalues of the
finite-difference Bloch operator, the Taylor polynomial on an eigenstate,
Hermiticity of H (stencil + KB), the density sum rule, the plane-wave current
and the dipole of a uniform density.
"""
import dataclasses

import numpy as np
import pytest

import _systems as S
from oracle import Oracle
from salmon2_b200 import synth


def plane_wave_system(num=12, kvec=(0.1, 0.2, -0.05)):
    s = S.no_pp(synth.periodic_system(a=10.26, num=num, nkgrid=1, no=1, seed=3))
    s.V_local[:] = 0.0
    s.vec_k[:, 0] = kvec
    return s


def fd_energy(g, q, kap):
    E = 0.0
    s_ = np.arange(1, 5)
    for d in range(3):
        h = g.hgs[d]
        lam = (synth.CN4[0] + 2 * np.sum(synth.CN4[1:] * np.cos(s_ * q[d] * h))) / h ** 2
        D = 2 * np.sum(synth.BN4 * np.sin(s_ * q[d] * h)) / h
        E += -0.5 * lam + 0.5 * kap[d] ** 2 + kap[d] * D
    return E


def pw(g, m):
    L = g.num * g.hgs
    q = 2 * np.pi * np.asarray(m) / L
    X, Y, Z = np.meshgrid(g.coordinate(0), g.coordinate(1), g.coordinate(2), indexing="ij")
    psi = np.zeros(g.shape_array + (1, 1, 1), complex, order="F")
    psi[g.interior_slices() + (0, 0, 0)] = np.exp(1j * (q[0] * X + q[1] * Y + q[2] * Z)) / np.sqrt(np.prod(L))
    return psi, q


@pytest.mark.parametrize("m", [(0, 0, 0), (1, 2, -3), (5, -4, 6)])
def test_plane_wave_eigenvalue(m):
    s = plane_wave_system()
    O = Oracle(s)
    ac = np.array([0.0, 0.0, 0.03])
    O.set_vec_Ac(ac)
    psi, q = pw(s.grid, m)
    h = O.hpsi(psi)
    sl = s.grid.interior_slices() + (0, 0, 0)
    E = fd_energy(s.grid, q, s.vec_k[:, 0] + ac)
    np.testing.assert_allclose(h[sl], E * psi[sl], rtol=0, atol=1e-13 * np.abs(psi[sl]).max() * max(1, abs(E)))


def test_taylor_on_eigenstate():
    s = plane_wave_system()
    O = Oracle(s)
    psi, q = pw(s.grid, (1, 0, 2))
    E = fd_energy(s.grid, q, s.vec_k[:, 0])
    dt = 0.08
    zc = synth.taylor_zc(dt)
    out = O.taylor(psi, zc)
    factor = 1 + sum(zc[n - 1] * E ** n for n in range(1, 5))
    sl = s.grid.interior_slices() + (0, 0, 0)
    np.testing.assert_allclose(out[sl], factor * psi[sl], rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("make", [S.periodic_small, S.isolated_small, S.isolated_odd], ids=lambda f: f.__name__)
def test_hermiticity(make):
    s = make()
    O = Oracle(s)
    O.set_vec_Ac((0.01, -0.02, 0.015))
    h = O.hpsi(s.psi)
    sl = s.grid.interior_slices()
    a, b = s.psi[sl + (0, 0, 0)], s.psi[sl + (0, 1, 0)]
    ha, hb = h[sl + (0, 0, 0)], h[sl + (0, 1, 0)]
    lhs, rhs = np.vdot(a, hb), np.conj(np.vdot(b, ha))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), np.abs(ha).max())


def test_density_sum_rule():
    s = S.periodic_small()
    O = Oracle(s)
    rho = O.density(s.psi)
    ne = rho.sum() * s.grid.hvol
    # orthonormal orbitals, occupation 2, k-weights summing to 1
    assert abs(ne - 2.0 * s.no) < 1e-10


def test_plane_wave_current():
    s = plane_wave_system()
    O = Oracle(s)
    ac = np.array([0.0, 0.0, 0.02])
    O.set_vec_Ac(ac)
    psi, q = pw(s.grid, (1, -2, 1))
    cur = O.current(psi)[:, 0]
    g = s.grid
    s_ = np.arange(1, 5)
    D = np.array([2 * np.sum(synth.BN4 * np.sin(s_ * q[d] * g.hgs[d])) / g.hgs[d] for d in range(3)])
    kac = s.vec_k[:, 0] + ac
    # J = occ * (kAc * <|psi|^2> + D) summed over the grid, / ngrid
    norm = np.sum(np.abs(psi) ** 2)
    expect = 2.0 * (kac * norm + D * norm) / s.ngrid
    np.testing.assert_allclose(cur, expect, rtol=1e-12, atol=1e-18)


def test_dipole_of_uniform_density():
    s = S.isolated_odd()
    O = Oracle(s)
    rho = np.ones(s.grid.shape + (1,), order="F")
    rb = O.dip(rho)
    g = s.grid
    for d in range(3):
        shift = 0.0 if g.num[d] % 2 == 1 else 0.5
        idx = np.arange(g.is_[d], g.ie[d] + 1) - shift
        expect = idx.sum() * np.prod(g.shape) / g.shape[d]
        assert abs(rb[d] - expect) < 1e-9
    assert rb[3] == np.prod(g.shape)


def test_norm_drift_taylor4():
    """Taylor-4 is not unitary: the norm drifts by O((dt*E)^6) per step."""
    s = S.periodic_small()
    O = Oracle(s)
    dt = 0.02
    out = O.taylor(s.psi, synth.taylor_zc(dt))
    sl = s.grid.interior_slices()
    n0 = np.sum(np.abs(s.psi[sl]) ** 2)
    n1 = np.sum(np.abs(out[sl]) ** 2)
    assert abs(n1 / n0 - 1.0) < 1e-5


def test_rt_run_matches_repeated_taylor():
    s = S.periodic_small()
    nt, dt = 3, 0.08
    Ac = synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 1e-2, tw=nt * dt)
    zc = synth.taylor_zc(dt)
    O = Oracle(s)
    res = O.rt_run(s.psi, nt, dt, zc, Ac_ext=Ac)
    O2 = Oracle(s)
    psi = s.psi
    for itt in range(1, nt + 1):
        O2.set_vec_Ac(0.5 * (Ac[:, itt] + Ac[:, itt - 1]))
        psi = O2.taylor(psi, zc)
        O2.set_vec_Ac_local_only(Ac[:, itt])
        np.testing.assert_allclose(O2.current(psi)[:, 0], res["curr"][:, itt - 1], rtol=1e-12, atol=1e-18)
    np.testing.assert_array_equal(psi, res["psi"])


def test_pp_tables_inside_grid():
    for s in (S.periodic_small(), S.isolated_small(), S.isolated_odd()):
        g, pp = s.grid, s.pp
        for ia in range(pp.natom):
            j = pp.jxyz[:, : pp.mps[ia], ia]
            assert np.all(j >= g.is_[:, None]) and np.all(j <= g.ie[:, None])
        # projectors of each atom are contiguous in ilma (set_lma ordering)
        assert np.all(np.diff(pp.ia_tbl) >= 0)


def test_kinetic_part_and_eigen_energy():
    """hpsi's optional ttpsi (stencil output minus V psi, before the nonlocal
    term) and calc_eigen_energy: H psi unchanged by asking for ttpsi, H psi =
    T psi + V psi + KB psi, esp = Re <psi|H|psi> hvol, E_kin and E_ion_nloc
    the occupation-weighted sums of <psi|T|psi> and <psi|KB|psi>; on a plane
    wave with V = 0 and no projectors T psi is the finite-difference energy
    times psi."""
    s = S.periodic_small()
    O = Oracle(s)
    O.set_vec_Ac((0.01, -0.02, 0.015))
    psi = s.psi
    h, tt = O.hpsi_tt(psi)
    assert np.array_equal(h, O.hpsi(psi))
    sl = s.grid.interior_slices()
    V = s.V_local
    nl = O.zpseudo(psi)
    for io in range(s.no):
        for ik in range(s.nk):
            p = psi[sl + (0, io, ik)]
            rebuilt = tt[sl + (0, io, ik)] + V[..., 0] * p + nl[sl + (0, io, ik)]
            np.testing.assert_allclose(rebuilt, h[sl + (0, io, ik)], rtol=0,
                                       atol=1e-12 * np.abs(h[sl + (0, io, ik)]).max())
    esp, ekin, enl = O.calc_eigen_energy(psi)
    hv = s.grid.hvol
    ref_esp = np.zeros_like(esp)
    ek = en = 0.0
    for ik in range(s.nk):
        for io in range(s.no):
            p = psi[sl + (0, io, ik)]
            ref_esp[io, ik, 0] = np.real(np.vdot(p, h[sl + (0, io, ik)])) * hv
            w = s.rocc[io, ik, 0] * s.wtk[ik]
            ek += w * np.real(np.vdot(p, tt[sl + (0, io, ik)])) * hv
            en += w * np.real(np.vdot(p, nl[sl + (0, io, ik)])) * hv
    np.testing.assert_allclose(esp, ref_esp, rtol=1e-12)
    assert abs(ekin - ek) <= 1e-12 * abs(ek)
    assert abs(enl - en) <= 1e-10 * max(abs(en), 1e-8)
    # plane wave: T psi = E_FD psi
    s2 = plane_wave_system()
    O2 = Oracle(s2)
    O2.set_vec_Ac((0.0, 0.0, 0.03))
    pwv, q = pw(s2.grid, (1, 2, -3))
    _, tt2 = O2.hpsi_tt(pwv)
    sl2 = s2.grid.interior_slices() + (0, 0, 0)
    E = fd_energy(s2.grid, q, s2.vec_k[:, 0] + np.array([0.0, 0.0, 0.03]))
    np.testing.assert_allclose(tt2[sl2], E * pwv[sl2], rtol=0, atol=1e-13 * np.abs(pwv[sl2]).max() * max(1, abs(E)))


@pytest.mark.parametrize("num,epdir", [(24, (0.0, 0.0, 1.0)), ((21, 19, 17), (0.6, 0.0, 0.8))])
def test_impulse_kick_oracle_equals_synth(num, epdir):
    """The oracle's restatement of the impulse kick (initialization_rt.f90:
    382-423 with the coordinates of set_gridcoordinate) equals the
    generator's numpy form, and keeps |psi| point by point."""
    from salmon2_b200 import synth
    s = synth.isolated_system(num=num, no=2, natom=1, seed=61, name="kick")
    O = Oracle(s)
    k = 1e-3
    a = O.impulse_kick(s.psi, k, epdir)
    b = synth.impulse_kick(s.grid, s.psi, k, epdir)
    assert np.max(np.abs(a - b)) <= 1e-15 * np.max(np.abs(b))
    assert np.max(np.abs(np.abs(a) - np.abs(s.psi))) <= 1e-15


def _fcc(a=10.26):
    h = a / 2.0
    return np.array([[0.0, h, h], [h, 0.0, h], [h, h, 0.0]]).T  # columns a1, a2, a3


def test_nonorthogonal_stencil_plane_wave_symbol():
    """The oracle's zstencil_nonorthogonal (stencil.f90:120-214) on a lattice
    plane wave exp(i sum_d theta_d n_d): H psi = lambda psi with the symbol of
    the finite-difference operator, lambda = lap0 - 1/2 sum_d F_d L_d
    - i sum_d Bk_d D_d - 1/2 (F_4 D_z D_y + F_5 D_z D_x + F_6 D_y D_x),
    L_d = sum_s 2 c_s cos(s theta_d) / h_d^2, D_d = 2 i sum_s b_s sin(s theta_d) / h_d
    (the mixed terms are the first-derivative stencil applied twice)."""
    import dataclasses
    import _systems as S
    from salmon2_b200 import synth
    s = S.no_pp(synth.nonorthogonal_system(_fcc(), (10, 12, 14), nkgrid=2, no=1, seed=61, with_pp=False))
    s = dataclasses.replace(s, V_local=np.zeros_like(s.V_local))
    g = s.grid
    nums = np.array(g.shape)
    m = np.array([2, -3, 5])
    th = 2 * np.pi * m / nums
    n = np.meshgrid(*[np.arange(k) for k in nums], indexing="ij")
    pw = np.exp(1j * (th[0] * n[0] + th[1] * n[1] + th[2] * n[2]))
    psi = np.zeros_like(s.psi)
    sl = g.interior_slices()
    for ik in range(s.nk):
        psi[sl + (0, 0, ik)] = pw
    O = Oracle(s)
    ac = (0.011, -0.02, 0.017)
    O.set_vec_Ac(ac)
    hp = O.hpsi(psi)
    lat = s.lattice
    F = lat.coef_F
    c = synth.CN4
    b = synth.BN4
    L = np.array([sum(2 * c[k] * np.cos(k * th[d]) for k in range(1, 5)) / g.hgs[d] ** 2 for d in range(3)])
    D = np.array([2j * sum(b[k - 1] * np.sin(k * th[d]) for k in range(1, 5)) / g.hgs[d] for d in range(3)])
    for ik in range(s.nk):
        kac = s.vec_k[:, ik] + np.array(ac)
        lap0 = g.coef_lap0 + 0.5 * kac @ kac
        bk = lat.rmatrix_B @ kac
        lam = (lap0 - 0.5 * (F[:3] @ L) - 1j * (bk @ D)
               - 0.5 * (F[3] * D[2] * D[1] + F[4] * D[2] * D[0] + F[5] * D[1] * D[0]))
        got = hp[sl + (0, 0, ik)]
        assert np.max(np.abs(got - lam * pw)) <= 1e-12 * np.max(np.abs(lam))


def test_nonorthogonal_path_on_a_cubic_cell_equals_the_orthogonal_stencil():
    """A cubic cell taken through the non-orthogonal branch (F = (1, 1, 1, 0,
    0, 0), B = 1) gives the orthogonal branch's H psi, KB term included."""
    import dataclasses
    from salmon2_b200 import synth
    s = synth.nonorthogonal_system(np.diag([8.0, 8.0, 8.0]), 12, nkgrid=2, no=2, seed=62)
    ortho = dataclasses.replace(s, lattice=None)
    a, b = Oracle(s), Oracle(ortho)
    for ac in ((0.0, 0.0, 0.0), (0.03, -0.01, 0.02)):
        a.set_vec_Ac(ac)
        b.set_vec_Ac(ac)
        ha, hb = a.hpsi(s.psi), b.hpsi(s.psi)
        assert np.max(np.abs(ha - hb)) <= 1e-13 * np.max(np.abs(hb))


def test_micro_ac_stencil_with_uniform_field_equals_the_macroscopic_stencil():
    """zstencil_microAc with Ac(r) = A0 everywhere and div A = 0 is the
    orthogonal stencil with vec_Ac = A0: |k + A0|^2 / 2 joins lap0 and (k + A0)
    weights the gradient (hamiltonian.f90:146-155); KB term included."""
    s = S.periodic_small()
    a0 = np.array([0.021, -0.013, 0.034])
    O1, O2 = Oracle(s), Oracle(s)
    O1.set_vec_Ac(a0)
    O2.set_vec_Ac(a0)
    g = s.grid
    O2.set_micro_ac(np.asfortranarray(np.broadcast_to(a0[:, None, None, None], (3,) + g.shape)),
                    np.zeros(g.shape, order="F"))
    h1, h2 = O1.hpsi(s.psi), O2.hpsi(s.psi)
    assert np.max(np.abs(h1 - h2)) <= 1e-13 * np.max(np.abs(h1))


def test_micro_ac_stencil_divergence_term():
    """The -i div(A) psi / 2 term: two fields differing only in div A give
    H psi differing by exactly -i (d1 - d2) psi / 2."""
    s = S.no_pp(S.periodic_small())
    g = s.grid
    rng = np.random.default_rng(7)
    acm = np.asfortranarray(rng.uniform(-0.02, 0.02, (3,) + g.shape))
    d1 = np.asfortranarray(rng.uniform(-0.1, 0.1, g.shape))
    O1, O2 = Oracle(s), Oracle(s)
    O1.set_micro_ac(acm, d1)
    O2.set_micro_ac(acm, np.zeros(g.shape, order="F"))
    h1, h2 = O1.hpsi(s.psi), O2.hpsi(s.psi)
    sl = g.interior_slices()
    for ik in range(s.nk):
        for io in range(s.no):
            diff = (h1 - h2)[sl + (0, io, ik)]
            assert np.max(np.abs(diff - (-0.5j) * d1 * s.psi[sl + (0, io, ik)])) <= 1e-13 * np.max(np.abs(h1))


def _micro_field(shape, seed, amp=0.03):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.uniform(-amp, amp, (3,) + tuple(shape)))


def test_symmetrized_micro_ac_stencil_with_uniform_field_equals_the_plain_form():
    """zstencil_microAc_symmetrized with Ac(r) = A0: the divergence of (k + A0)
    psi is (k + A0).grad psi, so -(i/2)(kAc.w + x) = -i kAc.w, the plain
    zstencil_microAc with div A = 0 (stencil.f90:319-411 against :295-315)."""
    s = S.periodic_small()
    g = s.grid
    a0 = np.array([0.021, -0.013, 0.034])
    field = np.asfortranarray(np.broadcast_to(a0[:, None, None, None], (3,) + g.shape))
    O1, O2 = Oracle(s), Oracle(s)
    O1.set_micro_ac(field, np.zeros(g.shape, order="F"))
    O2.set_micro_ac(field, None, symmetrized=True)
    h1, h2 = O1.hpsi(s.psi), O2.hpsi(s.psi)
    assert np.max(np.abs(h1 - h2)) <= 1e-13 * np.max(np.abs(h1))


def _hermitian_defect(O, s, phi, psi):
    """max over orbitals of |<phi|H psi> - conj(<psi|H phi>)| / |<phi|H psi>|-scale"""
    sl = s.grid.interior_slices()
    hpsi, hphi = O.hpsi(psi), O.hpsi(phi)
    worst, scale = 0.0, 0.0
    for o in np.ndindex(*psi.shape[3:]):
        a = np.vdot(phi[sl + o], hpsi[sl + o])
        b = np.conj(np.vdot(psi[sl + o], hphi[sl + o]))
        worst = max(worst, abs(a - b))
        scale = max(scale, np.linalg.norm(phi[sl + o]) * np.linalg.norm(hpsi[sl + o]))
    return worst / scale


def test_symmetrized_micro_ac_stencil_is_hermitian():
    """With a non-uniform A(r) on a periodic grid the symmetrized operator is
    Hermitian to rounding ((k + A).D + D (k + A) is real antisymmetric for the
    antisymmetric difference D), while the plain form is not (A D - D A)."""
    s = S.periodic_small()
    g = s.grid
    field = _micro_field(g.shape, 21)
    rng = np.random.default_rng(22)
    phi = np.asfortranarray(rng.standard_normal(s.psi.shape) + 1j * rng.standard_normal(s.psi.shape))
    Os, Op = Oracle(s), Oracle(s)
    Os.set_micro_ac(field, None, symmetrized=True)
    Op.set_micro_ac(field, np.zeros(g.shape, order="F"))
    assert _hermitian_defect(Os, s, phi, s.psi) < 1e-14
    assert _hermitian_defect(Op, s, phi, s.psi) > 1e-6


def test_microscopic_current_of_lattice_plane_waves():
    """calc_microscopic_current (density_matrix.f90:726-845) of orbitals
    c_o exp(i q_o.r), q on the grid: D psi = i psi sum_s 2 nab(s) sin(q s h),
    so j_d(r) = sum_o rocc wtk |c_o|^2 (sum_s 2 nab(s,d) sin(q_d s h_d) + k_d)
    at every point."""
    s = S.periodic_small(nspin=2)
    g = s.grid
    rng = np.random.default_rng(23)
    psi = np.zeros(s.psi.shape, dtype=np.complex128, order="F")
    sl = g.interior_slices()
    X = np.meshgrid(*[g.coordinate(d) for d in range(3)], indexing="ij")
    want = np.zeros(3)
    for ik in range(s.nk):
        for io in range(s.no):
            for isp in range(s.nspin):
                m = rng.integers(-3, 4, 3)
                q = 2 * np.pi * m / (g.num * g.hgs)
                c = rng.uniform(0.2, 1.0) * np.exp(1j * rng.uniform(0, 2 * np.pi))
                psi[sl + (isp, io, ik)] = c * np.exp(1j * (q[0] * X[0] + q[1] * X[1] + q[2] * X[2]))
                w = s.rocc[io, ik, isp] * s.wtk[ik]
                for d in range(3):
                    sfac = sum(2 * g.coef_nab[j, d] * np.sin(q[d] * (j + 1) * g.hgs[d]) for j in range(4))
                    want[d] += w * abs(c) ** 2 * (sfac + s.vec_k[d, ik])
    cur = Oracle(s).microscopic_current(psi)
    assert cur.shape == (3,) + g.shape
    for d in range(3):
        assert np.max(np.abs(cur[d] - want[d])) <= 1e-12 * max(1.0, np.max(np.abs(want)))


def test_absorbing_boundary_adds_minus_i_w_psi_on_the_edge_planes():
    """add_imaginary_potential_for_absorbing_boundary_z: hpsi with the absorbing
    boundary minus hpsi without is -i w(z) psi, w = w0 (dr - z)/dr for z <= dr,
    w0 (z - (L - dr))/dr for z >= L - dr, zero between (z = iz hgs(3))."""
    s = S.periodic_small()
    g = s.grid
    w0, dr = 0.3, 2.0
    L = float(g.num[2] * g.hgs[2])
    O1, O2 = Oracle(s), Oracle(s)
    O2.set_absorbing_boundary(w0, dr)
    h1, h2 = O1.hpsi(s.psi), O2.hpsi(s.psi)
    sl = g.interior_slices()
    z = np.arange(g.is_[2], g.ie[2] + 1) * g.hgs[2]
    w = np.where(z <= dr, w0 * (dr - z) / dr, np.where(z >= L - dr, w0 * (z - (L - dr)) / dr, 0.0))
    assert np.count_nonzero(w) >= 4 and np.count_nonzero(w == 0) >= 4
    d = (h2 - h1)[sl]
    want = -1j * w[None, None, :, None, None, None] * s.psi[sl]
    assert np.max(np.abs(d - want)) <= 1e-13 * np.max(np.abs(h1))


def test_length_gauge_with_a_constant_field_is_a_static_potential():
    """calcVbox: with Ac_ext(t) = -E t (a constant E = -dA/dt), every step takes
    V_local + E.r; the loop equals the fixed-potential loop with that potential
    built here from lg%coordinate (odd and even extents)."""
    import dataclasses as dc
    from salmon2_b200 import synth
    for s in (S.isolated_small(), S.isolated_odd()):
        g = s.grid
        nt, dt = 3, 0.05
        E = np.array([0.02, -0.01, 0.03])
        Ac = np.asfortranarray(-E[:, None] * (np.arange(nt + 2) * dt)[None, :])
        zc = synth.taylor_zc(dt)
        O = Oracle(s)
        O.set_length_gauge(True)
        a = O.rt_run(s.psi, nt, dt, zc, Ac_ext=Ac)
        X = np.meshgrid(*[g.coordinate(d) for d in range(3)], indexing="ij")
        vb = E[0] * X[0] + E[1] * X[1] + E[2] * X[2]
        s2 = dc.replace(s, V_local=np.asfortranarray(s.V_local + vb[..., None]))
        b = Oracle(s2).rt_run(s.psi, nt, dt, zc)
        assert np.max(np.abs(a["psi"] - b["psi"])) <= 1e-12 * np.max(np.abs(b["psi"]))
        assert np.max(np.abs(a["rbox"] - b["rbox"])) <= 1e-12 * np.max(np.abs(b["rbox"]))


def test_aetrs_step_with_a_static_hamiltonian_is_two_half_steps():
    """propagator = 'aetrs': with no field and a fixed potential the
    extrapolated V equals V and A(itt+1) equals A(itt), so a step is two
    applications of the half-step Taylor series (zc of -i dt/2)."""
    from salmon2_b200 import synth
    s = S.isolated_small()
    dt = 0.05
    zh = synth.taylor_zc(dt, aetrs=True)
    O = Oracle(s)
    want = O.taylor(O.taylor(s.psi, zh), zh)
    O.set_propagator("aetrs")
    got = O.rt_run(s.psi, 1, dt, zh)["psi"]
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))


def test_predictor_corrector_averages_the_potentials():
    """predictor_corrector with a fixed potential: V = (V_tmp + V0) / 2.  Without
    a field V_tmp = V0 and the loop is the plain one exactly; in the length
    gauge V_tmp = V0 + E.r, so the loop is the length-gauge loop of half the
    field."""
    from salmon2_b200 import synth
    s = S.isolated_small()
    nt, dt = 3, 0.05
    zc = synth.taylor_zc(dt)
    O1, O2 = Oracle(s), Oracle(s)
    O2.set_predictor_corrector(True)
    a, b = O1.rt_run(s.psi, nt, dt, zc), O2.rt_run(s.psi, nt, dt, zc)
    assert np.array_equal(a["psi"], b["psi"]) and np.array_equal(a["rbox"], b["rbox"])
    Ac = synth.asin2cos(nt, dt, omega=0.2, f0=0.05, tw=nt * dt, epdir=(0.3, -0.2, 0.93))
    O3, O4 = Oracle(s), Oracle(s)
    O3.set_length_gauge(True)
    O3.set_predictor_corrector(True)
    O4.set_length_gauge(True)
    c = O3.rt_run(s.psi, nt, dt, zc, Ac_ext=Ac)
    d = O4.rt_run(s.psi, nt, dt, zc, Ac_ext=np.asfortranarray(0.5 * Ac))
    assert np.max(np.abs(c["psi"] - d["psi"])) <= 1e-12 * np.max(np.abs(d["psi"]))


def test_gram_schmidt_interval_in_the_loop():
    """gram_schmidt every N steps of the loop (time_evolution_step.f90:149-152):
    the orbitals leave an N-step loop orthonormal (hvol metric) when N divides
    the step count, and a loop of N - 1 steps is the plain loop exactly."""
    from salmon2_b200 import synth
    s = S.periodic_small()
    g = s.grid
    dt = 0.02
    zc = synth.taylor_zc(dt)
    psi0 = s.psi * 1.3  # not normalised: the Gram-Schmidt step shows
    O1, O2 = Oracle(s), Oracle(s)
    O2.set_gram_schmidt_interval(3)
    a = O1.rt_run(psi0, 2, dt, zc)
    b = O2.rt_run(psi0, 2, dt, zc)
    assert np.array_equal(a["psi"], b["psi"])
    c = O2.rt_run(psi0, 3, dt, zc)["psi"][g.interior_slices()]
    for ik in range(s.nk):
        M = c[..., 0, :, ik].reshape(-1, s.no, order="F")
        G = g.hvol * (M.conj().T @ M)
        assert np.max(np.abs(G - np.eye(s.no))) < 1e-12
