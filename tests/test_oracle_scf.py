"""Known-answer tests of the oracle's per-step potential update (CPU):
the PZ-LDA exchange-correlation against the published Perdew-Zunger (1981)
parametrisation restated independently in numpy, the potential as the density
derivative of the energy, and the periodic Poisson solver on sampled plane
waves (exact for the discrete transform), neutrality and symmetry."""
import numpy as np
import pytest

import oracle as O

# Perdew & Zunger, Phys. Rev. B 23, 5048 (1981), unpolarised fit (Hartree):
# rs >= 1: gamma / (1 + beta1 sqrt(rs) + beta2 rs); rs < 1: A ln rs + B + C rs ln rs + D rs
PZ = dict(gamma=-0.1423, beta1=1.0529, beta2=0.3334, A=0.0311, B=-0.048, C=0.0020, D=-0.0116)
# Slater exchange energy per electron of the uniform gas: -(3/4) (3 rho / pi)^(1/3)


def eps_xc_published(rho):
    rho = np.asarray(rho, dtype=np.float64) + 1e-10  # the reference's regulariser
    rs = (3.0 / (4.0 * np.pi * rho)) ** (1.0 / 3.0)
    ex = -0.75 * (3.0 * rho / np.pi) ** (1.0 / 3.0)
    hi = PZ["gamma"] / (1.0 + PZ["beta1"] * np.sqrt(rs) + PZ["beta2"] * rs)
    lo = PZ["A"] * np.log(rs) + PZ["B"] + PZ["C"] * rs * np.log(rs) + PZ["D"] * rs
    return ex + np.where(rs > 1.0, hi, lo)


def test_pz_energy_matches_published_fit():
    # densities from rs = 0.2 to rs = 20, both branches and rs = 1 itself
    rs = np.concatenate([np.geomspace(0.2, 20.0, 61), [1.0]])
    rho = 3.0 / (4.0 * np.pi * rs ** 3)
    hvol = 0.37
    field = rho.reshape(62, 1, 1)
    v, E = O.exc_cor_pz(field, hvol)
    want = hvol * np.sum(rho * eps_xc_published(rho))
    assert abs(E - want) <= 1e-13 * abs(want)
    # per point: E of a one-point field is hvol * rho * eps_xc
    for r in rho[::7]:
        _, e1 = O.exc_cor_pz(np.full((1, 1, 1), r), 1.0)
        assert abs(e1 - r * eps_xc_published(r)) <= 1e-13 * abs(e1)


def test_pz_branches_meet_at_rs_one():
    # the fit is built continuous at rs = 1 (to the precision of its printed
    # constants): both branches agree to a few 1e-5 Ha
    hi = PZ["gamma"] / (1.0 + PZ["beta1"] + PZ["beta2"])
    lo = PZ["B"] + PZ["D"]
    assert abs(hi - lo) < 1e-4
    rho1 = 3.0 / (4.0 * np.pi)
    eps = 1e-7
    _, ea = O.exc_cor_pz(np.full((1, 1, 1), rho1 * (1 + eps)), 1.0)
    _, eb = O.exc_cor_pz(np.full((1, 1, 1), rho1 * (1 - eps)), 1.0)
    assert abs(ea / (rho1 * (1 + eps)) - eb / (rho1 * (1 - eps))) < 1e-4


@pytest.mark.parametrize("rs", [0.3, 0.7, 1.5, 4.0, 12.0])
def test_pz_potential_is_energy_derivative(rs):
    """Vxc = d(rho eps_xc)/d rho: central differences of E_xc in rho."""
    rho = 3.0 / (4.0 * np.pi * rs ** 3)
    v, _ = O.exc_cor_pz(np.full((1, 1, 1), rho), 1.0)
    h = 1e-5 * rho
    _, ep = O.exc_cor_pz(np.full((1, 1, 1), rho + h), 1.0)
    _, em = O.exc_cor_pz(np.full((1, 1, 1), rho - h), 1.0)
    fd = (ep - em) / (2 * h)
    assert abs(v.ravel()[0] - fd) <= 1e-7 * abs(fd)


def _grid(num, h):
    L = [n * h for n in num]
    xs = [np.arange(n) * h for n in num]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    return L, X, Y, Z


@pytest.mark.parametrize("num,m", [((12, 12, 12), (1, 0, 0)), ((12, 16, 20), (2, -1, 3)),
                                   ((15, 10, 9), (-7, 4, 4)), ((16, 16, 16), (8, 0, 1))])
def test_poisson_sampled_plane_wave(num, m):
    """cos and sin of G.r sampled on the grid are eigenvectors of the
    discrete transform: Vh = 4 pi / |G|^2 times the density."""
    L, X, Y, Z = _grid(num, 0.55)
    brl = O.primitive_b_orthogonal(L)
    G = [2 * np.pi * mi / Li for mi, Li in zip(m, L)]
    ph = G[0] * X + G[1] * Y + G[2] * Z
    G2 = sum(g * g for g in G)
    for rho in (np.cos(ph), np.sin(ph)):
        vh = O.poisson_ft(rho, brl)
        want = 4 * np.pi / G2 * rho
        assert np.max(np.abs(vh - want)) <= 1e-12 * np.max(np.abs(want)) + 1e-14


def test_poisson_neutral_linear_symmetric():
    num = (12, 14, 10)
    L, X, Y, Z = _grid(num, 0.6)
    brl = O.primitive_b_orthogonal(L)
    rng = np.random.default_rng(5)
    # the G = 0 term is dropped: a uniform density has no potential
    assert np.max(np.abs(O.poisson_ft(np.full(num, 0.3), brl))) < 1e-14
    r1 = rng.standard_normal(num)
    r2 = rng.standard_normal(num)
    v1, v2 = O.poisson_ft(r1, brl), O.poisson_ft(r2, brl)
    v12 = O.poisson_ft(r1 + 2.0 * r2, brl)
    assert np.max(np.abs(v12 - (v1 + 2.0 * v2))) <= 1e-12 * np.max(np.abs(v12))
    # the Coulomb kernel is symmetric and positive
    s12, s21 = np.sum(r1 * v2), np.sum(r2 * v1)
    assert abs(s12 - s21) <= 1e-12 * (abs(s12) + np.sum(np.abs(r1 * v2)))
    assert np.sum(r1 * v1) > 0
    # the coefficient table: 4 pi / |G|^2 with folded indices, zero at G = 0
    coef = O.poisson_coef(num, brl).reshape(num, order="F")
    assert coef[0, 0, 0] == 0.0
    kx = np.fft.fftfreq(num[0], d=1.0 / num[0])
    assert np.isclose(coef[num[0] - 1, 0, 0], 4 * np.pi / (2 * np.pi * kx[-1] / L[0]) ** 2, rtol=1e-14)


def test_update_vlocal_is_the_sum():
    rng = np.random.default_rng(6)
    num = (5, 6, 7)
    vpsl, vh = rng.standard_normal(num), rng.standard_normal(num)
    vxc = rng.standard_normal(num + (2,))
    v = O.update_vlocal(vpsl, vh, vxc)
    for s in range(2):
        assert np.array_equal(v[..., s], (vpsl + vh) + vxc[..., s])


@pytest.mark.parametrize("n", [24, 32])
def test_poisson_isolated_gaussian_charge(n):
    """The doubled-box solve of a unit Gaussian charge in the box centre equals
    erf(r / (sqrt(2) s)) / r up to what dropping G = 0 of the doubled cell
    implies: a constant plus the parabola 2 pi/3 * rho_bg * r^2 of the uniform
    background rho_bg = -1 / (8 L^3)."""
    from math import erf
    h = 0.4
    L = n * h
    x = (np.arange(n) - n / 2 + 0.5) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    s = 0.8
    rho = np.exp(-r ** 2 / (2 * s * s)) / (2 * np.pi * s * s) ** 1.5
    v = O.poisson_isolated_ft(rho, O.primitive_b_orthogonal([L, L, L]))
    exact = np.vectorize(lambda q: erf(q / (np.sqrt(2) * s)) / q)(r)
    d = v - exact - 2 * np.pi / 3 * (1.0 / (8 * L ** 3)) * r ** 2
    inner = r < 3.0
    assert np.ptp(d[inner]) < 2e-4 * np.max(exact)
    # odd, unequal extents run too
    rho2 = rho[: n - 1, : n - 2, :]
    v2 = O.poisson_isolated_ft(rho2, O.primitive_b_orthogonal([(n - 1) * h, (n - 2) * h, L]))
    assert v2.shape == rho2.shape and np.all(np.isfinite(v2))


@pytest.mark.parametrize("kind", ["periodic", "isolated"])
def test_rt_run_scf_equals_the_loop_written_out(kind):
    """sbo_rt_run_scf against the self-consistent loop spelled out call by call
    (taylor, calc_density, Hartree, PZ-LDA, update_vlocal) with no field."""
    import dataclasses

    import _systems as S
    from salmon2_b200 import synth

    s = S.periodic_small() if kind == "periodic" else S.isolated_small()
    s = dataclasses.replace(s, V_local=np.array(s.V_local, order="F"))
    g = s.grid
    brl = O.primitive_b_orthogonal([n * h for n, h in zip(g.shape, g.hgs)])
    poisson = O.poisson_ft if g.periodic else O.poisson_isolated_ft
    vpsl = np.array(s.V_local[..., 0])
    zc = synth.taylor_zc(0.05)
    nt = 3

    def potential(rho):
        return O.update_vlocal(vpsl, poisson(rho, brl), O.exc_cor_pz(rho, g.hvol)[0][..., None])

    orc = O.Oracle(s, threads=2)
    v0 = potential(orc.density(s.psi)[..., 0])[..., 0]
    ref = orc.rt_run_scf(s.psi, nt, 0.05, zc, vpsl, brl, v0)
    step = O.Oracle(dataclasses.replace(s, V_local=np.array(s.V_local, order="F")), threads=2)
    step.V[..., 0] = v0
    psi = s.psi
    for _ in range(nt):
        psi = step.taylor(psi, zc)
        step.V[...] = potential(step.density(psi)[..., 0])
    assert np.max(np.abs(ref["psi"] - psi)) <= 1e-13 * np.max(np.abs(psi))
    assert np.max(np.abs(ref["V_local"] - step.V[..., 0])) <= 1e-13 * np.max(np.abs(step.V))


def test_ylm_table_obeys_the_addition_theorem():
    """sum_m Ylm(a) Ylm(b) = P_l(a.b) for unit vectors a, b, l <= 4: the
    normalisation sqrt(4 pi / (2l + 1)) r^l Y_lm of the reference's Ylm
    (salmon_math.f90:386-426) on which the multipole boundary rests."""
    rng = np.random.default_rng(3)
    for _ in range(5):
        a = rng.normal(size=3)
        b = rng.normal(size=3)
        a /= np.linalg.norm(a)
        b /= np.linalg.norm(b)
        c = float(a @ b)
        leg = [1.0, c, (3 * c * c - 1) / 2, (5 * c ** 3 - 3 * c) / 2, (35 * c ** 4 - 30 * c * c + 3) / 8]
        for l in range(5):
            s = sum(O.ylm(*a, l * l + l + m) * O.ylm(*b, l * l + l + m) for m in range(-l, l + 1))
            assert abs(s - leg[l]) < 1e-14


def test_poisson_isolated_cg_gaussian_charge():
    """poisson_isolated_cg on a unit Gaussian charge off the box centre equals
    erf(r / (sqrt(2) s)) / r within 5e-5 of the peak with the origin pole
    (layout 1) and the cells of layout 3; the atom poles of layout 2 split the
    charge over the atoms' Voronoi cells and truncate at l = 4 (1e-2); with the
    threshold at zero the loop runs maxiter times and reports maxiter + 1."""
    from math import erf
    import _systems as S
    from salmon2_b200 import synth
    s = S.no_pp(synth.isolated_system(num=32, h_aa=0.25, no=1, natom=3, seed=5, name="gauss32"))
    g = s.grid
    x = [((np.arange(g.is_[d], g.ie[d] + 1) - (0.5 if g.num[d] % 2 == 0 else 0.0)) * g.hgs[d]) for d in range(3)]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    r = np.sqrt((X - 0.7) ** 2 + (Y + 0.4) ** 2 + (Z - 0.3) ** 2)
    rho = np.exp(-r ** 2 / 2) / (2 * np.pi) ** 1.5
    exact = np.vectorize(lambda q: erf(q / np.sqrt(2.0)) / q)(r)
    orc = O.Oracle(s)
    for layout, tol in ((1, 5e-5), (3, 5e-5), (2, 1e-2)):
        v, it = orc.poisson_isolated_cg(rho, layout=layout)
        assert it < 1000
        assert np.max(np.abs(v - exact)) < tol * np.max(exact)
    v, it = orc.poisson_isolated_cg(rho, layout=3, npole_xyz=(2, 2, 2))
    assert np.max(np.abs(v - exact)) < 5e-5 * np.max(exact)
    _, it = orc.poisson_isolated_cg(rho, threshold=0.0, maxiter=5)
    assert it == 6


def test_rt_run_scf_cg_equals_the_loop_written_out():
    """The isolated self-consistent loop with method_poisson = 'cg' against the
    loop spelled out call by call: Taylor step, density, the Vh extrapolation of
    time_evolution_step.f90:186-198 (none at the first step; 2 Vh_stock1 -
    Vh_stock2 after it, Vh_stock1 kept at the initial Vh through step 2), the
    CG solve from that start, PZ-LDA and update_vlocal."""
    import dataclasses

    import _systems as S
    from salmon2_b200 import synth

    s = S.isolated_small()
    s = dataclasses.replace(s, V_local=np.array(s.V_local, order="F"))
    g = s.grid
    vpsl = np.array(s.V_local[..., 0])
    zc = synth.taylor_zc(0.05)
    nt = 4
    orc = O.Oracle(s, threads=2)
    rho0 = orc.density(s.psi)[..., 0]
    vh0, _ = orc.poisson_isolated_cg(rho0)
    v0 = O.update_vlocal(vpsl, vh0, O.exc_cor_pz(rho0, g.hvol)[0][..., None])[..., 0]
    ref = orc.rt_run_scf(s.psi, nt, 0.05, zc, vpsl, None, v0, cg=dict(vh0=vh0))
    step = O.Oracle(dataclasses.replace(s, V_local=np.array(s.V_local, order="F")), threads=2)
    step.V[..., 0] = v0
    psi, vh, s1, s2 = s.psi, vh0.copy(), vh0.copy(), vh0.copy()
    iters = []
    for itt in range(1, nt + 1):
        psi = step.taylor(psi, zc)
        rho = step.density(psi)[..., 0]
        if itt != 1:
            vh = 2 * s1 - s2
            s2 = s1.copy()
        vh, it = step.poisson_isolated_cg(rho, vh0=vh)
        iters.append(it)
        if itt != 1:
            s1 = vh.copy()
        step.V[...] = O.update_vlocal(vpsl, vh, O.exc_cor_pz(rho, g.hvol)[0][..., None])
    assert list(ref["cg_iters"]) == iters and max(iters) < 1000
    assert np.max(np.abs(ref["psi"] - psi)) <= 1e-13 * np.max(np.abs(psi))
    assert np.max(np.abs(ref["Vh"] - vh)) <= 1e-13 * np.max(np.abs(vh))
    assert np.max(np.abs(ref["V_local"] - step.V[..., 0])) <= 1e-13 * np.max(np.abs(step.V))


def test_spin_polarised_pz_is_the_derivative_of_its_energy_and_meets_the_limits():
    """exc_cor_pz_sp (builtin_pz_sp.f90): Vxc_s = d(rho e_xc)/d rho_s (central
    differences on the two spin densities, both rs branches); at zeta = 0 the
    unpolarised PZ up to the two forms' density offsets (1e-10 against 1e-20);
    at zeta -> 1 the polarised exchange 2^(1/3) e_x plus the polarised
    correlation fit."""
    import oracle as OR
    rng = np.random.default_rng(41)
    up = rng.uniform(0.002, 0.6, (6, 5, 4))
    dn = rng.uniform(0.002, 0.6, (6, 5, 4))
    hv = 0.37
    v, e = OR.exc_cor_pz_sp(np.stack([up, dn], axis=-1), hv)
    for s in range(2):
        h = 1e-6 * (up if s == 0 else dn)
        # the energy is a sum of local terms: move one point's spin density at a time
        for idx in [(0, 0, 0), (3, 2, 1), (5, 4, 3)]:
            dp = [a.copy() for a in (up, dn)]
            dm = [a.copy() for a in (up, dn)]
            dp[s][idx] += h[idx]
            dm[s][idx] -= h[idx]
            Ep = OR.exc_cor_pz_sp(np.stack(dp, axis=-1), 1.0)[1]
            Em = OR.exc_cor_pz_sp(np.stack(dm, axis=-1), 1.0)[1]
            assert abs((Ep - Em) / (2 * h[idx]) - v[idx + (s,)]) < 1e-6 * abs(v[idx + (s,)])
    r = rng.uniform(0.05, 0.6, (4, 4, 4))
    v1, e1 = OR.exc_cor_pz(r, hv)
    v2, e2 = OR.exc_cor_pz_sp(np.stack([r / 2, r / 2], axis=-1), hv)
    assert np.max(np.abs(v2[..., 0] - v1)) < 1e-8 * np.max(np.abs(v1))
    assert np.array_equal(v2[..., 0], v2[..., 1]) and abs(e2 - e1) < 1e-8 * abs(e1)
    # fully polarised: E_xc / (hvol * sum rho) per point from the P fit
    for rho in (0.3, 0.02):  # rs < 1 and rs > 1
        E = OR.exc_cor_pz_sp(np.stack([np.full((1, 1, 1), rho), np.zeros((1, 1, 1))], axis=-1), 1.0)[1]
        t = rho + 1e-20
        rs = (3.0 / (4.0 * np.pi * t)) ** (1.0 / 3.0)
        cx = 0.75 * (3.0 / (2 * np.pi)) ** (2.0 / 3.0)
        if rs > 1:
            ec = -0.0843 / (1.0 + 1.3981 * np.sqrt(rs) + 0.2611 * rs)
        else:
            ec = 0.01555 * np.log(rs) - 0.0269 + 0.0007 * rs * np.log(rs) - 0.0048 * rs
        assert abs(E / t - (-(2.0 ** (1.0 / 3.0)) * cx / rs + ec)) < 1e-9 * abs(E / t)
