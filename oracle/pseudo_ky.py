"""CPU oracle (TEST INFRASTRUCTURE ONLY) for the set-up of the Kleinman-Bylander
tables from pseudopotential files with one projector per l (Yabana-Bertsch
`_rps.dat` 'KY', ABINIT `.pspnc`, ABINITFHI `.fhi`, FHI98PP `.cpi`):
a numpy restatement of read_ps_KY (src/atom/pp/input_pp.f90:288-341),
read_ps_abinit (:343-400), read_ps_abinitfhi (:402-496), read_ps_fhi
(:614-684), init_pp's choice by file name (src/atom/pp/salmon_pp.f90:66-100),
the masking filter (making_ps_with_masking, ps_masking, make_mask_function,
input_pp.f90:848-1016,1302-1542, with xjl of src/math/salmon_math.f90:289-335), the
radial domain and KB norms of input_pp (:96-193), making_ps_without_masking
(:1111-1240), init_ps's calc_nps / calc_jxyz / set_lma / calc_uv
(src/atom/pp/prep_pp.f90:22-525), calc_Vpsl_isolated (:550-620),
calc_Vpsl_periodic (:798-974, with the transform tables of
src/common/initialization.f90:632-784) and the natural
cubic spline of src/math/salmon_math.f90:500-584 (its linear system solved, as
the reference does, through the LU inverse of the dense matrix).  Arrays keep
the reference's 1-based / 0-based index conventions in comments.

Parity status: unpinned against reference outputs (the Fortran set-up cannot be
run here); the spline is checked by its defining properties in
tests/test_pseudo_ky.py (it passes through the nodes, first and second
derivatives continuous, natural end conditions, straight lines exact).
"""
from __future__ import annotations

import numpy as np

AU_LENGTH_AA = 0.52917721067   # src/io/inputoutput.f90:27
AU_ENERGY_EV = 27.21138505     # src/io/inputoutput.f90:26


def ylm(x, y, z, l, m):
    """Ylm polynomials (src/math/salmon_math.f90:386-426), l <= 3."""
    r2 = x * x + y * y + z * z
    tab = {
        (0, 0): lambda: np.ones_like(x),
        (1, -1): lambda: -y, (1, 0): lambda: z, (1, 1): lambda: -x,
        (2, -2): lambda: np.sqrt(3.0) * x * y, (2, -1): lambda: -np.sqrt(3.0) * y * z,
        (2, 0): lambda: (3.0 * z * z - r2) / 2.0, (2, 1): lambda: -np.sqrt(3.0) * x * z,
        (2, 2): lambda: np.sqrt(3.0 / 4.0) * (x * x - y * y),
        (3, -3): lambda: -np.sqrt(5.0 / 8.0) * y * (3 * x * x - y * y),
        (3, -2): lambda: np.sqrt(15.0) * x * y * z,
        (3, -1): lambda: -np.sqrt(3.0 / 8.0) * y * (5.0 * z * z - r2),
        (3, 0): lambda: z * (5.0 * z * z - 3 * r2) / 2.0,
        (3, 1): lambda: -np.sqrt(3.0 / 8.0) * x * (5.0 * z * z - r2),
        (3, 2): lambda: np.sqrt(15.0 / 4.0) * z * (x * x - y * y),
        (3, 3): lambda: -np.sqrt(5.0 / 8.0) * x * (x * x - 3.0 * y * y),
    }
    return tab[(l, m)]()


def spline(xn, yn):
    """salmon_math.f90:500-584: coefficients an, bn, cn, dn of the Np - 1
    intervals (y = a dx^3 + b dx^2 + c dx + d on interval i)."""
    Np = len(xn)
    n = Np - 2
    dxn = np.diff(xn)
    dyn = np.diff(yn)
    v = np.array([6.0 * (dyn[i] / dxn[i] - dyn[i - 1] / dxn[i - 1]) for i in range(1, n + 1)])
    A = np.zeros((n, n))
    for i in range(1, n + 1):
        A[i - 1, i - 1] = 2.0 * (dxn[i] + dxn[i - 1])
        if i < n:
            A[i - 1, i] = dxn[i]
        if i > 1:
            A[i - 1, i - 2] = dxn[i - 1]
    u = np.zeros(Np)
    u[1:n + 1] = np.linalg.inv(A) @ v
    bn = 0.5 * u[:Np - 1]
    an = (u[1:Np] - 2.0 * bn) / (6.0 * dxn)
    dn = np.asarray(yn[:Np - 1], dtype=np.float64)
    cn = dyn / dxn - dxn * (u[1:Np] + 2.0 * u[:Np - 1]) / 6.0
    return an, bn, cn, dn


class _Records:
    """Fortran list-directed input: every read starts at a new line and drops
    the rest of the last line it used; D exponents accepted."""

    def __init__(self, path):
        with open(path) as f:
            self.lines = f.read().split("\n")
        self.i = 0

    def skip(self):
        if self.i >= len(self.lines):
            raise EOFError
        self.i += 1

    def read(self, n):
        out = []
        while len(out) < n:
            if self.i >= len(self.lines):
                raise EOFError
            toks = self.lines[self.i].replace(",", " ").split()
            self.i += 1
            for t in toks:
                if len(out) == n:
                    break
                out.append(float(t.replace("D", "E").replace("d", "E")))
        return out


def _read_ky(el, path, nrmax):
    """read_ps_KY (input_pp.f90:288-341): angstrom / eV, linear grid."""
    with open(path) as f:
        tok = f.read().split()
    it = iter(tok)
    el.mr = int(next(it))
    step = float(next(it))
    mlps = int(next(it))
    el.zps = float(int(float(next(it)) + 1e-10))
    next(it)                                       # irPC
    rrc = np.array([float(next(it)) for _ in range(mlps + 1)])
    nr = max(nrmax, el.mr)
    el.vpp = np.zeros((nr + 1, mlps + 1))          # vpp(0:nr, 0:mlps)
    el.upp = np.zeros((nr + 1, mlps + 1))
    for i in range(el.mr + 1):
        next(it), next(it)                         # r, rhopp
        for l in range(mlps + 1):
            el.vpp[i, l] = float(next(it))
    for i in range(el.mr + 1):
        next(it)
        for l in range(mlps + 1):
            el.upp[i, l] = float(next(it))
    step = step / AU_LENGTH_AA
    rrc = rrc / AU_LENGTH_AA
    el.vpp[: el.mr + 1] /= AU_ENERGY_EV
    el.upp[: el.mr + 1] *= np.sqrt(AU_LENGTH_AA)
    el.rad = np.array([(i - 1) * step for i in range(1, nrmax + 2)])   # rad(i) at [i - 1]
    return mlps, rrc


def _read_abinit(el, path, nrmax):
    """read_ps_abinit (input_pp.f90:343-400), ABINIT format 1 (.pspnc)."""
    R = _Records(path)
    R.skip()
    zatom, zion, pspdat = R.read(3)
    el.zps = float(int(zion + 1e-10))
    pspcod, pspxc, lmaxabinit, lloc, mmax, r2well = R.read(6)
    mlps, mmax = int(lmaxabinit), int(mmax)
    el.mr = mmax - 1
    rrc = np.zeros(mlps + 1)
    for ll in range(mlps + 1):
        rrc[ll] = R.read(5)[4]
        R.read(4)
    R.read(3)
    nr = max(nrmax, el.mr)
    el.vpp = np.zeros((nr + 1, mlps + 1))
    el.upp = np.zeros((nr + 1, mlps + 1))
    for t in (el.vpp, el.upp):
        for ll in range(mlps + 1):
            R.skip()
            for i in range(1, (el.mr + 1) // 3 + 1):
                t[3 * (i - 1): 3 * (i - 1) + 3, ll] = R.read(3)
    el.rad = np.array([1.0e2 * (i / (mmax - 1) + 1.0e-2) ** 5 - 1.0e-8 for i in range(nrmax + 1)])
    return mlps, rrc


def _read_fhi(el, path, nrmax, abinit):
    """read_ps_abinitfhi (input_pp.f90:402-496, .fhi) and read_ps_fhi
    (:614-684, .cpi)."""
    R = _Records(path)
    if abinit:
        for _ in range(7):
            R.skip()
    rzps, m = R.read(2)
    el.zps = float(int(rzps + 1e-10))
    mlps = int(m) - 1
    for _ in range(10):
        R.read(1)
    mr_l, step_l = [], []
    rad = None
    for l in range(mlps + 1):
        a, b = R.read(2)
        mr_l.append(int(a))
        step_l.append(b)
        if rad is None:
            nr = max(nrmax, mr_l[0])
            rad = np.zeros(nr + 2)                 # rad(i) at [i - 1]
            el.vpp = np.zeros((nr + 1, mlps + 1))
            el.upp = np.zeros((nr + 1, mlps + 1))
        for i in range(1, mr_l[l] + 1):
            j, r, u, v = R.read(4)
            rad[i] = r
            el.upp[i, l] = u
            el.vpp[i, l] = v
        rad[0] = 0.0
        el.upp[0, l] = 0.0
        el.vpp[0, l] = el.vpp[1, l] - (el.vpp[2, l] - el.vpp[1, l]) / (rad[2] - rad[1]) * rad[1]
    if abinit:
        try:
            for i in range(1, mr_l[0] + 1):
                rad[i] = R.read(4)[0]
        except EOFError:
            pass
    assert min(mr_l) == max(mr_l) and max(step_l) - min(step_l) < 1e-14
    el.mr = mr_l[0]
    step = min(step_l)
    for i in range(el.mr + 1, (nrmax - 1 if abinit else nrmax) + 1):
        rad[i] = rad[i - 1] * step
    rrc = np.zeros(mlps + 1)
    for l in range(mlps + 1):
        best = -1.0
        for ll in range(mlps + 1):
            rm = -1.0
            for i in range(el.mr, 0, -1):
                if abs(el.vpp[i, l] - el.vpp[i, ll]) > 1e-10:
                    rm = rad[i + 1]
                    break
            best = max(best, rm)
        rrc[l] = best
    el.rad = rad
    return mlps, rrc


def _format_of(path):
    """init_pp's choice by file name (salmon_pp.f90:66-100)."""
    p = str(path)
    for suffix, fmt in (("_rps.dat", "KY"), (".pspnc", "ABINIT"), (".fhi", "ABINITFHI"), (".cpi", "FHI")):
        if p.endswith(suffix):
            return fmt
    raise ValueError("unsupported pseudopotential file " + p)


def _seqsum(a, axis):
    """left-to-right sum (the reference's loop order)"""
    return np.take(np.cumsum(a, axis=axis), -1, axis=axis)


def xjl(x, l):
    """x j_l(x) (salmon_math.f90:289-335): closed forms, Taylor series below 0.1."""
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        s, c = np.sin(x), np.cos(x)
        big = {0: s, 1: (1.0 / x) * s - c, 2: (3.0 / x ** 2 - 1.0) * s - (3.0 / x) * c,
               3: (15.0 / x ** 3 - 6.0 / x) * s - (15.0 / x ** 2 - 1.0) * c}[l]
    small = {0: x - x ** 3 / 6.0 + x ** 5 / 120.0 - x ** 7 / 5040.0 + x ** 9 / 362880.0,
             1: (2.0 / 6.0) * x ** 2 - (2.0 / 60.0) * x ** 4 + (1.0 / 840.0) * x ** 6 - (2.0 / 90720.0) * x ** 8,
             2: (4.0 / 60.0) * x ** 3 - (4.0 / 840.0) * x ** 5 + (2.0 / 15120.0) * x ** 7 - (2.0 / 997920.0) * x ** 9,
             3: (8.0 / 840.0) * x ** 4 - (8.0 / 15120.0) * x ** 6 + (4.0 / 332640.0) * x ** 8}[l]
    return np.where(x < 0.1, small, big)


def make_mask(rad, nrps, rps, eta):
    """make_mask_function (input_pp.f90:1437-1542); rmask[i - 1] at rad(i).
    numpy's symmetric eigensolver stands in for LAPACK dsyev."""
    M = 200
    x = np.arange(1, M + 1) / M
    mat = np.zeros((M, M))
    for i in range(M):
        xp = 2.0 * x[i]
        mat[i, i] = np.sin(xp * eta) / xp + M * np.pi - eta
        for j in range(i + 1, M):
            a, b = x[i] + x[j], x[i] - x[j]
            mat[i, j] = mat[j, i] = np.sin(a * eta) / a - np.sin(b * eta) / b
    w, V = np.linalg.eigh(mat)
    u = V[:, 0]
    n0 = 3.0 * u[0] / x[0] - 3.0 * u[1] / x[1] + u[2] / x[2]
    nm = u / x / n0
    k = np.pi * np.arange(1, M + 1)
    dx = x[1] - x[0]
    kx = k[:, None] * x[None, :]
    nmk = _seqsum(nm[None, :] * kx * np.sin(kx), 1) * dx / k ** 2
    dk = k[1] - k[0]
    rmask = np.zeros(nrps)
    r = rad[1:nrps]
    kx = k[None, :] * r[:, None] / rps
    rmask[1:] = (2.0 / np.pi) * _seqsum(nmk[None, :] * kx * np.sin(kx), 1) * dk * rps ** 2 / r ** 2
    rmask[0] = rmask[1] - (rmask[2] - rmask[1]) / (rad[2] - rad[1]) * (rad[1] - rad[0])
    i1, i2, i3 = nrps - 2, nrps - 1, nrps
    rmask[i3 - 1] = rmask[i2 - 1] + (rmask[i2 - 1] - rmask[i1 - 1]) / (rad[i2 - 1] - rad[i1 - 1]) * \
        (rad[i3 - 1] - rad[i2 - 1])
    return rmask


def mask_element(el, hmax, alpha, gamma, eta):
    """ps_masking (input_pp.f90:1302-1434) and the table part of
    making_ps_with_masking (:848-1016): returns uv[k, l] at rad(k + 1),
    k = 0..nrps-1, before the norm; el.rps / el.nrps widened."""
    rps = gamma * el.rps
    i = 1
    while i <= len(el.rad) and not (el.rad[i - 1] > rps):
        i += 1
    el.nrps = i
    el.rps = float(el.rad[i - 1])
    mask = make_mask(el.rad, el.nrps, el.rps, eta)
    mr, nl, nrps = el.mr, el.mlps + 1, el.nrps
    uv = el.upp[: mr + 1, :nl] * (el.vpp[: mr + 1, :nl] - el.vpp[: mr + 1, el.lref][:, None])
    uv[:nrps] = uv[:nrps] / mask[:, None]
    nkmax = 1000
    kmax = alpha * np.pi / hmax
    radk = kmax * (np.arange(nkmax) / (nkmax - 1))
    rad = el.rad
    wk = np.zeros((nkmax, nl))
    dr = rad[1:mr] - rad[0:mr - 1]                       # j = 1..mr-1: rad(j + 1) - rad(j)
    for l in range(nl):
        kr1 = radk[:, None] * rad[None, 0:mr - 1]
        kr2 = radk[:, None] * rad[None, 1:mr]
        t = 0.5 * (xjl(kr1, l) * uv[None, 0:mr - 1, l] + xjl(kr2, l) * uv[None, 1:mr, l]) * dr[None, :]
        wk[:, l] = _seqsum(t, 1)
    out = np.zeros((mr + 1, nl))
    dk = radk[1:] - radk[:-1]
    for l in range(nl):
        kr1 = radk[:-1, None] * rad[None, 0:mr]
        kr2 = radk[1:, None] * rad[None, 0:mr]
        t = 0.5 * (xjl(kr1, l) * wk[:-1, l][:, None] + xjl(kr2, l) * wk[1:, l][:, None]) * dk[:, None]
        out[0:mr, l] = _seqsum(t, 0)
    out[mr] = 2.0 * out[mr - 1] - out[mr - 2]
    out = (2.0 / np.pi) * out
    out[:nrps] = out[:nrps] * mask[:, None]
    for l in range(nl):
        cst = np.sqrt((2.0 * l + 1.0) / (4.0 * np.pi))
        out[1:mr + 1, l] = out[1:mr + 1, l] * cst / rad[1:mr + 1] ** (l + 1)
        out[0, l] = 2.0 * out[1, l] - out[2, l]
    return out[:nrps]


class KyElement:
    """One element read and prepared as input_pp does (ps_format 'KY' by
    default; fmt 'ABINIT', 'ABINITFHI' or 'FHI' for the other one-projector
    readers)."""

    def __init__(self, path, lmax_ps, lloc, nrmax, fmt="KY", mask=None, hmax=None):
        if fmt == "KY":
            mlps, rrc = _read_ky(self, path, nrmax)
        elif fmt == "ABINIT":
            mlps, rrc = _read_abinit(self, path, nrmax)
        else:
            mlps, rrc = _read_fhi(self, path, nrmax, fmt == "ABINITFHI")
        self.nrmax = nrmax
        if lmax_ps is not None and lmax_ps >= 0:
            mlps = lmax_ps
        self.mlps = mlps
        self.lref = lloc
        for i in range(self.mr + 1, nrmax + 1):
            r = self.rad[i - 1]
            if r > 0.0:
                self.vpp[i, : mlps + 1] = -self.zps / r
            self.upp[i, : mlps + 1] = 0.0
        self.rps = float(np.max(rrc[: mlps + 1]))
        i = 1
        while i <= nrmax and not (self.rad[i - 1] > self.rps):
            i += 1
        self.nrps = i
        # KB norms (trapezoid), input_pp.f90:179-193
        self.anorm = np.zeros(mlps + 1)
        self.inorm = np.zeros(mlps + 1, dtype=int)
        for l in range(mlps + 1):
            s = 0.0
            for k in range(1, self.mr):
                r1 = self.rad[k] - self.rad[k - 1]
                s = s + (self.upp[k, l] ** 2 * (self.vpp[k, l] - self.vpp[k, lloc])
                         + self.upp[k - 1, l] ** 2 * (self.vpp[k - 1, l] - self.vpp[k - 1, lloc])) * r1
            s = 0.5 * s
            self.inorm[l] = 1
            if s < 0.0:
                s, self.inorm[l] = -s, -1
            if abs(s) < 1e-10:
                self.inorm[l] = 0
            self.anorm[l] = np.sqrt(s)
        if mask is not None:  # yn_psmask = 'y': mask = (alpha_mask, gamma_mask, eta_mask)
            uvm = mask_element(self, hmax, *mask)
        else:  # making_ps_without_masking
            for l in range(mlps + 1):
                for k in range(1, self.mr + 1):
                    self.upp[k, l] = self.upp[k, l] * np.sqrt((2 * l + 1.0) / (4 * np.pi)) / self.rad[k] ** (l + 1)
                self.upp[0, l] = self.upp[1, l]
        self.coef = []
        xn = self.rad[: self.nrps]
        for l in range(mlps + 1):
            if mask is not None:
                yn = uvm[:, l].copy()
            else:
                yn = np.array([(self.vpp[k - 1, l] - self.vpp[k - 1, lloc]) * self.upp[k - 1, l]
                               for k in range(1, self.nrps + 1)])
            if self.inorm[l] != 0:
                yn = yn / self.anorm[l]
            self.coef.append(spline(xn, yn))


def _vpsl_periodic(el, rion, kion, num, al):
    """calc_Vpsl_periodic: zVG_ion per element by the midpoint rule on the
    local channel, the structure sum with exp(-i G.R) / det A, then the inverse
    transforms along z, y, x with egz / egy / egx; the real part."""
    n0, n1, n2 = num
    detA = al[0] * al[1] * al[2]

    def fold(m, n):
        return m - n if m - (n + 1) // 2 >= 0 else m

    vt = np.zeros((n0, n1, n2), dtype=np.complex128)
    for kz in range(n2):
        for ky in range(n1):
            for kx in range(n0):
                g = np.array([fold(kx, n0) * 2 * np.pi / al[0], fold(ky, n1) * 2 * np.pi / al[1],
                              fold(kz, n2) * 2 * np.pi / al[2]])
                G2 = float(g @ g)
                gzero = kx == 0 and ky == 0 and kz == 0
                coef = 0.0 if gzero else 4 * np.pi / G2
                gs = np.sqrt(G2)
                acc = 0.0 + 0.0j
                for a in range(rion.shape[1]):
                    e = el[kion[a] - 1]
                    s = 0.0
                    for i in range(2, e.nrps + 1):
                        r1 = 0.5 * (e.rad[i - 1] + e.rad[i - 2])
                        dr = e.rad[i - 1] - e.rad[i - 2]
                        vav = 0.5 * (e.vpp[i - 1, e.lref] + e.vpp[i - 2, e.lref])
                        if gzero:
                            s = s + 4 * np.pi * (r1 * r1 * vav + r1 * e.zps) * dr
                        else:
                            s = s + 4 * np.pi * np.sin(gs * r1) / gs * (r1 * vav + e.zps) * dr
                    gd = float(g @ rion[:, a])
                    acc = acc + (s - coef * e.zps) * (np.exp(-1j * gd) / detA)
                vt[kx, ky, kz] = acc

    def eg(n):  # eg[k, i] = exp(2 pi i (i)(k) / n), 0-based
        k = np.arange(n)
        return np.exp(2j * np.pi * np.outer(k, k) / n)

    vt = np.einsum("ki,abk->abi", eg(n2), vt)   # z
    vt = np.einsum("ki,akc->aic", eg(n1), vt)   # y
    vt = np.einsum("ki,kbc->ibc", eg(n0), vt)   # x
    return np.asfortranarray(vt.real)


def init_ps_ky(files, lloc_ps, grid, rion, kion, lmax_ps=None, by_name=False, mask=None):
    """(mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu, Vpsl or None) as init_ps builds them."""
    periodic = bool(grid.periodic)
    nrmax = 3000 if periodic else 20000
    el = [KyElement(f, None if lmax_ps is None else lmax_ps[k], lloc_ps[k], nrmax,
                    _format_of(f) if by_name else "KY", mask=mask, hmax=float(np.max(grid.hgs)))
          for k, f in enumerate(files)]
    rion = np.asarray(rion, dtype=np.float64).reshape(3, -1, order="F")
    natom = rion.shape[1]
    num = [int(n) for n in grid.num]
    is_ = [int(v) for v in grid.is_]
    ie = [is_[d] + num[d] - 1 for d in range(3)]
    hgs = [float(h) for h in grid.hgs]
    al = [num[d] * hgs[d] for d in range(3)]
    rshift = [-hgs[d] if periodic else (0.0 if num[d] % 2 == 1 else -0.5 * hgs[d]) for d in range(3)]
    rps_max = max(e.rps for e in el) + 1.5 * max(hgs) + 1e-2
    nc = [0, 0, 0]
    if periodic:
        for d in range(3):
            mn, mx = rion[d].min(), rion[d].max()
            nc[d] = 1 if (mn + 2 * al[d] > al[d] + rps_max and mx - 2 * al[d] < -rps_max) else 2
    pts = []
    for a in range(natom):
        e = el[kion[a] - 1]
        jl, rl = [], []
        for j1 in range(-nc[0], nc[0] + 1):
            t1 = rion[0, a] + j1 * al[0]
            if t1 <= is_[0] * hgs[0] - rps_max or t1 >= ie[0] * hgs[0] + rps_max:
                continue
            for j2 in range(-nc[1], nc[1] + 1):
                t2 = rion[1, a] + j2 * al[1]
                if t2 <= is_[1] * hgs[1] - rps_max or t2 >= ie[1] * hgs[1] + rps_max:
                    continue
                for j3 in range(-nc[2], nc[2] + 1):
                    t3 = rion[2, a] + j3 * al[2]
                    if t3 <= is_[2] * hgs[2] - rps_max or t3 >= ie[2] * hgs[2] + rps_max:
                        continue
                    for i3 in range(is_[2], ie[2] + 1):
                        z = i3 * hgs[2] + rshift[2] - t3
                        for i2 in range(is_[1], ie[1] + 1):
                            y = i2 * hgs[1] + rshift[1] - t2
                            i1 = np.arange(is_[0], ie[0] + 1)
                            x = i1 * hgs[0] + rshift[0] - t1
                            r = np.sqrt(x * x + y * y + z * z)
                            for k in np.nonzero(r < e.rps + 1e-12)[0]:
                                jl.append((int(i1[k]), i2, i3))
                                rl.append((float(x[k]), y, z))
        pts.append((jl, rl))
    nps = max(len(p[0]) for p in pts)
    lm = [[(l, m) for l in range(el[kion[a] - 1].mlps + 1) if el[kion[a] - 1].inorm[l] != 0
           for m in range(-l, l + 1)] for a in range(natom)]
    nlma = sum(len(x) for x in lm)
    mps = np.array([len(p[0]) for p in pts], dtype=np.int32)
    jxyz = np.zeros((3, nps, natom), dtype=np.int32, order="F")
    rxyz = np.zeros((3, nps, natom), order="F")
    uv = np.zeros((nps, nlma), order="F")
    ia = np.zeros(nlma, dtype=np.int32)
    rinv = np.zeros(nlma)
    lma = 0
    for a in range(natom):
        e = el[kion[a] - 1]
        jl, rl = pts[a]
        for j, (q, r) in enumerate(zip(jl, rl)):
            jxyz[:, j, a] = q
            rxyz[:, j, a] = r
        for (l, m) in lm[a]:
            ia[lma] = a + 1
            rinv[lma] = float(e.inorm[l]) * grid.hvol
            for j, (x, y, z) in enumerate(rl):
                rr = np.sqrt(x * x + y * y + z * z) + 1e-50
                ir = 1
                while ir <= e.nrps and not (e.rad[ir - 1] > rr):
                    ir += 1
                intr = ir - 1
                xx = rr - e.rad[intr - 1]
                an, bn, cn, dn = e.coef[l]
                s = intr - 1
                uvr = an[s] * xx ** 3 + bn[s] * xx ** 2 + cn[s] * xx + dn[s]
                uv[j, lma] = uvr * ylm(x, y, z, l, m)
            lma += 1
    vpsl = None
    if periodic:
        vpsl = _vpsl_periodic(el, rion, kion, num, al)
    else:
        vpsl = np.zeros(num, order="F")
        coord = [(np.arange(is_[d], ie[d] + 1) - (0.0 if num[d] % 2 == 1 else 0.5)) * hgs[d] for d in range(3)]
        X, Y, Z = np.meshgrid(*coord, indexing="ij")
        for a in range(natom):
            e = el[kion[a] - 1]
            r = np.sqrt((X - rion[0, a]) ** 2 + (Y - rion[1, a]) ** 2 + (Z - rion[2, a]) ** 2) + 1e-50
            # bisection over rad(1..nrmax): rad(intr) < r <= rad(intr + 1)
            intr = np.searchsorted(e.rad, r, side="left")   # count of rad < r (1-based intr)
            intr = np.clip(intr, 1, e.nrmax - 1)
            r0, r1 = e.rad[intr - 1], e.rad[intr]
            ratio1 = (r - r0) / (r1 - r0)
            ratio2 = 1.0 - ratio1
            vpsl = vpsl + ratio1 * e.vpp[intr, e.lref] + ratio2 * e.vpp[intr - 1, e.lref]
    return mps, jxyz, rxyz, uv, ia, rinv, vpsl
