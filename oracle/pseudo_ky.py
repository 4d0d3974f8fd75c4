"""CPU oracle (TEST INFRASTRUCTURE ONLY) for the set-up of the Kleinman-Bylander
tables from Yabana-Bertsch pseudopotential files (`_rps.dat`, ps_format 'KY'):
a numpy restatement of read_ps_KY (src/atom/pp/input_pp.f90:288-341), the
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


class KyElement:
    """One element read and prepared as input_pp does for ps_format 'KY'."""

    def __init__(self, path, lmax_ps, lloc, nrmax):
        with open(path) as f:
            tok = f.read().split()
        it = iter(tok)
        self.mr = int(next(it))
        step = float(next(it))
        mlps = int(next(it))
        self.zps = float(int(float(next(it)) + 1e-10))
        next(it)                                       # irPC
        rrc = np.array([float(next(it)) for _ in range(mlps + 1)])
        nr = max(nrmax, self.mr)
        self.vpp = np.zeros((nr + 1, mlps + 1))        # vpp(0:nr, 0:mlps)
        self.upp = np.zeros((nr + 1, mlps + 1))
        for i in range(self.mr + 1):
            next(it), next(it)                         # r, rhopp
            for l in range(mlps + 1):
                self.vpp[i, l] = float(next(it))
        for i in range(self.mr + 1):
            next(it)
            for l in range(mlps + 1):
                self.upp[i, l] = float(next(it))
        step = step / AU_LENGTH_AA
        rrc = rrc / AU_LENGTH_AA
        self.vpp[: self.mr + 1] /= AU_ENERGY_EV
        self.upp[: self.mr + 1] *= np.sqrt(AU_LENGTH_AA)
        self.nrmax = nrmax
        self.rad = np.array([(i - 1) * step for i in range(1, nrmax + 1)])   # rad(i) at [i - 1]
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
        # making_ps_without_masking
        for l in range(mlps + 1):
            for k in range(1, self.mr + 1):
                self.upp[k, l] = self.upp[k, l] * np.sqrt((2 * l + 1.0) / (4 * np.pi)) / self.rad[k] ** (l + 1)
            self.upp[0, l] = self.upp[1, l]
        self.coef = []
        xn = self.rad[: self.nrps]
        for l in range(mlps + 1):
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


def init_ps_ky(files, lloc_ps, grid, rion, kion, lmax_ps=None):
    """(mps, jxyz, rxyz, uv, ia_tbl, rinv_uvu, Vpsl or None) as init_ps builds them."""
    periodic = bool(grid.periodic)
    nrmax = 3000 if periodic else 20000
    el = [KyElement(f, None if lmax_ps is None else lmax_ps[k], lloc_ps[k], nrmax) for k, f in enumerate(files)]
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
