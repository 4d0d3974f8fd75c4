"""Seeded synthetic systems with the shapes of the RT-TDDFT hot-path workloads.

Everything here builds host-side inputs in the reference's own data layout
(Fortran column-major, x fastest, the reference's array bounds), exactly as
SALMON's set-up code would hand them to ``hpsi``/``taylor``:

* grid bounds, neighbour maps and stencil coefficients follow
  ``src/common/initialization.f90:241-256,398-418,508-611,1125-1190,1324-1450``;
* projector tables follow ``src/atom/pp/prep_pp.f90:280-525`` (sphere points by
  image then z, y, x; ``lma`` ordering atom-major, ``l`` then ``m``; ``uV`` =
  radial x ``Ylm`` monomial; ``rinv_uvu = inorm*hvol``), with the spline of a
  pseudopotential file replaced by a Gaussian radial function;
* the impulse kick follows ``src/rt/initialization_rt.f90:382-423``, the
  Taylor coefficients ``:492-507`` and the laser shapes
  ``src/rt/em_field.f90:86-306``.

No real pseudopotential or ground state is involved: orbitals are seeded random
fields times a smooth envelope (or, for periodic grids on request, band-limited
plane-wave sums), orthonormalised with the ``hvol`` metric.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

AU_LENGTH_AA = 0.52917721067  # src/io/inputoutput.f90:27
AU_ENERGY_EV = 27.21138505    # src/io/inputoutput.f90:26
ND = 4

# bNmat(:,4), cNmat(:,4): initialization.f90:1324-1371 (8th-order central FD)
BN4 = np.array([4.0 / 5.0, -1.0 / 5.0, 4.0 / 105.0, -1.0 / 280.0])
CN4 = np.array([-205.0 / 72.0, 8.0 / 5.0, -1.0 / 5.0, 8.0 / 315.0, -1.0 / 560.0])


@dataclasses.dataclass
class Grid:
    """``s_rgrid`` + ``s_stencil`` of one r-space domain holding the whole grid."""

    periodic: bool
    num: np.ndarray          # lg%num
    is_: np.ndarray          # mg%is
    ie: np.ndarray           # mg%ie
    is_array: np.ndarray     # mg%is_array
    ie_array: np.ndarray     # mg%ie_array
    idx: np.ndarray          # mg%idx(is-4:ie+4)
    idy: np.ndarray
    idz: np.ndarray
    hgs: np.ndarray
    hvol: float
    coef_lap0: float
    coef_lap: np.ndarray     # (4,3) Fortran order
    coef_nab: np.ndarray     # (4,3) Fortran order

    @property
    def shape_array(self):
        return tuple(int(v) for v in (self.ie_array - self.is_array + 1))

    @property
    def shape(self):
        return tuple(int(v) for v in (self.ie - self.is_ + 1))

    def coordinate(self, axis: int) -> np.ndarray:
        """lg%coordinate(is:ie, axis), initialization.f90:1125-1190."""
        i = np.arange(self.is_[axis], self.ie[axis] + 1, dtype=np.float64)
        h = self.hgs[axis]
        if self.periodic:
            return (i - 1.0) * h
        if self.num[axis] % 2 == 1:
            return i * h
        return (i - 0.5) * h

    def interior_slices(self):
        return tuple(slice(int(self.is_[d] - self.is_array[d]),
                           int(self.ie[d] - self.is_array[d] + 1)) for d in range(3))


def make_grid(num, h, periodic: bool, pad_y: bool = True) -> Grid:
    num = np.asarray(num, dtype=np.int32).reshape(3)
    hgs = np.broadcast_to(np.asarray(h, dtype=np.float64), (3,)).copy()
    if periodic:
        is_ = np.ones(3, np.int32)
        ie = num.copy()
    else:
        ie = (num // 2).astype(np.int32)
        is_ = np.where(num % 2 == 1, -(num // 2), -(num // 2) + 1).astype(np.int32)
    if periodic:
        is_array, ie_array = is_.copy(), ie.copy()
    else:
        is_array, ie_array = is_ - ND, ie + ND
    if pad_y:  # USE_OPT_ARRAY_PADDING, initialization.f90:606-609
        ie_array = ie_array.copy()
        ie_array[1] += 1
    maps = []
    for d in range(3):
        j = np.arange(is_[d] - ND, ie[d] + ND + 1, dtype=np.int64)
        if periodic:
            maps.append(((j + num[d] - 1) % num[d] + 1).astype(np.int32))
        else:
            maps.append(j.astype(np.int32))
    coef_lap0 = -0.5 * CN4[0] * float(np.sum(1.0 / hgs ** 2))
    coef_lap = np.zeros((4, 3), order="F")
    coef_nab = np.zeros((4, 3), order="F")
    for d in range(3):
        coef_lap[:, d] = CN4[1:] / hgs[d] ** 2
        coef_nab[:, d] = BN4 / hgs[d]
    return Grid(periodic, num, is_, ie, is_array, ie_array, maps[0], maps[1], maps[2],
                hgs, float(np.prod(hgs)), coef_lap0, coef_lap, coef_nab)


def ylm(x, y, z, l, m):
    """Ylm monomials for l <= 1 (src/math/salmon_math.f90:386-424)."""
    if l == 0:
        return np.ones_like(x)
    if l == 1:
        return {-1: -y, 0: z, 1: -x}[m]
    raise ValueError("only l <= 1 projectors are generated")


@dataclasses.dataclass
class PPGrid:
    """``s_pp_grid`` subset read by zpseudo / calc_current_nonlocal."""

    natom: int
    nps: int
    nlma: int
    mps: np.ndarray       # (natom,) int32
    jxyz: np.ndarray      # (3,nps,natom) int32, Fortran order
    rxyz: np.ndarray      # (3,nps,natom) float64, Fortran order
    uv: np.ndarray        # (nps,nlma) float64, Fortran order
    ia_tbl: np.ndarray    # (nlma,) int32, 1-based
    rinv_uvu: np.ndarray  # (nlma,)


def make_pp(grid: Grid, rion: np.ndarray, rc: float, sigma, amp, inorm, lmax: int = 1,
            cell=None) -> PPGrid:
    """Gaussian KB projectors on the grid (prep_pp.f90 calc_jxyz/set_lma/calc_uv).

    ``sigma``/``amp`` are per-atom arrays; ``inorm`` is (natom, lmax+1) of +-1.
    """
    natom = rion.shape[1]
    nc = 1 if grid.periodic else 0
    cell = np.zeros(3) if cell is None else np.asarray(cell, dtype=np.float64)
    coords = [grid.coordinate(d) for d in range(3)]
    idx = [np.arange(grid.is_[d], grid.ie[d] + 1) for d in range(3)]
    # grid point coordinates in (z, y, x) loop order (x fastest)
    Z, Y, X = np.meshgrid(coords[2], coords[1], coords[0], indexing="ij")
    IZ, IY, IX = np.meshgrid(idx[2], idx[1], idx[0], indexing="ij")
    X, Y, Z = X.ravel(), Y.ravel(), Z.ravel()
    IX, IY, IZ = IX.ravel(), IY.ravel(), IZ.ravel()
    pts = []
    for ia in range(natom):
        jl, rl = [], []
        for j1 in range(-nc, nc + 1):
            for j2 in range(-nc, nc + 1):
                for j3 in range(-nc, nc + 1):
                    t = rion[:, ia] + np.array([j1, j2, j3]) * cell
                    x, y, z = X - t[0], Y - t[1], Z - t[2]
                    r = np.sqrt(x * x + y * y + z * z)
                    sel = r < rc + 1e-12
                    jl.append(np.stack([IX[sel], IY[sel], IZ[sel]]))
                    rl.append(np.stack([x[sel], y[sel], z[sel]]))
        pts.append((np.concatenate(jl, axis=1), np.concatenate(rl, axis=1)))
    mps = np.array([p[0].shape[1] for p in pts], dtype=np.int32)
    nps = int(mps.max()) if natom else 0
    jxyz = np.zeros((3, nps, natom), dtype=np.int32, order="F")
    rxyz = np.zeros((3, nps, natom), dtype=np.float64, order="F")
    for ia, (j, r) in enumerate(pts):
        jxyz[:, : j.shape[1], ia] = j
        rxyz[:, : r.shape[1], ia] = r
    lm_list = [(l, m) for l in range(lmax + 1) for m in range(-l, l + 1)]
    nlma = natom * len(lm_list)
    uv = np.zeros((nps, nlma), dtype=np.float64, order="F")
    ia_tbl = np.zeros(nlma, dtype=np.int32)
    rinv = np.zeros(nlma, dtype=np.float64)
    lma = 0
    sigma = np.broadcast_to(np.asarray(sigma, dtype=np.float64), (natom,))
    amp = np.broadcast_to(np.asarray(amp, dtype=np.float64), (natom,))
    inorm = np.asarray(inorm).reshape(natom, lmax + 1)
    for ia in range(natom):
        m_ = mps[ia]
        x, y, z = rxyz[0, :m_, ia], rxyz[1, :m_, ia], rxyz[2, :m_, ia]
        r2 = x * x + y * y + z * z
        g = amp[ia] * np.exp(-r2 / (2.0 * sigma[ia] ** 2))
        for (l, m) in lm_list:
            uv[:m_, lma] = g * ylm(x, y, z, l, m)
            ia_tbl[lma] = ia + 1
            rinv[lma] = float(inorm[ia, l]) * grid.hvol
            lma += 1
    return PPGrid(natom, nps, nlma, mps, jxyz, rxyz, uv, ia_tbl, rinv)


@dataclasses.dataclass
class System:
    grid: Grid
    pp: PPGrid
    nspin: int
    no: int
    nk: int
    vec_k: np.ndarray      # (3,nk) Fortran order
    rocc: np.ndarray       # (no,nk,nspin) Fortran order
    wtk: np.ndarray        # (nk,)
    V_local: np.ndarray    # (nx,ny,nz,nspin) Fortran order, interior
    rion: np.ndarray       # (3,natom)
    psi: np.ndarray        # (nxa,nya,nza,nspin,no,nk) complex128 Fortran order
    ngrid: int
    seed: int
    name: str = ""
    lattice: "Lattice | None" = None   # non-orthogonal cell (None: orthogonal)

    @property
    def norb(self):
        return self.nspin * self.no * self.nk


@dataclasses.dataclass
class Lattice:
    """system%primitive_a / rmatrix_A / rmatrix_B and stencil%coef_F of a
    non-orthogonal cell (init_lattice, src/common/lattice.f90:23-75)."""

    primitive_a: np.ndarray  # (3,3), column d = a_d
    rmatrix_A: np.ndarray    # (3,3), columns the unit vectors u, v, w
    rmatrix_B: np.ndarray    # inverse of rmatrix_A
    coef_F: np.ndarray       # (6,) f_uu, f_vv, f_ww, f_vw, f_uw, f_uv
    det_a: float


def init_lattice(primitive_a) -> Lattice:
    """init_lattice (lattice.f90:23-75): A = [u v w] the unit lattice vectors,
    B = A^-1, F = B B^T; coef_F = (F11, F22, F33, F23 + F32, F13 + F31, F12 + F21)."""
    a = np.asarray(primitive_a, dtype=np.float64)
    det = float(np.linalg.det(a))
    A = a / np.linalg.norm(a, axis=0)[None, :]
    B = np.linalg.inv(A)
    F = B @ B.T
    coef_F = np.array([F[0, 0], F[1, 1], F[2, 2], F[1, 2] + F[2, 1], F[0, 2] + F[2, 0], F[0, 1] + F[1, 0]])
    return Lattice(a, A, B, coef_F, det)


def nonorthogonal_system(primitive_a, num, nkgrid=1, no=3, seed=50, natom=2, rc_aa=1.0, nspin=1,
                         name="nonorth", with_pp=True) -> System:
    """Periodic system on a non-orthogonal cell (columns of primitive_a the
    lattice vectors, bohr): grid spacing |a_d| / num_d along each lattice
    vector, coef_lap0 = -cN0 / 2 sum_d F_d / h_d^2 and hvol = det(A) / N
    (initialization.f90:242-249, lattice.f90:38-39); Monkhorst-Pack k-points
    on the reciprocal vectors; Gaussian V_local and Gaussian KB projectors
    (l <= 1) at seeded atoms, evaluated at the Cartesian grid points
    r = sum_d i_d h_d u_d with their periodic images."""
    rng = np.random.default_rng(seed)
    lat = init_lattice(primitive_a)
    a = lat.primitive_a
    nums = [int(num)] * 3 if np.isscalar(num) else [int(v) for v in num]
    h = np.linalg.norm(a, axis=0) / np.array(nums, dtype=np.float64)
    grid = make_grid(nums, h, periodic=True)
    coef_lap0 = -0.5 * CN4[0] * float(np.sum(lat.coef_F[:3] / h ** 2))
    grid = dataclasses.replace(grid, coef_lap0=coef_lap0, hvol=lat.det_a / float(np.prod(nums)))
    # Cartesian grid points, x fastest
    fr = np.meshgrid(*[np.arange(n) / float(n) for n in nums], indexing="ij")
    R = np.einsum("dk,kxyz->dxyz", a, np.stack(fr))
    frac_ion = rng.uniform(0.0, 1.0, size=(3, natom))
    rion = np.asfortranarray(a @ frac_ion)
    images = [a @ np.array([i, j, k], dtype=np.float64) for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)]
    amps, widths = rng.uniform(-2.0, -0.5, natom), rng.uniform(0.8, 1.6, natom)
    V = np.zeros(nums)
    for ia in range(natom):
        for t in images:
            d = R - (rion[:, ia] + t)[:, None, None, None]
            V += amps[ia] * np.exp(-np.sum(d * d, axis=0) / (2.0 * widths[ia] ** 2))
    V_local = np.asfortranarray(np.repeat(V[..., None], nspin, axis=3))
    if with_pp:
        rc = rc_aa / AU_LENGTH_AA
        sigma, amp = rng.uniform(0.5, 0.8, natom), rng.uniform(0.3, 0.6, natom)
        inorm = rng.choice([-1, 1], size=(natom, 2))
        idx = np.stack(np.meshgrid(*[np.arange(1, n + 1) for n in nums], indexing="ij"))
        Rf = R.reshape(3, -1, order="F")
        If = idx.reshape(3, -1, order="F")
        pts = []
        for ia in range(natom):
            jl, rl = [], []
            for t in images:
                d = Rf - (rion[:, ia] + t)[:, None]
                sel = np.sqrt(np.sum(d * d, axis=0)) < rc + 1e-12
                jl.append(If[:, sel])
                rl.append(d[:, sel])
            pts.append((np.concatenate(jl, axis=1), np.concatenate(rl, axis=1)))
        mps = np.array([p[0].shape[1] for p in pts], dtype=np.int32)
        nps = int(mps.max())
        jxyz = np.zeros((3, nps, natom), dtype=np.int32, order="F")
        rxyz = np.zeros((3, nps, natom), dtype=np.float64, order="F")
        for ia, (j, r) in enumerate(pts):
            jxyz[:, : j.shape[1], ia] = j
            rxyz[:, : r.shape[1], ia] = r
        nlma = 4 * natom
        uv = np.zeros((nps, nlma), order="F")
        ia_tbl = np.zeros(nlma, dtype=np.int32)
        rinv = np.zeros(nlma)
        lma = 0
        for ia in range(natom):
            m_ = mps[ia]
            x, y, z = rxyz[0, :m_, ia], rxyz[1, :m_, ia], rxyz[2, :m_, ia]
            g = amp[ia] * np.exp(-(x * x + y * y + z * z) / (2.0 * sigma[ia] ** 2))
            for (l, m) in [(0, 0), (1, -1), (1, 0), (1, 1)]:
                uv[:m_, lma] = g * ylm(x, y, z, l, m)
                ia_tbl[lma] = ia + 1
                rinv[lma] = float(inorm[ia, l]) * grid.hvol
                lma += 1
        pp = PPGrid(natom, nps, nlma, mps, jxyz, rxyz, uv, ia_tbl, rinv)
    else:
        pp = PPGrid(0, 0, 0, np.zeros(0, np.int32), np.zeros((3, 0, 0), np.int32, order="F"),
                    np.zeros((3, 0, 0), order="F"), np.zeros((0, 0), order="F"), np.zeros(0, np.int32), np.zeros(0))
    n = int(nkgrid)
    f = (2.0 * np.arange(1, n + 1) - n - 1) / (2.0 * n)
    brec = 2.0 * np.pi * np.linalg.inv(a).T  # columns b_d
    ks = [brec @ np.array([f[i], f[j], f[k]]) for k in range(n) for j in range(n) for i in range(n)]
    vec_k = np.asfortranarray(np.array(ks).T)
    nk = vec_k.shape[1]
    psi = random_orbitals(grid, rng, nspin, no, nk)
    psi *= math.sqrt(float(np.prod(h)) / grid.hvol)  # orthonormal in the det(A) / N metric
    return System(grid, pp, nspin, no, nk, vec_k, np.asfortranarray(np.full((no, nk, nspin), 2.0)),
                  np.full(nk, 1.0 / nk), V_local, rion, psi, int(np.prod(nums)), seed, name, lat)


def gaussian_potential(grid: Grid, centers: np.ndarray, amps, widths, cell=None) -> np.ndarray:
    nx, ny, nz = grid.shape
    X, Y, Z = np.meshgrid(grid.coordinate(0), grid.coordinate(1), grid.coordinate(2), indexing="ij")
    V = np.zeros((nx, ny, nz))
    shifts = [np.zeros(3)]
    if grid.periodic and cell is not None:
        shifts = [np.array([a, b, c]) * cell for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)]
    for a in range(centers.shape[1]):
        for s in shifts:
            c = centers[:, a] + s
            r2 = (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2
            V += amps[a] * np.exp(-r2 / (2.0 * widths[a] ** 2))
    return V


def _cholesky_qr2(a):
    """Orthonormal columns spanning a (tall, well conditioned): two passes of
    Cholesky QR (Gram matrix, Cholesky factor, triangular inverse)."""
    for _ in range(2):
        g = a.conj().T @ a
        L = np.linalg.cholesky(g)
        a = a @ np.linalg.inv(L).conj().T
    return a


def random_orbitals(grid: Grid, rng, nspin, no, nk, envelope_width=None, real=False,
                    fast=False, ecut=None) -> np.ndarray:
    """Seeded orbitals, orthonormal per (k, spin) in the hvol metric, in the
    reference array layout with a zero halo (structures.f90:646-669).
    fast=True orthonormalises by Cholesky QR instead of Householder QR.
    ecut (Hartree): the random field keeps only the Fourier components of the
    box with |G|^2/2 <= ecut before the envelope is applied (smooth orbitals
    whose spectral weight lies at low energy, like occupied states)."""
    nx, ny, nz = grid.shape
    X, Y, Z = np.meshgrid(grid.coordinate(0), grid.coordinate(1), grid.coordinate(2), indexing="ij")
    if envelope_width is None:
        env = np.ones((nx, ny, nz))
    else:
        if grid.periodic:
            env = np.ones((nx, ny, nz))
        else:
            env = np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / (2.0 * envelope_width ** 2))
    npt = nx * ny * nz
    dt = np.float64 if real else np.complex128
    out = np.zeros(grid.shape_array + (nspin, no, nk), dtype=dt, order="F")
    sl = grid.interior_slices()
    for ik in range(nk):
        for isp in range(nspin):
            a = rng.standard_normal((npt, no))
            if not real:
                a = a + 1j * rng.standard_normal((npt, no))
            if ecut is not None:
                L = grid.hgs * np.array([nx, ny, nz], dtype=np.float64)
                g = [2.0 * math.pi * np.fft.fftfreq(n, 1.0 / n) / L[d] for d, n in enumerate((nx, ny, nz))]
                kin = 0.5 * (g[0][:, None, None] ** 2 + g[1][None, :, None] ** 2 + g[2][None, None, :] ** 2)
                f = np.fft.fftn(a.reshape((nx, ny, nz, no), order="F"), axes=(0, 1, 2))
                f[kin > ecut] = 0.0
                a = np.fft.ifftn(f, axes=(0, 1, 2)).reshape((npt, no), order="F")
                if real:
                    a = a.real
            a *= env.reshape(-1, order="F")[:, None]
            q = _cholesky_qr2(a) if fast else np.linalg.qr(a)[0]
            q = q / math.sqrt(grid.hvol)
            for io in range(no):
                out[sl + (isp, io, ik)] = q[:, io].reshape((nx, ny, nz), order="F")
    return out


def band_limited_orbitals(grid: Grid, rng, nspin, no, vec_k, ecut) -> np.ndarray:
    """Seeded Bloch orbitals (periodic part u_k on the grid) built only from
    plane waves with kinetic energy |k+G|^2/2 <= ecut (Hartree), orthonormal
    per (k, spin) in the hvol metric.  A stand-in for occupied states, whose
    spectral weight lies at low energy, unlike white-noise fields."""
    if not grid.periodic:
        raise ValueError("band-limited orbitals are defined for periodic grids")
    nx, ny, nz = grid.shape
    npt = nx * ny * nz
    L = grid.hgs * np.array([nx, ny, nz], dtype=np.float64)
    g = [2.0 * math.pi * np.fft.fftfreq(n, 1.0 / n) / L[d] for d, n in enumerate((nx, ny, nz))]
    out = np.zeros(grid.shape_array + (nspin, no, vec_k.shape[1]), dtype=np.complex128, order="F")
    sl = grid.interior_slices()
    for ik in range(vec_k.shape[1]):
        k = vec_k[:, ik]
        kin = 0.5 * ((g[0][:, None, None] + k[0]) ** 2 + (g[1][None, :, None] + k[1]) ** 2
                     + (g[2][None, None, :] + k[2]) ** 2)
        mask = kin <= ecut
        ng = int(mask.sum())
        if ng < no:
            raise ValueError(f"ecut={ecut} admits {ng} plane waves at k-point {ik}, fewer than {no} orbitals")
        for isp in range(nspin):
            c = np.zeros((nx, ny, nz, no), dtype=np.complex128)
            c[mask] = rng.standard_normal((ng, no)) + 1j * rng.standard_normal((ng, no))
            a = np.fft.ifftn(c, axes=(0, 1, 2)).reshape((npt, no), order="F")
            q = _cholesky_qr2(a) / math.sqrt(grid.hvol)
            for io in range(no):
                out[sl + (isp, io, ik)] = q[:, io].reshape((nx, ny, nz), order="F")
    return out


def mp_kpoints(nkgrid, cell):
    """Monkhorst-Pack k-points, cubic cell, Cartesian, weights 1/nk."""
    n = int(nkgrid)
    f = (2.0 * np.arange(1, n + 1) - n - 1) / (2.0 * n)
    b = 2.0 * np.pi / np.asarray(cell, dtype=np.float64)
    ks = [(f[i] * b[0], f[j] * b[1], f[k] * b[2]) for k in range(n) for j in range(n) for i in range(n)]
    vec_k = np.asfortranarray(np.array(ks).T)
    return vec_k, np.full(vec_k.shape[1], 1.0 / vec_k.shape[1])


def taylor_zc(dt: float, n_hamil: int = 4, aetrs: bool = False) -> np.ndarray:
    """rt%zc, initialization_rt.f90:492-507."""
    zc = np.zeros(n_hamil, dtype=np.complex128)
    step = (-1j * dt / 2.0) if aetrs else (-1j * dt)
    for n in range(1, n_hamil + 1):
        v = step ** n
        for m in range(1, n + 1):
            v = v / m
        zc[n - 1] = v
    return zc


def impulse_kick(grid: Grid, psi: np.ndarray, e_impulse: float, epdir=(0.0, 0.0, 1.0)) -> np.ndarray:
    """psi <- exp(i e_impulse epdir.r) psi on interior points (initialization_rt.f90:382-423)."""
    X, Y, Z = np.meshgrid(grid.coordinate(0), grid.coordinate(1), grid.coordinate(2), indexing="ij")
    R1 = epdir[0] * X + epdir[1] * Y + epdir[2] * Z
    ph = np.exp(1j * e_impulse * R1)
    sl = grid.interior_slices()
    out = psi.copy(order="F")
    out[sl] = ph[(...,) + (None,) * (psi.ndim - 3)] * psi[sl]
    return out


def asin2cos(nt: int, dt: float, omega: float, f0: float, tw: float, epdir=(0.0, 0.0, 1.0),
             phi_cep: float = 0.0) -> np.ndarray:
    """Ac_ext(3, 0:nt+1) for ae_shape1='Asin2cos' (em_field.f90:177-186)."""
    Ac = np.zeros((3, nt + 2), order="F")
    ep = np.asarray(epdir, dtype=np.float64)
    for i in range(nt + 2):
        t = i * dt
        if t < tw:
            Ac[:, i] = -ep * f0 / omega * math.sin(math.pi * t / tw) ** 2 * math.cos(omega * t + phi_cep * 2.0 * math.pi)
    return Ac


# --------------------------------------------------------------------------
# workload builders
# --------------------------------------------------------------------------

def isolated_system(num=64, h_aa=0.25, no=5, natom=4, seed=1, rc_aa=1.2, nspin=1,
                    real=False, name="isolated", fast=False, ecut=None) -> System:
    """Isolated molecule: Dirichlet box, seeded atoms in the central 60 %.
    ecut: band-limit the orbitals (random_orbitals)."""
    rng = np.random.default_rng(seed)
    h = h_aa / AU_LENGTH_AA
    nums = [int(num)] * 3 if np.isscalar(num) else [int(v) for v in num]
    grid = make_grid(nums, h, periodic=False)
    L = min(nums) * h
    rion = np.asfortranarray(rng.uniform(-0.3 * L, 0.3 * L, size=(3, natom)))
    rc = rc_aa / AU_LENGTH_AA
    pp = make_pp(grid, rion, rc, sigma=rng.uniform(0.5, 0.8, natom), amp=rng.uniform(0.3, 0.6, natom),
                 inorm=rng.choice([-1, 1], size=(natom, 2)))
    V = gaussian_potential(grid, rion, rng.uniform(-2.0, -0.5, natom), rng.uniform(0.8, 1.6, natom))
    V_local = np.asfortranarray(np.repeat(V[..., None], nspin, axis=3))
    psi = random_orbitals(grid, rng, nspin, no, 1, envelope_width=0.2 * L, real=real, fast=fast, ecut=ecut)
    return System(grid, pp, nspin, no, 1, np.zeros((3, 1), order="F"),
                  np.asfortranarray(np.full((no, 1, nspin), 2.0)), np.ones(1), V_local, rion, psi,
                  int(np.prod(grid.num)), seed, name)


def kpoint_shard(system: System, rank: int, world: int, a_cell: float, nkgrid: int) -> System:
    """Weak-scaling shard of a periodic system for rank `rank` of `world`: the
    k-mesh shifted by rank/world of one mesh spacing along every axis (so the
    shards together sample a `world`-times denser mesh) and the k-weights
    divided by `world`; orbitals, grid and potential are shared.  The current
    of the whole job is the sum of the shards' currents (calc_current sums
    occupation x k-weight terms, density_matrix.f90:240-463)."""
    import dataclasses
    if world <= 1:
        return system
    shift = (2.0 * np.pi / a_cell) * (rank / world) / nkgrid
    return dataclasses.replace(system, vec_k=np.asfortranarray(system.vec_k + shift),
                               wtk=np.asarray(system.wtk) / world)


def uneven_batch(nsys=16, seed=4):
    """Independent isolated systems of uneven size from one seed: cubic grids
    n^3 with n in {32, 40, ..., 96}, 4..64 orbitals, 2..16 atoms (h = 0.25 A,
    Gaussian KB projectors, seeded Gaussian V_local), as in the batch workload
    of the propagation benchmark."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nsys):
        n = int(rng.choice(np.arange(32, 97, 8)))
        no = int(rng.integers(4, 65))
        natom = int(rng.integers(2, 17))
        out.append(isolated_system(num=n, no=no, natom=natom, seed=int(rng.integers(1 << 30)),
                                   name=f"batch{i}_{n}^3_{no}orb_{natom}at", fast=True))
    return out


DIAMOND = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5],
                    [0.25, 0.25, 0.25], [0.75, 0.75, 0.25], [0.75, 0.25, 0.75], [0.25, 0.75, 0.75]])


def periodic_system(a=10.26, num=16, nkgrid=4, no=32, supercell=1, seed=2, rc_aa=1.2,
                    nspin=1, name="periodic", ecut=None) -> System:
    """Periodic bulk (diamond positions), Monkhorst-Pack k-points.  Orbitals are
    white-noise fields, or with ``ecut`` (Hartree) band-limited to plane waves
    of kinetic energy <= ecut."""
    rng = np.random.default_rng(seed)
    cell = np.full(3, a * supercell)
    grid = make_grid([num * supercell] * 3, cell[0] / (num * supercell), periodic=True)
    frac = np.concatenate([(DIAMOND + np.array([i, j, k])) / supercell
                           for k in range(supercell) for j in range(supercell) for i in range(supercell)])
    rion = np.asfortranarray((frac * cell[0]).T)
    natom = rion.shape[1]
    rc = rc_aa / AU_LENGTH_AA
    pp = make_pp(grid, rion, rc, sigma=rng.uniform(0.5, 0.8, natom), amp=rng.uniform(0.3, 0.6, natom),
                 inorm=rng.choice([-1, 1], size=(natom, 2)), cell=cell)
    V = gaussian_potential(grid, rion, rng.uniform(-2.0, -0.5, natom), rng.uniform(0.8, 1.6, natom), cell=cell)
    V_local = np.asfortranarray(np.repeat(V[..., None], nspin, axis=3))
    vec_k, wtk = mp_kpoints(nkgrid, cell)
    nk = vec_k.shape[1]
    if ecut is None:
        psi = random_orbitals(grid, rng, nspin, no, nk)
    else:
        psi = band_limited_orbitals(grid, rng, nspin, no, vec_k, ecut)
    return System(grid, pp, nspin, no, nk, vec_k, np.asfortranarray(np.full((no, nk, nspin), 2.0)), wtk,
                  V_local, rion, psi, int(np.prod(grid.num)), seed, name)
