"""ctypes binding of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as the checker or the timed CPU baseline.
The product library never calls it.  See ``salmon_oracle.h`` for what each
function restates and for the parity status of the oracle.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsalmon_oracle.so")
_SOURCES = ("salmon_oracle.cpp", "salmon_oracle_gs.cpp", "salmon_oracle_scf.cpp", "salmon_oracle.h")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class SboSystem(C.Structure):
    _fields_ = [
        ("is_", C.c_int * 3), ("ie", C.c_int * 3), ("is_array", C.c_int * 3), ("ie_array", C.c_int * 3),
        ("idx", _ip), ("idy", _ip), ("idz", _ip),
        ("lg_num", C.c_int * 3),
        ("coef_lap0", C.c_double), ("coef_lap", C.c_double * 12), ("coef_nab", C.c_double * 12),
        ("periodic", C.c_int), ("nspin", C.c_int), ("no", C.c_int), ("nk", C.c_int),
        ("hgs", C.c_double * 3), ("hvol", C.c_double), ("ngrid", C.c_int),
        ("vec_k", _dp), ("vec_Ac", C.c_double * 3), ("rocc", _dp), ("wtk", _dp),
        ("BT", C.c_double * 9), ("V_local", _dp),
        ("natom", C.c_int), ("nps", C.c_int), ("nlma", C.c_int),
        ("mps", _ip), ("jxyz", _ip), ("rxyz", _dp), ("uv", _dp), ("ia_tbl", _ip), ("rinv_uvu", _dp),
        ("zekr", _dp),
        ("stencil_rgrid_mode", C.c_int),
        ("nonorth", C.c_int), ("rmatrix_B", C.c_double * 9), ("coef_F", C.c_double * 6),
        ("ac_micro", _dp), ("div_ac", _dp),
        ("symmetrized", C.c_int),
        ("cap_on", C.c_int), ("cap_w0", C.c_double), ("cap_dr", C.c_double), ("cap_al", C.c_double),
        ("length_gauge", C.c_int), ("aetrs", C.c_int), ("pred_corr", C.c_int), ("gs_interval", C.c_int),
    ]


def build(force: bool = False) -> str:
    src_mtime = max(os.path.getmtime(os.path.join(HERE, f)) for f in _SOURCES)
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < src_mtime:
        subprocess.run(["make", "-s", "-C", HERE], check=True, env=dict(os.environ, ORACLE_CXX="g++"))
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        for name in ("sbo_zstencil", "sbo_dstencil", "sbo_update_kvector_nonlocalpt", "sbo_zpseudo",
                     "sbo_dpseudo", "sbo_zprojections", "sbo_hpsi", "sbo_hpsi_tt", "sbo_calc_eigen_energy",
                     "sbo_hpsi_real", "sbo_taylor",
                     "sbo_calc_density", "sbo_calc_current", "sbo_calc_microscopic_current", "sbo_current_parts", "sbo_calc_dip",
                     "sbo_calc_Ac_ext_t", "sbo_rt_run", "sbo_set_threads", "sbo_get_threads",
                     "sbo_precond_real", "sbo_gscg_rwf", "sbo_gram_schmidt_real", "sbo_gram_schmidt_complex",
                     "sbo_subspace_diag_real", "sbo_inner_product_real", "sbo_exc_cor_pz", "sbo_poisson_coef",
                     "sbo_dft_table", "sbo_poisson_ft", "sbo_update_vlocal", "sbo_rt_run_scf",
                     "sbo_poisson_isolated_ft", "sbo_impulse_kick", "sbo_exc_cor_pz_sp", "sbo_poisson_isolated_cg", "sbo_ylm", "sbo_rt_run_scf_cg"):
            getattr(L, name)
        L.sbo_rt_run.restype = C.c_int
        L.sbo_rt_run_scf.restype = C.c_int
        L.sbo_rt_run_scf_cg.restype = C.c_int
        L.sbo_get_threads.restype = C.c_int
        L.sbo_ylm.restype = C.c_double
        _lib = L
    return _lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class Oracle:
    """Holds one ``sbo_system`` built from a :class:`salmon2_b200.synth.System`."""

    def __init__(self, system, threads: int | None = None, rgrid_mode: bool | None = None):
        self.sys = system
        g, pp = system.grid, system.pp
        self._keep = []
        s = SboSystem()
        for d in range(3):
            s.is_[d], s.ie[d] = int(g.is_[d]), int(g.ie[d])
            s.is_array[d], s.ie_array[d] = int(g.is_array[d]), int(g.ie_array[d])
            s.lg_num[d] = int(g.num[d])
            s.hgs[d] = float(g.hgs[d])
        self.idx, self.idy, self.idz = (np.ascontiguousarray(a, dtype=np.int32) for a in (g.idx, g.idy, g.idz))
        s.idx, s.idy, s.idz = _p(self.idx, _ip), _p(self.idy, _ip), _p(self.idz, _ip)
        s.coef_lap0 = g.coef_lap0
        for i, v in enumerate(np.asarray(g.coef_lap).ravel(order="F")):
            s.coef_lap[i] = v
        for i, v in enumerate(np.asarray(g.coef_nab).ravel(order="F")):
            s.coef_nab[i] = v
        s.periodic = 1 if g.periodic else 0
        s.nspin, s.no, s.nk = system.nspin, system.no, system.nk
        s.hvol = g.hvol
        s.ngrid = system.ngrid
        self.vec_k = np.asfortranarray(system.vec_k, dtype=np.float64)
        self.rocc = np.asfortranarray(system.rocc, dtype=np.float64)
        self.wtk = np.ascontiguousarray(system.wtk, dtype=np.float64)
        self.V = np.asfortranarray(system.V_local, dtype=np.float64)
        s.vec_k, s.rocc, s.wtk, s.V_local = _p(self.vec_k), _p(self.rocc), _p(self.wtk), _p(self.V)
        lat = getattr(system, "lattice", None)
        rB = np.eye(3) if lat is None else np.asarray(lat.rmatrix_B, dtype=np.float64)
        bt = rB.T
        for i in range(9):
            s.BT[i] = float(bt.ravel(order="F")[i])
            s.rmatrix_B[i] = float(rB.ravel(order="F")[i])
        if lat is not None:
            s.nonorth = 1
            for i in range(6):
                s.coef_F[i] = float(lat.coef_F[i])
        s.natom, s.nps, s.nlma = pp.natom, pp.nps, pp.nlma
        self.mps = np.ascontiguousarray(pp.mps, dtype=np.int32)
        self.jxyz = np.asfortranarray(pp.jxyz, dtype=np.int32)
        self.rxyz = np.asfortranarray(pp.rxyz, dtype=np.float64)
        self.uv = np.asfortranarray(pp.uv, dtype=np.float64)
        self.ia_tbl = np.ascontiguousarray(pp.ia_tbl, dtype=np.int32)
        self.rinv = np.ascontiguousarray(pp.rinv_uvu, dtype=np.float64)
        nk_z = system.nk if g.periodic else 1
        self.zekr = np.zeros((max(pp.nps, 1), max(pp.nlma, 1), nk_z), dtype=np.complex128, order="F")
        s.mps, s.jxyz, s.rxyz, s.uv = _p(self.mps, _ip), _p(self.jxyz, _ip), _p(self.rxyz), _p(self.uv)
        s.ia_tbl, s.rinv_uvu, s.zekr = _p(self.ia_tbl, _ip), _p(self.rinv), _p(self.zekr)
        if rgrid_mode is None:  # code_optimization.f90:59-63
            rgrid_mode = int(np.prod(g.shape)) >= 32 ** 3
        s.stencil_rgrid_mode = 1 if rgrid_mode else 0
        self.s = s
        if threads:
            lib().sbo_set_threads(int(threads))
        self.set_vec_Ac((0.0, 0.0, 0.0))

    # -- state ------------------------------------------------------------
    def set_vec_Ac(self, ac):
        for d in range(3):
            self.s.vec_Ac[d] = float(ac[d])
        if self.sys.pp.nlma > 0:
            lib().sbo_update_kvector_nonlocalpt(C.byref(self.s))

    def set_micro_ac(self, ac_micro, div_ac=None, symmetrized=False):
        """system%Ac_micro%v (3, nx, ny, nz) and system%div_Ac%f (nx, ny, nz) for the
        single-scale hpsi branch; None switches it off (div_ac None: zero).
        symmetrized: yn_symmetrized_stencil = 'y'."""
        self.s.symmetrized = 1 if symmetrized else 0
        if ac_micro is None:
            self._acm = self._div = None
            self.s.ac_micro = self.s.div_ac = None
            return
        self._acm = np.asfortranarray(ac_micro, dtype=np.float64)
        if div_ac is None:
            div_ac = np.zeros(self._acm.shape[1:])
        self._div = np.asfortranarray(div_ac, dtype=np.float64)
        self.s.ac_micro, self.s.div_ac = _p(self._acm), _p(self._div)

    def set_vec_Ac_local_only(self, ac):
        """Change system%vec_Ac without refreshing zekr (calc_current's order)."""
        for d in range(3):
            self.s.vec_Ac[d] = float(ac[d])

    # -- operators ---------------------------------------------------------
    def _orb(self, psi):
        a = np.asfortranarray(psi, dtype=np.complex128)
        assert a.shape[:3] == self.sys.grid.shape_array
        return a

    def hpsi(self, psi):
        a = self._orb(psi)
        out = np.zeros_like(a, order="F")
        lib().sbo_hpsi(C.byref(self.s), _p(a), _p(out))
        return out

    def hpsi_tt(self, psi):
        """(H psi, T psi): hpsi with its optional kinetic output ttpsi."""
        a = self._orb(psi)
        h = np.zeros_like(a, order="F")
        tt = np.zeros_like(a, order="F")
        lib().sbo_hpsi_tt(C.byref(self.s), _p(a), _p(h), _p(tt))
        return h, tt

    def calc_eigen_energy(self, psi):
        """(esp(no,nk,nspin), E_kin, E_ion_nloc) of calc_eigen_energy."""
        a = self._orb(psi)
        h = np.zeros_like(a, order="F")
        tt = np.zeros_like(a, order="F")
        esp = np.zeros((self.sys.no, self.sys.nk, self.sys.nspin), order="F")
        e = np.zeros(2)
        lib().sbo_calc_eigen_energy(C.byref(self.s), _p(a), _p(h), _p(tt), _p(esp), _p(e))
        return esp, float(e[0]), float(e[1])

    def hpsi_real(self, psi):
        a = np.asfortranarray(psi, dtype=np.float64)
        out = np.zeros_like(a, order="F")
        lib().sbo_hpsi_real(C.byref(self.s), _p(a), _p(out))
        return out

    def zpseudo(self, psi):
        """Nonlocal term alone: zpseudo applied to a zero htpsi."""
        a = self._orb(psi)
        out = np.zeros_like(a, order="F")
        lib().sbo_zpseudo(C.byref(self.s), _p(a), _p(out))
        return out

    def projections(self, psi):
        a = self._orb(psi)
        out = np.zeros((self.sys.pp.nlma, self.sys.norb), dtype=np.complex128, order="F")
        lib().sbo_zprojections(C.byref(self.s), _p(a), _p(out))
        return out

    def taylor(self, psi, zc):
        tin = self._orb(psi).copy(order="F")
        tout = np.zeros_like(tin, order="F")
        work = np.zeros_like(tin, order="F")
        zc = np.ascontiguousarray(zc, dtype=np.complex128)
        lib().sbo_taylor(C.byref(self.s), _p(tin), _p(tout),
                         _p(work), _p(zc), C.c_int(len(zc)))
        return tout

    def impulse_kick(self, psi, e_impulse, epdir=(0.0, 0.0, 1.0)):
        """Kicked copy of psi: exp(i e_impulse epdir.r) psi (initialization_rt.f90:382-423)."""
        a = self._orb(psi).copy(order="F")
        ep = np.ascontiguousarray(epdir, dtype=np.float64)
        lib().sbo_impulse_kick(C.byref(self.s), _p(a), C.c_double(e_impulse), _p(ep))
        return a

    def poisson_isolated_cg(self, rho, vh0=None, layout=3, lmax=4, rion=None, npole_xyz=None,
                            threshold=1e-15, maxiter=1000):
        """Isolated Hartree potential by CG with the multipole boundary
        (poisson_isolated_cg, src/poisson/poisson_isolated.f90:30-690).  rho,
        vh0: (nx, ny, nz) interior; rion: (3, natom) (default: the system's
        atoms); npole_xyz: cells of layout 3 (default: about 8 A each,
        init_poisson.f90:112-115).  Returns (Vh, iterations)."""
        g = self.sys.grid
        r = _flat_f(rho)
        v = _flat_f(np.zeros(g.shape) if vh0 is None else vh0).copy()
        ri = np.asarray(self.sys.rion if rion is None else rion, dtype=np.float64).reshape(3, -1, order="F")
        rflat = np.ascontiguousarray(ri.T)
        npx = np.asarray(multipole_cells(g.num, g.hgs) if npole_xyz is None else npole_xyz, dtype=np.int32)
        it = C.c_int(0)
        lib().sbo_poisson_isolated_cg(C.byref(self.s), _p(r), _p(v), C.c_int(layout), C.c_int(lmax), _p(rflat),
                                      C.c_int(rflat.shape[0]), npx.ctypes.data_as(_ip), C.c_double(threshold),
                                      C.c_int(maxiter), C.byref(it))
        return v.reshape(g.shape, order="F"), it.value

    def density(self, psi):
        a = self._orb(psi)
        rho = np.zeros(self.sys.grid.shape + (self.sys.nspin,), order="F")
        lib().sbo_calc_density(C.byref(self.s), _p(a), _p(rho))
        return rho

    def current(self, psi):
        a = self._orb(psi)
        cur = np.zeros((3, self.sys.nspin), order="F")
        lib().sbo_calc_current(C.byref(self.s), _p(a), _p(cur))
        return cur

    def set_gram_schmidt_interval(self, n):
        self.s.gs_interval = int(n)

    def set_predictor_corrector(self, on=True):
        """yn_predictor_corrector = 'y' (time_evolution_step's predictor_corrector)."""
        self.s.pred_corr = 1 if on else 0

    def set_propagator(self, name="middlepoint"):
        """propagator: 'middlepoint' (default) or 'aetrs' (give it the zc of the
        half step, synth.taylor_zc(dt, aetrs=True))."""
        self.s.aetrs = 1 if name == "aetrs" else 0

    def set_length_gauge(self, on=True):
        """ae_shape1 /= 'impulse' on an isolated grid: each step's Taylor expansion
        takes V_local + E_ext(itt).r (calcVbox)."""
        self.s.length_gauge = 1 if on else 0

    def set_absorbing_boundary(self, w0=None, dr=None, al_z=None):
        """absorbing_boundary = 'z' (imagnary_potential_w0 / _dr, al(3); default the
        grid's nz * hgs(3)); w0 None switches it off."""
        if w0 is None:
            self.s.cap_on = 0
            return
        g = self.sys.grid
        self.s.cap_on = 1
        self.s.cap_w0, self.s.cap_dr = float(w0), float(dr)
        self.s.cap_al = float(g.num[2] * g.hgs[2]) if al_z is None else float(al_z)

    def microscopic_current(self, psi):
        """calc_microscopic_current: (3, nx, ny, nz), Fortran order."""
        a = self._orb(psi)
        cur = np.zeros((3,) + self.sys.grid.shape, order="F")
        lib().sbo_calc_microscopic_current(C.byref(self.s), _p(a), _p(cur))
        return cur

    def current_parts(self, psi):
        a = self._orb(psi)
        out = np.zeros((10, self.sys.norb), order="F")
        lib().sbo_current_parts(C.byref(self.s), _p(a), _p(out))
        return out

    def dip(self, rho):
        r = np.asfortranarray(rho, dtype=np.float64)
        out = np.zeros(4)
        lib().sbo_calc_dip(C.byref(self.s), _p(r), _p(out))
        return out

    def rt_run(self, psi0, nt, dt, zc, Ac_ext=None, trans_longi=0):
        """nt steps of time_evolution_step; returns dict of histories + psi."""
        a = self._orb(psi0).copy(order="F")
        b = np.zeros_like(a, order="F")
        work = np.zeros_like(a, order="F")
        if Ac_ext is None:
            Ac_ext = np.zeros((3, nt + 2), order="F")
        Ac_ext = np.asfortranarray(Ac_ext, dtype=np.float64)
        Ac_ind = np.zeros_like(Ac_ext, order="F")
        Ac_tot = Ac_ext.copy(order="F")
        curr = np.zeros((3, nt), order="F")
        rbox = np.zeros((4, nt), order="F")
        rho = np.zeros(self.sys.grid.shape + (self.sys.nspin,), order="F")
        zc = np.ascontiguousarray(zc, dtype=np.complex128)
        which = lib().sbo_rt_run(C.byref(self.s), _p(a), _p(b),
                                 _p(work), C.c_int(nt), C.c_double(dt),
                                 _p(zc), C.c_int(len(zc)), _p(Ac_ext), _p(Ac_ind),
                                 _p(Ac_tot), C.c_int(trans_longi), _p(curr), _p(rbox), _p(rho))
        psi = a if which == 0 else b
        return dict(psi=psi, curr=curr, rbox=rbox, Ac_tot=Ac_tot, Ac_ind=Ac_ind, rho=rho)

    def rt_run_scf(self, psi0, nt, dt, zc, vpsl, brl, v0, Ac_ext=None, trans_longi=0, cg=None):
        """rt_run with the self-consistent potential update every step
        (time_evolution_step.f90:184-207; nspin = 1 or 2, periodic or isolated).  v0:
        V_local (nx, ny, nz) or (nx, ny, nz, 2) for the first step.  The oracle's own V_local is untouched.
        cg (isolated grids): dict(vh0=..., layout=3, lmax=4, rion=None,
        npole_xyz=None, threshold=1e-15, maxiter=1000) selects the CG Hartree
        solve with the Vh extrapolation; the result then has "Vh" and "cg_iters"."""
        a = self._orb(psi0).copy(order="F")
        b = np.zeros_like(a, order="F")
        work = np.zeros_like(a, order="F")
        if Ac_ext is None:
            Ac_ext = np.zeros((3, nt + 2), order="F")
        Ac_ext = np.asfortranarray(Ac_ext, dtype=np.float64)
        Ac_ind = np.zeros_like(Ac_ext, order="F")
        Ac_tot = Ac_ext.copy(order="F")
        curr = np.zeros((3, nt), order="F")
        rbox = np.zeros((4, nt), order="F")
        rho = np.zeros(self.sys.grid.shape + (self.sys.nspin,), order="F")
        zc = np.ascontiguousarray(zc, dtype=np.complex128)
        vp = _flat_f(vpsl)
        bb = np.ascontiguousarray(np.asarray(brl, dtype=np.float64).ravel(order="F"))
        vl = _flat_f(v0).copy()
        extra = {}
        if cg is None:
            which = lib().sbo_rt_run_scf(C.byref(self.s), _p(a), _p(b), _p(work), C.c_int(nt), C.c_double(dt),
                                         _p(zc), C.c_int(len(zc)), _p(Ac_ext), _p(Ac_ind), _p(Ac_tot),
                                         C.c_int(trans_longi), _p(curr), _p(rbox), _p(rho), _p(vp), _p(bb), _p(vl))
        else:
            g = self.sys.grid
            vh = _flat_f(cg["vh0"]).copy()
            ri = np.asarray(self.sys.rion if cg.get("rion") is None else cg["rion"], dtype=np.float64)
            rflat = np.ascontiguousarray(ri.reshape(3, -1, order="F").T)
            npx = cg.get("npole_xyz")
            npx = np.asarray(multipole_cells(g.num, g.hgs) if npx is None else npx, dtype=np.int32)
            iters = np.zeros(nt, dtype=np.int32)
            which = lib().sbo_rt_run_scf_cg(
                C.byref(self.s), _p(a), _p(b), _p(work), C.c_int(nt), C.c_double(dt), _p(zc), C.c_int(len(zc)),
                _p(Ac_ext), _p(Ac_ind), _p(Ac_tot), C.c_int(trans_longi), _p(curr), _p(rbox), _p(rho), _p(vp),
                _p(vl), _p(vh), C.c_int(cg.get("layout", 3)), C.c_int(cg.get("lmax", 4)), _p(rflat),
                C.c_int(rflat.shape[0]), npx.ctypes.data_as(_ip), C.c_double(cg.get("threshold", 1e-15)),
                C.c_int(cg.get("maxiter", 1000)), iters.ctypes.data_as(_ip))
            extra = dict(Vh=vh.reshape(g.shape, order="F"), cg_iters=iters)
        assert which in (0, 1), "rt_run_scf with cg needs an isolated system"
        psi = a if which == 0 else b
        vshape = self.sys.grid.shape + ((self.sys.nspin,) if self.sys.nspin == 2 else ())
        return dict(psi=psi, curr=curr, rbox=rbox, Ac_tot=Ac_tot, rho=rho,
                    V_local=vl.reshape(vshape, order="F"), **extra)

    # -- ground state (real orbitals, one k) --------------------------------
    def _real(self, psi):
        a = np.asfortranarray(psi, dtype=np.float64)
        assert a.shape[:3] == self.sys.grid.shape_array
        return a

    def precond_real(self, g, alpha=0.6):
        a = self._real(g)
        out = np.zeros_like(a, order="F")
        lib().sbo_precond_real(C.byref(self.s), _p(a), _p(out), C.c_double(alpha))
        return out

    def gscg(self, psi, ncg=4, precondition=False, alpha=0.6):
        a = self._real(psi).copy(order="F")
        work = np.zeros((7,) + a.shape, order="F")
        esp = np.zeros(self.sys.nspin * self.sys.no)
        lib().sbo_gscg_rwf(C.byref(self.s), C.c_int(ncg), _p(a), _p(work), C.c_int(1 if precondition else 0),
                           C.c_double(alpha), _p(esp))
        return a, esp

    def gram_schmidt_real(self, psi):
        a = self._real(psi).copy(order="F")
        lib().sbo_gram_schmidt_real(C.byref(self.s), _p(a))
        return a

    def gram_schmidt_complex(self, psi):
        a = self._orb(psi).copy(order="F")
        lib().sbo_gram_schmidt_complex(C.byref(self.s), _p(a))
        return a

    def subspace_diag_real(self, psi):
        a = self._real(psi).copy(order="F")
        work = np.zeros_like(a, order="F")
        ev = np.zeros(self.sys.nspin * self.sys.no)
        lib().sbo_subspace_diag_real(C.byref(self.s), _p(a), _p(work), _p(ev))
        return a, ev

    def inner_real(self, x, y):
        out = np.zeros(self.sys.nspin * self.sys.no)
        lib().sbo_inner_product_real(C.byref(self.s), _p(self._real(x)), _p(self._real(y)), _p(out))
        return out


# ---- per-step potential update (salmon_oracle_scf.cpp) ----------------------

def _flat_f(a):
    """(nx, ny, nz[, ...]) array -> contiguous float64 vector, x fastest."""
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))


def multipole_cells(num, hgs):
    """Cells per axis of multipole layout 3 when num_multipole_xyz is 0:
    int((al + s) / s - 1e-8) with s = 8 A (src/poisson/init_poisson.f90:112-115)."""
    sp = 8.0 / 0.52917721067
    return [int((float(n) * float(h) + sp) / sp - 1e-8) for n, h in zip(num, hgs)]


def ylm(x, y, z, lm):
    return lib().sbo_ylm(C.c_double(x), C.c_double(y), C.c_double(z), C.c_int(lm))


def exc_cor_pz(rho, hvol):
    """PZ-LDA for nspin = 1 (builtin_pz.f90, salmon_xc.f90:86-254).  rho: (nx, ny, nz)
    interior, Fortran order.  Returns (Vxc with rho's shape, E_xc)."""
    r = _flat_f(rho)
    v = np.zeros_like(r)
    e = C.c_double(0.0)
    lib().sbo_exc_cor_pz(C.c_long(r.size), _p(r), C.c_double(hvol), _p(v), C.byref(e))
    return v.reshape(np.shape(rho), order="F"), e.value


def exc_cor_pz_sp(rho_s, hvol):
    """PZ-LDA for nspin = 2 (builtin_pz_sp.f90).  rho_s: (nx, ny, nz, 2) interior,
    Fortran order.  Returns (Vxc_s with rho_s's shape, E_xc)."""
    r = _flat_f(rho_s)
    v = np.zeros_like(r)
    e = C.c_double(0.0)
    lib().sbo_exc_cor_pz_sp(C.c_long(r.size // 2), _p(r), C.c_double(hvol), _p(v), C.byref(e))
    return v.reshape(np.shape(rho_s), order="F"), e.value


def primitive_b_orthogonal(lengths):
    """Reciprocal primitive vectors 2 pi / L_d of an orthogonal cell, (3,3) with
    column j = b_j (system%primitive_b)."""
    return np.diag([2.0 * np.pi / float(L) for L in lengths])


def poisson_coef(num, brl):
    out = np.zeros(int(np.prod(num)))
    n = np.asarray(num, dtype=np.int32)
    b = np.ascontiguousarray(np.asarray(brl, dtype=np.float64).ravel(order="F"))
    lib().sbo_poisson_coef(n.ctypes.data_as(C.POINTER(C.c_int)), _p(b), _p(out))
    return out


def poisson_ft(rho, brl):
    """Periodic Hartree potential (poisson_ft, poisson_periodic.f90:23-242).
    rho: (nx, ny, nz) interior, Fortran order; brl: (3,3) primitive_b."""
    r = _flat_f(rho)
    v = np.zeros_like(r)
    n = np.asarray(np.shape(rho), dtype=np.int32)
    b = np.ascontiguousarray(np.asarray(brl, dtype=np.float64).ravel(order="F"))
    lib().sbo_poisson_ft(n.ctypes.data_as(C.POINTER(C.c_int)), _p(b), _p(r), _p(v))
    return v.reshape(np.shape(rho), order="F")


def poisson_isolated_ft(rho, brl):
    """Isolated Hartree potential by transforms on a doubled box
    (poisson_isolated_ft, poisson_isolated.f90:692-836).  rho: (nx, ny, nz)
    interior, Fortran order; brl: (3,3) primitive_b of the (orthogonal) box."""
    r = _flat_f(rho)
    v = np.zeros_like(r)
    n = np.asarray(np.shape(rho), dtype=np.int32)
    b = np.ascontiguousarray(np.asarray(brl, dtype=np.float64).ravel(order="F"))
    lib().sbo_poisson_isolated_ft(n.ctypes.data_as(C.POINTER(C.c_int)), _p(b), _p(r), _p(v))
    return v.reshape(np.shape(rho), order="F")


def update_vlocal(vpsl, vh, vxc):
    """update_vlocal (hamiltonian.f90:813-843).  vpsl, vh: (nx, ny, nz);
    vxc: (nx, ny, nz, nspin).  Returns V_local (nx, ny, nz, nspin)."""
    vxc = np.asarray(vxc, dtype=np.float64)
    nspin = vxc.shape[3]
    a, b, c = _flat_f(vpsl), _flat_f(vh), _flat_f(vxc)
    out = np.zeros_like(c)
    lib().sbo_update_vlocal(C.c_long(a.size), C.c_int(nspin), _p(a), _p(b), _p(c), _p(out))
    return out.reshape(vxc.shape, order="F")
