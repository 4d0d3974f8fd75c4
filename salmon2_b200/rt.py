"""Host-side mirror of SALMON's hpsi / taylor call surface over the C ABI.

``Context`` holds one device-resident copy of the tables the reference passes
to ``hpsi`` (``src/common/hamiltonian.f90:27``) and ``taylor``
(``src/rt/taylor.f90:21``): the grid and stencil (``s_rgrid``, ``s_stencil``),
the orbital block (``info``/``system``: nspin, io, ik, vec_k, rocc, wtk),
``V_local`` and the projector tables (``s_pp_grid``).  Orbitals live on the GPU
in the library's resident layout as torch ``complex128`` tensors of shape
``[norb, nz, ny, nx]``; :meth:`Context.upload` / :meth:`Context.download`
convert from / to the reference's Fortran layout.

Errors raise :class:`salmon2_b200._lib.SB200Error` (the reference stops the
program; here the caller gets the library's status code and message).  PyTorch
only provides device memory and streams; all arithmetic runs in
``libsalmon_b200.so``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import SB200Error, check, lib  # noqa: F401

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def _i3(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def nccl_unique_id() -> bytes:
    """128-byte NCCL id (on rank 0) for :meth:`Context.set_density_comm`."""
    buf = (C.c_ubyte * 128)()
    check(lib().sb200_nccl_unique_id(buf))
    return bytes(buf)


class Context:
    """Device context for one orbital block (one ``(ik, io, ispin)`` set)."""

    def __init__(self, system, device: int = 0, precision: str = "fp64"):
        import torch

        self.torch = torch
        self.sys = system
        self.device = device
        h = C.c_void_p()
        check(lib().sb200_ctx_create(int(device), C.byref(h)))
        self.h = h
        g = system.grid
        self._keep = []
        idx = [np.ascontiguousarray(a, dtype=np.int32) for a in (g.idx, g.idy, g.idz)]
        lap = np.ascontiguousarray(np.asarray(g.coef_lap).ravel(order="F"))
        nab = np.ascontiguousarray(np.asarray(g.coef_nab).ravel(order="F"))
        hgs = np.ascontiguousarray(g.hgs, dtype=np.float64)
        check(lib().sb200_set_grid(self.h, _i3(g.is_), _i3(g.ie), _i3(g.is_array), _i3(g.ie_array),
                                   _ptr(idx[0], _ip), _ptr(idx[1], _ip), _ptr(idx[2], _ip), _i3(g.num),
                                   _ptr(hgs), g.hvol, g.coef_lap0, _ptr(lap), _ptr(nab)))
        vec_k = np.asfortranarray(system.vec_k, dtype=np.float64)
        rocc = np.asfortranarray(system.rocc, dtype=np.float64)
        wtk = np.ascontiguousarray(system.wtk, dtype=np.float64)
        check(lib().sb200_set_orbitals(self.h, system.nspin, system.no, system.nk, _ptr(vec_k), _ptr(rocc),
                                       _ptr(wtk)))
        V = np.asfortranarray(system.V_local, dtype=np.float64)
        check(lib().sb200_set_vlocal(self.h, _ptr(V)))
        lat = getattr(system, "lattice", None)
        if lat is not None:  # non-orthogonal cell: rmatrix_B and coef_F of init_lattice
            rB = np.asfortranarray(lat.rmatrix_B, dtype=np.float64)
            F = np.ascontiguousarray(lat.coef_F, dtype=np.float64)
            check(lib().sb200_set_lattice(self.h, _ptr(rB), _ptr(F)))
        self.set_pp(system.pp)
        self.set_precision(precision)
        self.shape = (system.norb, g.shape[2], g.shape[1], g.shape[0])

    # -- set-up -------------------------------------------------------------
    def set_pp(self, pp):
        mps = np.ascontiguousarray(pp.mps, dtype=np.int32)
        jxyz = np.asfortranarray(pp.jxyz, dtype=np.int32)
        rxyz = np.asfortranarray(pp.rxyz, dtype=np.float64)
        uv = np.asfortranarray(pp.uv, dtype=np.float64)
        ia = np.ascontiguousarray(pp.ia_tbl, dtype=np.int32)
        rinv = np.ascontiguousarray(pp.rinv_uvu, dtype=np.float64)
        check(lib().sb200_set_pp(self.h, pp.natom, pp.nps, pp.nlma, _ptr(mps, _ip), _ptr(jxyz, _ip), _ptr(rxyz),
                                 _ptr(uv), _ptr(ia, _ip), _ptr(rinv)))

    def set_micro_ac(self, ac_micro, div_ac=None, symmetrized=False):
        """Single-scale hpsi (hamiltonian.f90:236-298): Ac_micro (3, nx, ny, nz)
        and div_Ac (nx, ny, nz), Fortran order; None turns it off (div_ac None:
        zero).  symmetrized: yn_symmetrized_stencil = 'y'
        (zstencil_microAc_symmetrized, stencil.f90:319-411)."""
        check(lib().sb200_set_symmetrized_stencil(self.h, 1 if symmetrized else 0))
        if ac_micro is None:
            check(lib().sb200_set_micro_ac(self.h, None, None))
            return
        a = np.asfortranarray(ac_micro, dtype=np.float64)
        d = None if div_ac is None else np.asfortranarray(div_ac, dtype=np.float64)
        check(lib().sb200_set_micro_ac(self.h, C.c_void_p(a.ctypes.data),
                                       None if d is None else C.c_void_p(d.ctypes.data)))

    def set_gram_schmidt_interval(self, n):
        """gram_schmidt_interval: rt_propagate orthonormalises psi(t+dt) every n steps."""
        check(lib().sb200_set_gram_schmidt_interval(self.h, int(n)))

    def set_predictor_corrector(self, on=True):
        """yn_predictor_corrector = 'y' (time_evolution_step's predictor_corrector)."""
        check(lib().sb200_set_predictor_corrector(self.h, 1 if on else 0))

    def set_propagator(self, name="middlepoint"):
        """propagator = 'middlepoint' or 'aetrs' (rt_propagate then takes the zc of
        the half step, synth.taylor_zc(dt, aetrs=True))."""
        check(lib().sb200_set_propagator(self.h, {"middlepoint": 0, "aetrs": 1}[name]))

    def set_length_gauge(self, on=True):
        """An isolated system driven by a pulse in the length gauge (ae_shape1 /=
        'impulse'): rt_propagate adds E_ext(itt).r to V_local every step."""
        check(lib().sb200_set_length_gauge(self.h, 1 if on else 0))

    def set_absorbing_boundary(self, w0=None, dr=None, al_z=None):
        """absorbing_boundary = 'z' with imagnary_potential_w0 / _dr and the cell
        length al(3) (default: the grid's nz * hgs(3)); w0 None switches it off."""
        if w0 is None:
            check(lib().sb200_set_absorbing_boundary(self.h, 0, 0.0, 0.0, 0.0))
            return
        g = self.sys.grid
        L = float(g.num[2] * g.hgs[2]) if al_z is None else float(al_z)
        check(lib().sb200_set_absorbing_boundary(self.h, 1, float(w0), float(dr), L))

    def calc_microscopic_current(self, psi):
        """calc_microscopic_current (density_matrix.f90:726-845): (3, nx, ny, nz),
        Fortran order."""
        g = self.sys.grid
        cur = np.zeros((3,) + g.shape, order="F")
        check(lib().sb200_calc_microscopic_current(self.h, C.c_void_p(psi.data_ptr()), C.c_void_p(cur.ctypes.data)))
        return cur

    def set_vec_Ac(self, vec_Ac):
        a = np.ascontiguousarray(vec_Ac, dtype=np.float64)
        check(lib().sb200_set_vec_Ac(self.h, _ptr(a)))

    def impulse_kick(self, psi, e_impulse, epdir=(0.0, 0.0, 1.0)):
        """psi <- exp(i e_impulse epdir.r) psi on the device (initialization_rt's impulse)."""
        ep = np.ascontiguousarray(epdir, dtype=np.float64)
        check(lib().sb200_impulse_kick(self.h, C.c_void_p(psi.data_ptr()), float(e_impulse), _ptr(ep)))
        return psi

    def set_precision(self, precision: str):
        mode = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[precision]
        check(lib().sb200_set_precision(self.h, mode))

    def close(self):
        if getattr(self, "h", None):
            lib().sb200_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        check(lib().sb200_ctx_sync(self.h))

    def set_stream(self, stream):
        """Run on a caller-owned stream (a torch.cuda.Stream), or None."""
        check(lib().sb200_ctx_set_stream(self.h, None if stream is None else C.c_void_p(stream.cuda_stream)))

    def set_timing(self, enable: bool):
        check(lib().sb200_set_timing(self.h, 1 if enable else 0))

    def kernel_times(self, reset: bool = True):
        ms = (C.c_double * 8)()
        cnt = (C.c_long * 8)()
        check(lib().sb200_kernel_times(self.h, ms, cnt, 1 if reset else 0))
        return {_lib.KIND_NAMES[i]: (ms[i], cnt[i]) for i in range(8) if cnt[i] > 0}

    # -- orbital blocks -------------------------------------------------------
    def empty(self):
        return self.torch.empty(self.shape, dtype=self.torch.complex128, device=f"cuda:{self.device}")

    def zeros(self):
        return self.torch.zeros(self.shape, dtype=self.torch.complex128, device=f"cuda:{self.device}")

    def upload(self, zwf_ref, out=None):
        """Reference-layout orbitals (numpy, Fortran order, or a pinned torch
        tensor holding the same bytes) -> resident device block."""
        out = self.empty() if out is None else out
        if isinstance(zwf_ref, np.ndarray):
            src = np.asfortranarray(zwf_ref, dtype=np.complex128)
            check(lib().sb200_orbitals_from_ref(self.h, C.c_void_p(src.ctypes.data), C.c_void_p(out.data_ptr())))
        else:
            check(lib().sb200_orbitals_from_ref(self.h, C.c_void_p(zwf_ref.data_ptr()),
                                                C.c_void_p(out.data_ptr())))
        return out

    def download(self, psi, out=None):
        g = self.sys.grid
        if out is None:
            out = np.zeros(g.shape_array + (self.sys.nspin, self.sys.no, self.sys.nk), dtype=np.complex128,
                           order="F")
            check(lib().sb200_orbitals_to_ref(self.h, C.c_void_p(psi.data_ptr()), C.c_void_p(out.ctypes.data)))
        else:
            check(lib().sb200_orbitals_to_ref(self.h, C.c_void_p(psi.data_ptr()), C.c_void_p(out.data_ptr())))
        return out

    # -- the hot path -----------------------------------------------------------
    def hpsi(self, tpsi, htpsi):
        check(lib().sb200_hpsi(self.h, C.c_void_p(tpsi.data_ptr()), C.c_void_p(htpsi.data_ptr())))
        return htpsi

    def hpsi_tt(self, tpsi, htpsi, ttpsi):
        """H psi and its kinetic part T psi (hpsi's optional ttpsi)."""
        check(lib().sb200_hpsi_tt(self.h, C.c_void_p(tpsi.data_ptr()), C.c_void_p(htpsi.data_ptr()),
                                  C.c_void_p(ttpsi.data_ptr())))
        return htpsi, ttpsi

    def calc_eigen_energy(self, psi, htpsi=None, ttpsi=None):
        """(esp(no,nk,nspin), E_kin, E_ion_nloc) of calc_eigen_energy; htpsi and
        ttpsi are work blocks (allocated when not given)."""
        htpsi = self.zeros() if htpsi is None else htpsi
        ttpsi = self.zeros() if ttpsi is None else ttpsi
        esp = np.zeros((self.sys.no, self.sys.nk, self.sys.nspin), order="F")
        ek, en = np.zeros(1), np.zeros(1)
        check(lib().sb200_calc_eigen_energy(self.h, C.c_void_p(psi.data_ptr()), C.c_void_p(htpsi.data_ptr()),
                                            C.c_void_p(ttpsi.data_ptr()), _ptr(esp), _ptr(ek), _ptr(en)))
        return esp, float(ek[0]), float(en[0])

    def taylor(self, tspsi_in, tspsi_out, sshtpsi, zc):
        z = np.ascontiguousarray(zc, dtype=np.complex128)
        check(lib().sb200_taylor(self.h, C.c_void_p(tspsi_in.data_ptr()), C.c_void_p(tspsi_out.data_ptr()),
                                 C.c_void_p(sshtpsi.data_ptr()), z.ctypes.data_as(_dp), len(z)))
        return tspsi_out

    def calc_density(self, psi):
        g = self.sys.grid
        rho = np.zeros(g.shape + (self.sys.nspin,), order="F")
        check(lib().sb200_calc_density(self.h, C.c_void_p(psi.data_ptr()), C.c_void_p(rho.ctypes.data)))
        return rho

    def calc_current(self, psi, vec_Ac):
        a = np.ascontiguousarray(vec_Ac, dtype=np.float64)
        cur = np.zeros((3, self.sys.nspin), order="F")
        check(lib().sb200_calc_current(self.h, C.c_void_p(psi.data_ptr()), _ptr(a), _ptr(cur)))
        return cur

    def calc_dip(self, rho):
        if isinstance(rho, np.ndarray):
            r = np.asfortranarray(rho, dtype=np.float64)
            p = C.c_void_p(r.ctypes.data)
        else:
            p = C.c_void_p(rho.data_ptr())
        out = np.zeros(4)
        check(lib().sb200_calc_dip(self.h, p, _ptr(out)))
        return out

    # ---- per-step potential update (time_evolution_step.f90:184-207) ----

    @staticmethod
    def _scalar_field(a):
        """(pointer, keep-alive) of an interior field: a numpy array (any order,
        converted to x fastest) or a contiguous torch device tensor."""
        if isinstance(a, np.ndarray):
            f = np.asfortranarray(a, dtype=np.float64)
            return C.c_void_p(f.ctypes.data), f
        return C.c_void_p(a.data_ptr()), a

    def exc_cor_pz(self, rho):
        """exchange_correlation with xc = 'PZ' (salmon_xc.f90:58-343): nspin = 1,
        rho (nx, ny, nz) -> (Vxc (nx, ny, nz), E_xc); nspin = 2, the spin
        densities (nx, ny, nz, 2) -> (Vxc_s (nx, ny, nz, 2), E_xc), Fortran order."""
        g = self.sys.grid
        p, keep = self._scalar_field(rho)
        v = np.zeros(g.shape + ((2,) if self.sys.nspin == 2 else ()), order="F")
        e = C.c_double(0.0)
        check(lib().sb200_exc_cor_pz(self.h, p, C.c_void_p(v.ctypes.data), C.byref(e)))
        return v, e.value

    def hartree_periodic(self, rho, primitive_b):
        """hartree -> poisson_ft (poisson_periodic.f90:23-242) on a periodic grid;
        primitive_b (3, 3) with column j = b_j.  Returns Vh (nx, ny, nz)."""
        g = self.sys.grid
        b = np.asfortranarray(primitive_b, dtype=np.float64)
        p, keep = self._scalar_field(rho)
        v = np.zeros(g.shape, order="F")
        check(lib().sb200_hartree_periodic(self.h, _ptr(b), p, C.c_void_p(v.ctypes.data)))
        return v

    def hartree_isolated_ft(self, rho, primitive_b):
        """hartree -> poisson_isolated_ft (poisson_isolated.f90:692-836) on an
        isolated grid; primitive_b (3, 3) of the box.  Returns Vh (nx, ny, nz)."""
        g = self.sys.grid
        b = np.asfortranarray(primitive_b, dtype=np.float64)
        p, keep = self._scalar_field(rho)
        v = np.zeros(g.shape, order="F")
        check(lib().sb200_hartree_isolated_ft(self.h, _ptr(b), p, C.c_void_p(v.ctypes.data)))
        return v

    def hartree_isolated_cg(self, rho, vh0=None, layout=3, lmax=4, rion=None, npole_xyz=None,
                            threshold=1e-15, maxiter=1000):
        """hartree -> poisson_isolated_cg (poisson_isolated.f90:30-690) on an
        isolated grid: CG on the 25-point Laplacian from vh0 (default zero) with
        multipole boundary values (layout_multipole 1 / 2 / 3, lmax <= 4).
        rion (3, natom): atom positions (default: the system's); npole_xyz:
        cells of layout 3 (default about 8 A each).  Returns (Vh, iterations)."""
        g = self.sys.grid
        p, keep = self._scalar_field(rho)
        v = np.zeros(g.shape, order="F") if vh0 is None else np.array(vh0, dtype=np.float64, order="F")
        ri = np.asarray(self.sys.rion if rion is None else rion, dtype=np.float64).reshape(3, -1, order="F")
        rflat = np.ascontiguousarray(ri.T)
        npx = (C.c_int * 3)(*([0, 0, 0] if npole_xyz is None else [int(n) for n in npole_xyz]))
        it = C.c_int(0)
        check(lib().sb200_hartree_isolated_cg(self.h, p, C.c_void_p(v.ctypes.data), int(layout), int(lmax),
                                              _ptr(rflat), rflat.shape[0], npx, float(threshold), int(maxiter),
                                              C.byref(it)))
        return v, it.value

    def set_hartree_cg(self, vh0, layout=3, lmax=4, rion=None, npole_xyz=None, threshold=1e-15, maxiter=1000):
        """method_poisson = 'cg' for the isolated self-consistent loop
        (time_evolution_step.f90:184-198): vh0 (nx, ny, nz) the potential of the
        initial density; later steps start from the extrapolated potential.
        vh0 = None returns to the transforms."""
        if vh0 is None:
            check(lib().sb200_set_hartree_cg(self.h, None, 0, 0, None, 0, None, 0.0, 0))
            return
        p, keep = self._scalar_field(vh0)
        ri = np.asarray(self.sys.rion if rion is None else rion, dtype=np.float64).reshape(3, -1, order="F")
        rflat = np.ascontiguousarray(ri.T)
        npx = (C.c_int * 3)(*([0, 0, 0] if npole_xyz is None else [int(n) for n in npole_xyz]))
        check(lib().sb200_set_hartree_cg(self.h, p, int(layout), int(lmax), _ptr(rflat), rflat.shape[0], npx,
                                         float(threshold), int(maxiter)))

    def update_vlocal(self, vpsl, vh, vxc):
        """update_vlocal (hamiltonian.f90:813-843): V_local = Vpsl + Vh + Vxc on the
        device.  vxc: (nx, ny, nz, nspin) or (nx, ny, nz) for nspin = 1."""
        pa, ka = self._scalar_field(vpsl)
        pb, kb = self._scalar_field(vh)
        pc, kc = self._scalar_field(vxc)
        check(lib().sb200_update_vlocal(self.h, pa, pb, pc))

    def set_self_consistent(self, enable, vpsl=None, primitive_b=None):
        """Self-consistent time loop (time_evolution_step.f90:160-207 with
        yn_fix_func = 'n'): rt_propagate recomputes V_local = Vpsl + Vh[rho] +
        Vxc[rho] after every step.  enable = False returns to the fixed potential."""
        if not enable:
            check(lib().sb200_set_self_consistent(self.h, 0, None, None))
            return
        b = np.asfortranarray(primitive_b, dtype=np.float64)
        p, keep = self._scalar_field(vpsl)
        check(lib().sb200_set_self_consistent(self.h, 1, p, _ptr(b)))

    def set_density_comm(self, nranks, rank, unique_id: bytes):
        """All-reduce the density over `nranks` k-point shards (one process per
        GPU) in calc_density and the self-consistent loop; nranks = 0 removes it."""
        buf = (C.c_ubyte * 128).from_buffer_copy(unique_id) if unique_id is not None else None
        check(lib().sb200_set_density_comm(self.h, int(nranks), int(rank), buf))

    def update_potential(self, psi, vpsl, primitive_b, poisson="ft"):
        """The self-consistent part of one time step on the device
        (time_evolution_step.f90:160-207, nspin = 1 or 2; Hartree by poisson_ft on a
        periodic grid, poisson_isolated_ft on an isolated one, or with
        poisson = "cg" poisson_isolated_cg from zero with the default multipole
        boundary): rho = calc_density(psi), Vh = hartree(rho),
        Vxc = exchange_correlation(rho), V_local = Vpsl + Vh + Vxc.  vpsl: a
        device tensor (nx*ny*nz, x fastest) or a numpy array.  Nothing is copied
        to the host; returns E_xc.  The potential stays in self.last_vh.  With
        nspin = 2 the Hartree potential is that of rho_up + rho_dn and Vxc the
        spin-polarised form."""
        torch = self.torch
        ns = self.sys.nspin
        n = int(np.prod(self.sys.grid.shape))
        if getattr(self, "_pot_buf", None) is None:
            self._pot_buf = torch.empty((2 * ns + 2, n), dtype=torch.float64, device=f"cuda:{self.device}")
        buf = self._pot_buf
        rho_s, vh, vxc = buf[0:ns], buf[ns], buf[ns + 1:2 * ns + 1]
        b = np.asfortranarray(primitive_b, dtype=np.float64)
        check(lib().sb200_calc_density(self.h, C.c_void_p(psi.data_ptr()), C.c_void_p(rho_s.data_ptr())))
        rho = rho_s[0]
        if ns == 2:  # rho = sum of rho_s (time_evolution_step.f90:160-170)
            rho = buf[2 * ns + 1]
            torch.add(rho_s[0], rho_s[1], out=rho)
        if poisson == "cg" and not self.sys.grid.periodic:
            vh.zero_()
            ri = np.ascontiguousarray(np.asarray(self.sys.rion, dtype=np.float64).reshape(3, -1, order="F").T)
            it = C.c_int(0)
            check(lib().sb200_hartree_isolated_cg(self.h, C.c_void_p(rho.data_ptr()), C.c_void_p(vh.data_ptr()), 3,
                                                  4, _ptr(ri), ri.shape[0], None, 1e-15, 1000, C.byref(it)))
        else:
            hartree = lib().sb200_hartree_periodic if self.sys.grid.periodic else lib().sb200_hartree_isolated_ft
            check(hartree(self.h, _ptr(b), C.c_void_p(rho.data_ptr()), C.c_void_p(vh.data_ptr())))
        self.last_vh = vh
        e = C.c_double(0.0)
        check(lib().sb200_exc_cor_pz(self.h, C.c_void_p(rho_s.data_ptr()), C.c_void_p(vxc.data_ptr()), C.byref(e)))
        pa, keep = self._scalar_field(vpsl)
        check(lib().sb200_update_vlocal(self.h, pa, C.c_void_p(vh.data_ptr()), C.c_void_p(vxc.data_ptr())))
        return e.value

    def rt_propagate(self, psi_a, psi_b, work, nt, dt, zc, Ac_ext=None, trans_longi="tr"):
        z = np.ascontiguousarray(zc, dtype=np.complex128)
        ac = None if Ac_ext is None else np.asfortranarray(Ac_ext, dtype=np.float64)
        curr = np.zeros((3, max(nt, 1)), order="F")
        rbox = np.zeros((4, max(nt, 1)), order="F")
        act = np.zeros((3, nt + 2), order="F")
        fin = C.c_void_p()
        tl = {"tr": _lib.TRANS_TR, "lo": _lib.TRANS_LO}[trans_longi]
        check(lib().sb200_rt_propagate(self.h, C.c_void_p(psi_a.data_ptr()), C.c_void_p(psi_b.data_ptr()),
                                       C.c_void_p(work.data_ptr()), int(nt), float(dt), z.ctypes.data_as(_dp),
                                       len(z), None if ac is None else _ptr(ac), tl, _ptr(curr), _ptr(rbox),
                                       _ptr(act), C.byref(fin)))
        final = psi_a if fin.value == psi_a.data_ptr() else psi_b
        return dict(psi=final, curr=curr[:, :nt], rbox=rbox[:, :nt], Ac_tot=act)

    def rt_set_start(self, mit, ac_tot=None, ac_ind=None):
        """The next rt_propagate runs steps mit + 1 .. mit + nt (restart_rt's Mit),
        its field history from Ac_tot / Ac_ind (3, 2) at steps mit, mit + 1."""
        t = None if ac_tot is None else np.asfortranarray(ac_tot, dtype=np.float64).reshape(3, 2, order="F")
        i = None if ac_ind is None else np.asfortranarray(ac_ind, dtype=np.float64).reshape(3, 2, order="F")
        check(lib().sb200_rt_set_start(self.h, int(mit), None if t is None else _ptr(t), None if i is None else _ptr(i)))

    def rt_get_state(self):
        """(Mit, Ac_tot (3, 2), Ac_ind (3, 2)) after the last rt_propagate."""
        mit = C.c_int(0)
        t = np.zeros((3, 2), order="F")
        i = np.zeros((3, 2), order="F")
        check(lib().sb200_rt_get_state(self.h, C.byref(mit), _ptr(t), _ptr(i)))
        return mit.value, t, i

    def write_restart(self, directory, psi, iter, method="single", nblock=1, real=False, trans_longi="tr"):
        """checkpoint_rt / checkpoint_gs in the reference's file layouts."""
        tl = {"tr": _lib.TRANS_TR, "lo": _lib.TRANS_LO}[trans_longi]
        check(lib().sb200_write_restart(self.h, str(directory).encode(), {"single": 0, "slice": 1}[method],
                                        int(nblock), C.c_void_p(psi.data_ptr()), 1 if real else 0, int(iter), tl))

    def read_restart(self, directory, psi, method="single", nblock=1, yn_restart=True, ik_s=1, io_s=1):
        """restart_rt / restart_gs into the complex block psi; returns (iter,
        rocc (no, nk, nspin))."""
        it = C.c_int(0)
        rocc = np.zeros((self.sys.no, self.sys.nk, self.sys.nspin), order="F")
        check(lib().sb200_read_restart(self.h, str(directory).encode(), {"single": 0, "slice": 1}[method],
                                       int(nblock), 1 if yn_restart else 0, int(ik_s), int(io_s),
                                       C.c_void_p(psi.data_ptr()), C.byref(it), _ptr(rocc)))
        return it.value, rocc

    # -- ground state: real orbitals, one k-point ---------------------------------
    def gs_empty(self):
        return self.torch.empty(self.shape, dtype=self.torch.float64, device=f"cuda:{self.device}")

    def gs_upload(self, rwf_ref, out=None):
        out = self.gs_empty() if out is None else out
        src = np.asfortranarray(rwf_ref, dtype=np.float64)
        check(lib().sb200_gs_from_ref(self.h, C.c_void_p(src.ctypes.data), C.c_void_p(out.data_ptr())))
        return out

    def gs_download(self, psi):
        g = self.sys.grid
        out = np.zeros(g.shape_array + (self.sys.nspin, self.sys.no, 1), order="F")
        check(lib().sb200_gs_to_ref(self.h, C.c_void_p(psi.data_ptr()), C.c_void_p(out.ctypes.data)))
        return out

    def hpsi_real(self, tpsi, htpsi):
        check(lib().sb200_hpsi_real(self.h, C.c_void_p(tpsi.data_ptr()), C.c_void_p(htpsi.data_ptr())))
        return htpsi

    def gscg(self, psi, ncg=4, precondition="none", alpha=0.6):
        mode = {"none": _lib.PRECOND_NONE, "lowpass": _lib.PRECOND_LOWPASS, "learned": _lib.PRECOND_LEARNED}[
            precondition]
        esp = np.zeros(self.sys.nspin * self.sys.no)
        check(lib().sb200_gscg(self.h, C.c_void_p(psi.data_ptr()), int(ncg), mode, float(alpha), _ptr(esp)))
        return esp

    def gram_schmidt_real(self, psi):
        check(lib().sb200_gram_schmidt_real(self.h, C.c_void_p(psi.data_ptr())))
        return psi

    def gram_schmidt_complex(self, psi):
        """Column Gram-Schmidt of the resident complex orbitals, per (k, spin)."""
        check(lib().sb200_gram_schmidt_complex(self.h, C.c_void_p(psi.data_ptr())))
        return psi

    def subspace_diag_real(self, psi):
        ev = np.zeros(self.sys.no)
        check(lib().sb200_subspace_diag_real(self.h, C.c_void_p(psi.data_ptr()), _ptr(ev)))
        return ev


class Batch:
    """Independent isolated systems advanced together (sb200_batch_*).

    ``contexts`` are fully set-up :class:`Context` objects of isolated grids;
    the batch keeps references to them so they outlive it."""

    def __init__(self, contexts):
        self.ctxs = list(contexts)
        self.n = len(self.ctxs)
        arr = (C.c_void_p * self.n)(*[c.h for c in self.ctxs])
        h = C.c_void_p()
        check(lib().sb200_batch_create(arr, self.n, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().sb200_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ptrs(self, tensors):
        return (C.c_void_p * self.n)(*[t.data_ptr() for t in tensors])

    def tiles(self):
        sh = np.zeros(self.n, np.int32)
        zc = np.zeros(self.n, np.int32)
        check(lib().sb200_batch_get_tiles(self.h, sh.ctypes.data_as(_ip), zc.ctypes.data_as(_ip)))
        return sh, zc

    def set_tiles(self, shape, zchunk):
        sh = np.ascontiguousarray(shape, np.int32)
        zc = np.ascontiguousarray(zchunk, np.int32)
        check(lib().sb200_batch_set_tiles(self.h, sh.ctypes.data_as(_ip), zc.ctypes.data_as(_ip)))

    def autotune(self, psi, work, reps=3):
        sh = np.zeros(self.n, np.int32)
        zc = np.zeros(self.n, np.int32)
        check(lib().sb200_batch_autotune(self.h, self._ptrs(psi), self._ptrs(work), int(reps),
                                         sh.ctypes.data_as(_ip), zc.ctypes.data_as(_ip)))
        return sh, zc

    def propagate(self, psi_a, psi_b, work, nt, dt, zc, rbox=True):
        z = np.ascontiguousarray(zc, dtype=np.complex128)
        boxes = [np.zeros((4, max(nt, 1)), order="F") for _ in range(self.n)]
        rb = (C.c_void_p * self.n)(*[b.ctypes.data for b in boxes]) if rbox else None
        fin = (C.c_void_p * self.n)()
        check(lib().sb200_batch_propagate(self.h, self._ptrs(psi_a), self._ptrs(psi_b), self._ptrs(work), int(nt),
                                          float(dt), z.ctypes.data_as(_dp), len(z), rb, fin))
        finals = [a if fin[i] == a.data_ptr() else b for i, (a, b) in enumerate(zip(psi_a, psi_b))]
        return dict(psi=finals, rbox=[b[:, :nt] for b in boxes] if rbox else None)
