"""Kleinman-Bylander tables and the local potential from pseudopotential
files through the library's host-side builder: Yabana-Bertsch files
(`_rps.dat`, ps_format = 'KY') with sb200_init_ps_ky, and any one-projector
format chosen by the file name (`_rps.dat`, `.pspnc` ABINIT, `.fhi`
ABINITFHI, `.cpi` FHI) with sb200_init_ps (input_pp.f90 read_ps_*,
making_ps_without_masking, prep_pp.f90 init_ps, calc_Vpsl_isolated /
calc_Vpsl_periodic)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib
from .synth import PPGrid

_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)


def init_ps_ky(files, lloc_ps, grid, rion, kion, lmax_ps=None, vpsl=True):
    """files: one path per element; lloc_ps / lmax_ps: per element (Lloc_ps,
    Lmax_ps; lmax_ps None keeps the file's); grid: a synth.Grid (orthogonal);
    rion: (3, natom) bohr; kion: 1-based element of each atom.  Returns
    (PPGrid, Vpsl (nx, ny, nz) Fortran order, or None with vpsl=False)."""
    return _init_ps("sb200_init_ps_ky", files, lloc_ps, grid, rion, kion, lmax_ps, vpsl)


def init_ps(files, lloc_ps, grid, rion, kion, lmax_ps=None, vpsl=True):
    """init_ps_ky for every one-projector format, chosen by the file name."""
    return _init_ps("sb200_init_ps", files, lloc_ps, grid, rion, kion, lmax_ps, vpsl)


def _init_ps(entry, files, lloc_ps, grid, rion, kion, lmax_ps, vpsl):
    fn = getattr(lib(), entry)
    nelem = len(files)
    arr = (C.c_char_p * nelem)(*[str(f).encode() for f in files])
    lloc = np.ascontiguousarray(lloc_ps, dtype=np.int32)
    lmax = None if lmax_ps is None else np.ascontiguousarray(lmax_ps, dtype=np.int32)
    num = np.ascontiguousarray(grid.num, dtype=np.int32)
    is_ = np.ascontiguousarray(grid.is_, dtype=np.int32)
    hgs = np.ascontiguousarray(grid.hgs, dtype=np.float64)
    r = np.ascontiguousarray(np.asarray(rion, dtype=np.float64).reshape(3, -1, order="F").T)
    natom = r.shape[0]
    k = np.ascontiguousarray(kion, dtype=np.int32)
    nps, nlma = C.c_int(0), C.c_int(0)
    P = lambda a, t=_dp: None if a is None else a.ctypes.data_as(t)
    args = [nelem, arr, P(lmax, _ip), P(lloc, _ip), 1 if grid.periodic else 0, P(num, _ip), P(is_, _ip), P(hgs),
            float(grid.hvol), natom, P(k, _ip), P(r)]
    check(fn(*args, C.byref(nps), C.byref(nlma), None, None, None, None, None, None, None))
    n, m = nps.value, nlma.value
    mps = np.zeros(natom, dtype=np.int32)
    jxyz = np.zeros((3, n, natom), dtype=np.int32, order="F")
    rxyz = np.zeros((3, n, natom), dtype=np.float64, order="F")
    uv = np.zeros((n, m), dtype=np.float64, order="F")
    ia = np.zeros(m, dtype=np.int32)
    rinv = np.zeros(m, dtype=np.float64)
    v = np.zeros(tuple(grid.num), dtype=np.float64, order="F") if vpsl else None
    check(fn(*args, C.byref(nps), C.byref(nlma), P(mps, _ip), P(jxyz, _ip), P(rxyz), P(uv),
                                 P(ia, _ip), P(rinv), P(v)))
    return PPGrid(natom, n, m, mps, jxyz, rxyz, uv, ia, rinv), v


def set_psmask(yn_psmask, alpha_mask=0.8, gamma_mask=1.8, eta_mask=15.0):
    """yn_psmask and its parameters for the following set-ups (process-wide, as
    the reference's input variables): masked radial KB functions
    (making_ps_with_masking, input_pp.f90:848-1016)."""
    check(lib().sb200_set_psmask(1 if yn_psmask else 0, float(alpha_mask), float(gamma_mask), float(eta_mask)))
