"""ctypes binding of the reference's own CUDA kernels (test infrastructure).

``oracle/_ref/libsalmon_ref_cuda.so`` is compiled, unmodified, from the
reference's ``src/common/zpseudo.cu`` and ``src/common/stencil_current.cu``
(recipe: ``make -C oracle ref``).  The two exported C functions are the
reference's GPU implementations of the KB nonlocal term and of the local part
of the current; running them on the same inputs as the oracle pins the
oracle's restatement of ``zpseudo`` and ``stencil_current``.

Both functions take the reference's Fortran array layout.  ``zpseudo_cuda``
dereferences every array pointer on the device (the reference runs it on
OpenACC-managed memory), so all its arrays are passed as device tensors.
``stencil_current_core_gpu`` copies its small tables from host memory itself
and only reads ``psi`` on the device; it supports periodic grids whose point
count is a multiple of its 128-thread block.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libsalmon_ref_cuda.so")
REF_AVX512_LIB = os.path.join(HERE, "_ref", "libsalmon_ref_avx512.so")

_lib = None


def available() -> bool:
    return os.path.exists(REF_LIB)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(REF_LIB)
        i = C.c_int
        vp = C.c_void_p
        L.zpseudo_cuda.restype = None
        L.zpseudo_cuda.argtypes = [vp] + [i] * 17 + [vp] * 6
        L.stencil_current_core_gpu.restype = None
        L.stencil_current_core_gpu.argtypes = [i, i, i, i, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i, i, i, vp, vp,
                                               vp, vp, vp, vp, vp]
        _lib = L
    return _lib


def _dev(torch, a, dtype):
    arr = np.asfortranarray(a)
    t = torch.from_numpy(np.ascontiguousarray(arr.ravel(order="F"))).to(dtype)
    return t.cuda()


def zpseudo(system, tpsi_ref, zekr):
    """Nonlocal term H_nl psi (only) from the reference's zpseudo_cuda.

    ``tpsi_ref``: complex128 Fortran array (x,y,z,spin,io,ik);
    ``zekr``: complex128 (nps, nlma, nk_z).  Returns the same shape as tpsi_ref.
    """
    import torch
    g, pp = system.grid, system.pp
    t = _dev(torch, tpsi_ref, torch.complex128)
    h = torch.zeros_like(t)
    ia = _dev(torch, pp.ia_tbl.astype(np.int32), torch.int32)
    mps = _dev(torch, pp.mps.astype(np.int32), torch.int32)
    jxyz = _dev(torch, pp.jxyz.astype(np.int32), torch.int32)
    zk = _dev(torch, zekr, torch.complex128)
    rinv = _dev(torch, pp.rinv_uvu, torch.float64)
    natom = pp.natom
    n = pp.nlma // natom
    lib().zpseudo_cuda(h.data_ptr(), n, 1, 1, 1, system.nk, 1, system.no, system.nspin, pp.nlma, pp.nps, natom,
                       int(g.is_array[0]), int(g.ie_array[0]), int(g.is_array[1]), int(g.ie_array[1]),
                       int(g.is_array[2]), int(g.ie_array[2]), ia.data_ptr(), mps.data_ptr(), jxyz.data_ptr(),
                       zk.data_ptr(), rinv.data_ptr(), t.data_ptr())
    torch.cuda.synchronize()
    out = h.cpu().numpy()
    return np.reshape(out, tpsi_ref.shape, order="F")


def stencil_current(system, psi_ref, vec_Ac, ispin=1):
    """(jx, jy, jz) accumulated by stencil_current_core_gpu: the local part
    sum_{k,o} (kAc*rtmp + BT*2Im(...)) * rocc * wtk, before the 1/ngrid."""
    import torch
    g = system.grid
    assert g.periodic and int(np.prod(g.shape)) % 128 == 0
    psi = _dev(torch, psi_ref, torch.complex128)
    vec_k = np.asfortranarray(system.vec_k, dtype=np.float64)
    vac = np.ascontiguousarray(vec_Ac, dtype=np.float64)
    i3 = lambda v: np.ascontiguousarray(np.asarray(v, dtype=np.int32))
    isa, iea, is_, ie = i3(g.is_array), i3(g.ie_array), i3(g.is_), i3(g.ie)
    # the reference passes mg%idx(1:), i.e. the map starting at index 1
    idx = [np.ascontiguousarray(m[4:], dtype=np.int32) for m in (g.idx, g.idy, g.idz)]
    nab = np.ascontiguousarray(np.asarray(g.coef_nab).ravel(order="F"))
    BT = np.ascontiguousarray(np.eye(3).ravel(order="F"))
    rocc = np.asfortranarray(system.rocc[:, :, ispin - 1], dtype=np.float64)
    wtk = np.ascontiguousarray(system.wtk, dtype=np.float64)
    j = np.zeros(3)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    jx, jy, jz = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0)
    lib().stencil_current_core_gpu(1, system.nk, 1, system.no, P(vec_k), P(vac), P(isa), P(iea), P(is_), P(ie),
                                   P(idx[0]), P(idx[1]), P(idx[2]), P(nab), ispin, 1, system.nspin,
                                   psi.data_ptr(), P(BT), P(rocc), P(wtk), C.addressof(jx), C.addressof(jy),
                                   C.addressof(jz))
    torch.cuda.synchronize()
    j[:] = (jx.value, jy.value, jz.value)
    return j


def time_zpseudo(system, tpsi_ref, zekr, reps=5):
    """Milliseconds per call of the reference's zpseudo_cuda on device-resident
    inputs (median of `reps` calls after one warm-up; each call ends with the
    reference's own cudaDeviceSynchronize)."""
    import torch
    g, pp = system.grid, system.pp
    t = _dev(torch, tpsi_ref, torch.complex128)
    h = torch.zeros_like(t)
    ia = _dev(torch, pp.ia_tbl.astype(np.int32), torch.int32)
    mps = _dev(torch, pp.mps.astype(np.int32), torch.int32)
    jxyz = _dev(torch, pp.jxyz.astype(np.int32), torch.int32)
    zk = _dev(torch, zekr, torch.complex128)
    rinv = _dev(torch, pp.rinv_uvu, torch.float64)
    n = pp.nlma // pp.natom
    args = (h.data_ptr(), n, 1, 1, 1, system.nk, 1, system.no, system.nspin, pp.nlma, pp.nps, pp.natom,
            int(g.is_array[0]), int(g.ie_array[0]), int(g.is_array[1]), int(g.ie_array[1]),
            int(g.is_array[2]), int(g.ie_array[2]), ia.data_ptr(), mps.data_ptr(), jxyz.data_ptr(),
            zk.data_ptr(), rinv.data_ptr(), t.data_ptr())
    lib().zpseudo_cuda(*args)
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        lib().zpseudo_cuda(*args)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return float(np.median(times))


def time_stencil_current(system, psi_ref, vec_Ac, reps=2):
    """Milliseconds per call of the reference's stencil_current_core_gpu over
    every orbital of spin 1 (one launch and one device-to-host copy per (k,
    orbital), as the reference issues it)."""
    import time
    import torch
    g = system.grid
    assert g.periodic and int(np.prod(g.shape)) % 128 == 0
    psi = _dev(torch, psi_ref, torch.complex128)
    vec_k = np.asfortranarray(system.vec_k, dtype=np.float64)
    vac = np.ascontiguousarray(vec_Ac, dtype=np.float64)
    i3 = lambda v: np.ascontiguousarray(np.asarray(v, dtype=np.int32))
    isa, iea, is_, ie = i3(g.is_array), i3(g.ie_array), i3(g.is_), i3(g.ie)
    idx = [np.ascontiguousarray(m[4:], dtype=np.int32) for m in (g.idx, g.idy, g.idz)]
    nab = np.ascontiguousarray(np.asarray(g.coef_nab).ravel(order="F"))
    BT = np.ascontiguousarray(np.eye(3).ravel(order="F"))
    rocc = np.asfortranarray(system.rocc[:, :, 0], dtype=np.float64)
    wtk = np.ascontiguousarray(system.wtk, dtype=np.float64)
    P = lambda a: a.ctypes.data_as(C.c_void_p)

    def call():
        jx, jy, jz = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0)
        lib().stencil_current_core_gpu(1, system.nk, 1, system.no, P(vec_k), P(vac), P(isa), P(iea), P(is_), P(ie),
                                       P(idx[0]), P(idx[1]), P(idx[2]), P(nab), 1, 1, system.nspin,
                                       psi.data_ptr(), P(BT), P(rocc), P(wtk), C.addressof(jx), C.addressof(jy),
                                       C.addressof(jz))
        torch.cuda.synchronize()

    call()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        call()
        times.append((time.perf_counter() - t0) * 1e3)
    return float(np.median(times))


# ---- the reference's hand-vectorised AVX-512 stencil (CPU) -------------------

_avx = None


def cpu_has_avx512() -> bool:
    try:
        return any(" avx512f" in line for line in open("/proc/cpuinfo") if line.startswith("flags"))
    except OSError:
        return False


def avx512_available() -> bool:
    return os.path.exists(REF_AVX512_LIB) and cpu_has_avx512()


def _avx_lib():
    global _avx
    if _avx is None:
        L = C.CDLL(REF_AVX512_LIB)
        L.zstencil_tuned_seq_.restype = None
        L.zstencil_tuned_seq_.argtypes = [C.c_void_p] * 15
        _avx = L
    return _avx


def _aligned(shape, dtype, order="C"):
    """Zeroed array whose data starts on a 64-byte boundary (the reference
    kernel uses aligned vector loads and streaming stores)."""
    n = int(np.prod(shape)) * np.dtype(dtype).itemsize
    raw = np.zeros(n + 64, dtype=np.uint8)
    off = (-raw.ctypes.data) % 64
    return raw[off:off + n].view(dtype).reshape(shape, order=order)


def zstencil_avx512(system, psi_ref, vec_Ac):
    """Local H psi (25-point stencil, k+A gradient, V_local) of every orbital
    from the reference's zstencil_tuned_seq_ (zstencil_core/avx512/seq.c),
    called as stencil.f90:101 calls it: modulo tables of
    code_optimization.f90:88-104, k_lap0 / k_nabt of hamiltonian.f90:146-155.
    Periodic grids whose x extent is a multiple of 4.  Returns the reference
    array layout (interior points; padding rows zero)."""
    g = system.grid
    assert g.periodic
    nl = [int(v) for v in g.shape]
    assert nl[0] % 4 == 0
    i3 = lambda v: np.ascontiguousarray(np.asarray(v, dtype=np.int32))
    isa, iea, is_, ie = i3(g.is_array), i3(g.ie_array), i3(g.is_), i3(g.ie)
    mods = [np.ascontiguousarray(np.arange(3 * n, dtype=np.int32) % n) for n in nl]
    lapt = np.ascontiguousarray(np.asarray(g.coef_lap, dtype=np.float64).ravel(order="F"))
    nab = np.asarray(g.coef_nab, dtype=np.float64).reshape((4, 3), order="F")
    out = np.zeros_like(psi_ref, order="F")
    P = lambda a: C.c_void_p(a.ctypes.data)
    shp = tuple(psi_ref.shape[:3])
    E = _aligned(shp[::-1], np.complex128)
    F = _aligned(shp[::-1], np.complex128)
    V = _aligned(tuple(nl[::-1]), np.float64)
    for ik in range(system.nk):
        kac = system.vec_k[:, ik] + np.asarray(vec_Ac, dtype=np.float64)
        lap0 = np.array([g.coef_lap0 + 0.5 * float(np.dot(kac, kac))])
        knab = np.ascontiguousarray((nab * kac[None, :]).ravel(order="F"))
        for isp in range(system.nspin):
            V[...] = np.asarray(system.V_local[..., isp]).transpose(2, 1, 0)
            for io in range(system.no):
                E[...] = psi_ref[:, :, :, isp, io, ik].transpose(2, 1, 0)
                F[...] = 0.0
                _avx_lib().zstencil_tuned_seq_(P(isa), P(iea), P(is_), P(ie), P(mods[0]), P(mods[1]), P(mods[2]),
                                               P(is_), P(ie), P(E), P(F), P(V), P(lap0), P(lapt), P(knab))
                out[:, :, :, isp, io, ik] = F.transpose(2, 1, 0)
    return out
