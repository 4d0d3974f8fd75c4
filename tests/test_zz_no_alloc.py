"""sb200_hpsi_noalloc: H psi for callers that cannot allocate device memory.

Hosts whose device arrays are owned by another runtime (an OpenACC or
OpenMP-offload Fortran program), memory-capped environments, or time loops
that must not allocate cannot call cudaMalloc or create a library context.
This entry point takes only caller-owned device arrays and keeps its scratch
(the KB projections) in a fixed array inside the library.  The test calls it
through the C ABI twice in a row and checks both results against sb200_hpsi
on the same inputs, within the 1e-12 relative tolerance of the other H psi
parity tests.  The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu

TOL_H = 1e-12


def _dev(torch, a, dtype):
    flat = np.ascontiguousarray(np.asarray(a).ravel(order="F"))
    return torch.from_numpy(flat).to(dtype).cuda()


def _noalloc_hpsi(system, psi_dev, ac):
    import torch
    from salmon2_b200 import _lib

    g, pp = system.grid, system.pp
    kac = np.asfortranarray(system.vec_k + np.asarray(ac, dtype=np.float64)[:, None])
    dev = dict(
        V=_dev(torch, system.V_local, torch.float64),
        kac=_dev(torch, kac, torch.float64),
        mps=_dev(torch, pp.mps.astype(np.int32), torch.int32),
        jxyz=_dev(torch, pp.jxyz.astype(np.int32), torch.int32),
        rxyz=_dev(torch, pp.rxyz, torch.float64),
        uv=_dev(torch, pp.uv, torch.float64),
        ia=_dev(torch, pp.ia_tbl.astype(np.int32), torch.int32),
        rinv=_dev(torch, pp.rinv_uvu, torch.float64),
    )
    out = torch.zeros_like(psi_dev)
    lap = np.ascontiguousarray(np.asarray(g.coef_lap).ravel(order="F"))
    nab = np.ascontiguousarray(np.asarray(g.coef_nab).ravel(order="F"))
    is3 = (C.c_int * 3)(*[int(v) for v in g.is_])
    P = lambda t: C.c_void_p(t.data_ptr())
    dp = C.POINTER(C.c_double)
    nx, ny, nz = g.shape
    rc = _lib.lib().sb200_hpsi_noalloc(
        nx, ny, nz, 1 if g.periodic else 0, system.nspin, system.no, system.nk, is3, g.coef_lap0,
        lap.ctypes.data_as(dp), nab.ctypes.data_as(dp), P(dev["kac"]), P(dev["V"]), pp.natom, pp.nps, pp.nlma,
        P(dev["mps"]), P(dev["jxyz"]), P(dev["rxyz"]), P(dev["uv"]), P(dev["ia"]), P(dev["rinv"]), P(psi_dev),
        P(out), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("make", [S.periodic_small, S.isolated_small], ids=lambda f: f.__name__)
def test_noalloc_matches_hpsi_twice(make):
    from salmon2_b200.rt import Context

    s = make()
    ctx = Context(s)
    ac = (0.013, -0.021, 0.034) if s.grid.periodic else (0.0, 0.0, 0.0)
    ctx.set_vec_Ac(ac)
    psi = ctx.upload(s.psi)
    ref = ctx.zeros()
    ctx.hpsi(psi, ref)
    ctx.sync()
    ref_np = ref.cpu().numpy()
    scale = np.max(np.abs(ref_np))
    for _ in range(2):  # the scratch keeps the previous call's contents
        got = _noalloc_hpsi(s, psi, ac).cpu().numpy()
        assert np.max(np.abs(got - ref_np)) <= TOL_H * scale
    ctx.close()


def test_noalloc_rejects_oversized_projection_scratch():
    import torch
    from salmon2_b200 import _lib

    s = S.periodic_small()
    g = s.grid
    tiny = torch.zeros(16, dtype=torch.float64, device="cuda")
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    ti = torch.zeros(16, dtype=torch.int32, device="cuda")
    is3 = (C.c_int * 3)(1, 1, 1)
    arr = (C.c_double * 12)()
    P = lambda t: C.c_void_p(t.data_ptr())
    # 2 * 1024 * 1 orbitals x 256 projectors > 262144: refused before any launch
    rc = _lib.lib().sb200_hpsi_noalloc(g.shape[0], g.shape[1], g.shape[2], 1, 2, 1024, 1, is3, 0.0, arr, arr,
                                       P(tiny), P(tiny), 64, 100, 256, P(ti), P(ti), P(tiny), P(tiny), P(ti),
                                       P(tiny), P(tiny), P(out), None)
    assert rc == 2  # SB200_ERR_BAD_SHAPE
    assert b"SB200_NOALLOC_MAX_PROJECTIONS" in _lib.lib().sb200_last_error()
