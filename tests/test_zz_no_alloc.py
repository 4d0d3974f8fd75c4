"""sb200_hpsi_noalloc: H psi for callers that cannot allocate device memory.

Hosts whose device arrays are owned by another runtime (an OpenACC or
OpenMP-offload Fortran program), memory-capped environments, or time loops
that must not allocate cannot call cudaMalloc or create a library context.
This entry point takes only caller-owned device arrays and keeps its scratch
(the KB projections) in a fixed array inside the library.  The tests call it
through the C ABI twice in a row and check both results against sb200_hpsi and
against the oracle on the same inputs, within the 1e-12 relative tolerance of
the other H psi parity tests: one and two spins, isolated grids, and a
periodic cell whose projector spheres reach some grid points through two
images.  They also check that a projector table pointing outside the grid is
reported in the status word instead of being read, and that more orbitals than
one launch dimension holds (65,535) are all computed.  The file is named so
that pytest collects it last.
"""
import ctypes as C
import functools

import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_H = 1e-12


@functools.lru_cache(maxsize=None)
def _wrap_cell():
    # spheres (rc = 1.8 A) wider than half the 6-bohr cell: some grid points
    # are reached twice by one projector through two periodic images
    from salmon2_b200 import synth
    return synth.periodic_system(a=6.0, num=12, nkgrid=1, no=2, seed=38, rc_aa=1.8, name="wrap")


def _two_spins():
    return S.periodic_small(nspin=2)


def _dev(torch, a, dtype):
    flat = np.ascontiguousarray(np.asarray(a).ravel(order="F"))
    return torch.from_numpy(flat).to(dtype).cuda()


def _noalloc_hpsi(system, psi_dev, ac, jxyz=None, with_status=True):
    """Calls the entry point on device copies of the system's tables; returns
    (H psi in the resident layout, status word or None)."""
    import torch
    from salmon2_b200 import _lib

    g, pp = system.grid, system.pp
    kac = np.asfortranarray(system.vec_k + np.asarray(ac, dtype=np.float64)[:, None])
    dev = dict(
        V=_dev(torch, system.V_local, torch.float64),
        kac=_dev(torch, kac, torch.float64),
        mps=_dev(torch, pp.mps.astype(np.int32), torch.int32),
        jxyz=_dev(torch, (pp.jxyz if jxyz is None else jxyz).astype(np.int32), torch.int32),
        rxyz=_dev(torch, pp.rxyz, torch.float64),
        uv=_dev(torch, pp.uv, torch.float64),
        ia=_dev(torch, pp.ia_tbl.astype(np.int32), torch.int32),
        rinv=_dev(torch, pp.rinv_uvu, torch.float64),
    )
    out = torch.zeros_like(psi_dev)
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda") if with_status else None
    lap = np.ascontiguousarray(np.asarray(g.coef_lap).ravel(order="F"))
    nab = np.ascontiguousarray(np.asarray(g.coef_nab).ravel(order="F"))
    is3 = (C.c_int * 3)(*[int(v) for v in g.is_])
    P = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    dp = C.POINTER(C.c_double)
    nx, ny, nz = g.shape
    rc = _lib.lib().sb200_hpsi_noalloc(
        nx, ny, nz, 1 if g.periodic else 0, system.nspin, system.no, system.nk, is3, g.coef_lap0,
        lap.ctypes.data_as(dp), nab.ctypes.data_as(dp), P(dev["kac"]), P(dev["V"]), pp.natom, pp.nps, pp.nlma,
        P(dev["mps"]), P(dev["jxyz"]), P(dev["rxyz"]), P(dev["uv"]), P(dev["ia"]), P(dev["rinv"]), P(psi_dev),
        P(out), P(status), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out, (int(status.item()) if status is not None else None)


@pytest.mark.parametrize("make", [S.periodic_small, _two_spins, S.isolated_small, _wrap_cell],
                         ids=["periodic12", "periodic12_two_spins", "isolated24", "wrap_cell"])
def test_noalloc_matches_hpsi_and_oracle_twice(make):
    from salmon2_b200.rt import Context

    s = make()
    ctx = Context(s)
    ac = (0.013, -0.021, 0.034) if s.grid.periodic else (0.0, 0.0, 0.0)
    ctx.set_vec_Ac(ac)
    O = Oracle(s)
    O.set_vec_Ac(ac)
    psi = ctx.upload(s.psi)
    ref = ctx.zeros()
    ctx.hpsi(psi, ref)
    ctx.sync()
    ref_np = ref.cpu().numpy()
    ref_or = O.hpsi(s.psi)
    scale = np.max(np.abs(ref_np))
    for _ in range(2):  # the scratch keeps the previous call's contents
        got, status = _noalloc_hpsi(s, psi, ac)
        assert status == 0
        assert np.max(np.abs(got.cpu().numpy() - ref_np)) <= TOL_H * scale
        assert S.rel_err(ctx.download(got), ref_or) <= TOL_H
    ctx.close()


def test_noalloc_flags_a_table_outside_the_grid():
    """A jxyz entry past the grid's upper bound is skipped and reported; the
    call after it with the right table is clean again."""
    from salmon2_b200.rt import Context

    s = S.periodic_small()
    ctx = Context(s)
    ac = (0.0, 0.0, 0.01)
    psi = ctx.upload(s.psi)
    bad = np.array(s.pp.jxyz, copy=True, order="F")
    bad[0, 0, 0] = s.grid.ie[0] + 3
    got, status = _noalloc_hpsi(s, psi, ac, jxyz=bad)
    assert status == 2  # SB200_ERR_BAD_SHAPE
    assert np.all(np.isfinite(got.cpu().numpy()))
    _, status = _noalloc_hpsi(s, psi, ac)
    assert status == 0
    ctx.close()


def test_noalloc_more_orbitals_than_one_launch_dimension():
    """70,000 orbitals on a small periodic grid without projectors: every
    orbital is computed (orbital o repeats orbital o mod 4 of a small call, so
    the outputs agree bit for bit)."""
    import dataclasses
    import torch
    from salmon2_b200 import synth

    small = S.no_pp(synth.periodic_system(a=6.0, num=8, nkgrid=1, no=4, seed=41, name="tiny8"))
    from salmon2_b200.rt import Context
    ctx = Context(small)
    psi_s = ctx.upload(small.psi)
    ref, status = _noalloc_hpsi(small, psi_s, (0.0, 0.0, 0.0))
    assert status == 0
    assert S.rel_err(ctx.download(ref), Oracle(small).hpsi(small.psi)) <= TOL_H
    nbig = 70000
    big = dataclasses.replace(small, no=nbig)
    psi_b = psi_s.repeat(nbig // 4, 1, 1, 1)  # resident layout (orbital, z, y, x)
    got, status = _noalloc_hpsi(big, psi_b, (0.0, 0.0, 0.0))
    assert status == 0
    reps = got.reshape(nbig // 4, *ref.shape)
    assert torch.equal(reps[-1], ref) and torch.equal(reps[nbig // 8], ref)
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
                                       P(tiny), P(tiny), P(out), None, None)
    assert rc == 2  # SB200_ERR_BAD_SHAPE
    assert b"SB200_NOALLOC_MAX_PROJECTIONS" in _lib.lib().sb200_last_error()
