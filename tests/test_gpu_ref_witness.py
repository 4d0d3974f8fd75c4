"""Live three-way check on the GPU: the reference's own CUDA kernels
(oracle/_ref, built from the reference sources), the CPU oracle and this
library, on the same seeded inputs."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden as MG  # noqa: E402
import ref_witness  # noqa: E402
from oracle import Oracle  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_witness.available(), reason="oracle/_ref not built")]


def test_zpseudo_reference_vs_oracle_vs_library():
    from salmon2_b200.rt import Context
    import _systems as S
    per, iso = MG.witness_systems()
    for s in (per, iso):
        O = Oracle(s)
        ac = (0.013, -0.021, 0.034)
        O.set_vec_Ac(ac)
        h_ref = ref_witness.zpseudo(s, s.psi, O.zekr)
        h_orc = O.zpseudo(s.psi)
        assert S.rel_err(h_orc, h_ref) < 1e-12
        # library: H psi - H_local psi = nonlocal term
        ctx = Context(s)
        ctx.set_vec_Ac(ac)
        t = ctx.upload(s.psi)
        h_full = ctx.zeros()
        ctx.hpsi(t, h_full)
        ctx_loc = Context(S.no_pp(s))
        ctx_loc.set_vec_Ac(ac)
        h_loc = ctx_loc.zeros()
        ctx_loc.hpsi(ctx_loc.upload(s.psi), h_loc)
        nl = ctx.download(h_full) - ctx_loc.download(h_loc)
        assert S.rel_err(nl, h_ref) < 1e-11


def test_stencil_current_reference_vs_oracle():
    per, _ = MG.witness_systems()
    O = Oracle(per)
    for ac in MG.A_VALUES:
        O.set_vec_Ac(ac)
        ref = ref_witness.stencil_current(per, per.psi, ac)
        parts = O.current_parts(per.psi)
        local = np.zeros(3)
        for o in range(per.norb):
            ik = o // (per.nspin * per.no)
            io = (o // per.nspin) % per.no
            local += ((per.vec_k[:, ik] + np.asarray(ac)) * parts[0, o] + parts[1:4, o]) * per.rocc[io, ik, 0] * per.wtk[ik]
        assert np.max(np.abs(local - ref)) <= 1e-12 * max(np.max(np.abs(ref)), 1e-300)


def _timed(ctx, fn, reps=5):
    """Milliseconds per call of fn on the context's stream (median)."""
    import torch
    st = torch.cuda.Stream()
    ctx.set_stream(st)
    fn()
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ctx.set_stream(None)
    return float(np.median(times))


@pytest.mark.parametrize("which", ["bulk", "supercell"])
def test_reference_gpu_kernels_timed_beside_library(which):
    """The reference's own GPU kernels for the two sub-steps it ships in CUDA,
    timed on the B200 beside this library on the same inputs (one line per
    workload starting with REFTIME): zpseudo_cuda (the KB nonlocal term alone;
    one thread per (orbital, projector), atomics) against sb200_hpsi (the
    whole H psi: stencil, k+A gradient, V_local and KB), and
    stencil_current_core_gpu (the local current; one launch and one copy back
    per (k, orbital)) against sb200_calc_current (local and nonlocal current).
    Their results are compared with the oracle by the tests above."""
    import json
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    if which == "bulk":
        s = synth.periodic_system(a=10.26, num=16, nkgrid=4, no=32, seed=2, name="periodic_bulk")
    else:
        s = synth.periodic_system(a=10.26, num=16, nkgrid=2, no=256, supercell=2, seed=3, ecut=2.0,
                                  name="periodic_supercell")
    ac = (0.0, 0.0, 1e-3)
    O = Oracle(s)
    O.set_vec_Ac(ac)
    ref_ms = ref_witness.time_zpseudo(s, s.psi, O.zekr)
    ctx = Context(s)
    ctx.set_vec_Ac(ac)
    t = ctx.upload(s.psi)
    h = ctx.zeros()
    lib_ms = _timed(ctx, lambda: ctx.hpsi(t, h))
    out = dict(workload=which, orbitals=s.norb, grid=list(s.grid.shape), projectors=s.pp.nlma,
               ref_zpseudo_cuda_ms=ref_ms, lib_hpsi_ms=lib_ms)
    if which == "bulk":
        out["ref_stencil_current_core_gpu_ms"] = ref_witness.time_stencil_current(s, s.psi, ac)
        out["lib_calc_current_ms"] = _timed(ctx, lambda: ctx.calc_current(t, ac), reps=3)
    print("REFTIME " + json.dumps(out))
    ctx.close()
    assert ref_ms > 0 and lib_ms > 0


@pytest.mark.skipif(not ref_witness.avx512_available(), reason="reference AVX-512 stencil not built or no AVX-512 CPU")
@pytest.mark.parametrize("num,nkgrid,nspin", [(12, 2, 1), (16, 1, 2)])
def test_stencil_reference_avx512_vs_library(num, nkgrid, nspin):
    """The library's local H psi (no projectors; tensor-copy sweep on 12^3, the
    per-term orbital kernel on 16^3) against the reference's own AVX-512 stencil
    on the same inputs: 1e-12 relative."""
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    import _systems as S
    s = S.no_pp(synth.periodic_system(a=10.26, num=num, nkgrid=nkgrid, no=2, seed=90 + num, nspin=nspin,
                                      name=f"avxg{num}"))
    ac = (0.013, -0.021, 0.034)
    ref = ref_witness.zstencil_avx512(s, s.psi, ac)
    ctx = Context(s)
    ctx.set_vec_Ac(ac)
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(s.psi), h)
    sl = s.grid.interior_slices()
    got = ctx.download(h)
    assert np.max(np.abs(got[sl] - ref[sl])) <= 1e-12 * np.max(np.abs(ref[sl]))
    ctx.close()
