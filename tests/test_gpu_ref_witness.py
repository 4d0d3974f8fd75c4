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
