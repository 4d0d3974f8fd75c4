"""The oracle's stencil against the reference's own hand-vectorised AVX-512
stencil (zstencil_core/avx512/seq.c, built unmodified from the reference tree
into oracle/_ref by `make -C oracle ref`), run live on the CPU: periodic
grids, several k-points, two spins, nonzero vector potentials.  Skipped where
the library is not built or the CPU lacks AVX-512."""
import numpy as np
import pytest

import _systems as S
import ref_witness
from oracle import Oracle

pytestmark = pytest.mark.skipif(not ref_witness.avx512_available(),
                                reason="reference AVX-512 stencil not built or no AVX-512 CPU")


@pytest.mark.parametrize("num,nkgrid,nspin", [(12, 2, 1), (12, 1, 2), (16, 1, 1), (20, 1, 1)])
def test_oracle_local_hpsi_equals_reference_avx512_stencil(num, nkgrid, nspin):
    from salmon2_b200 import synth
    s = S.no_pp(synth.periodic_system(a=10.26, num=num, nkgrid=nkgrid, no=2, seed=80 + num, nspin=nspin,
                                      name=f"avx{num}"))
    O = Oracle(s)
    sl = s.grid.interior_slices()
    for ac in ((0.0, 0.0, 0.0), (0.02, -0.01, 0.03)):
        O.set_vec_Ac(ac)
        ref = ref_witness.zstencil_avx512(s, s.psi, ac)[sl]
        got = O.hpsi(s.psi)[sl]
        assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
