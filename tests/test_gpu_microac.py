"""The single-scale (microscopic vector potential) hpsi on the GPU
(sb200_set_micro_ac; the reference's zstencil_microAc_typical_seq with
per-point k + A(r) and the -i div A / 2 term; with
sb200_set_symmetrized_stencil the zstencil_microAc_symmetrized form) and the
microscopic current (sb200_calc_microscopic_current, calc_microscopic_current)
against the oracle, through the C ABI: H psi with and without the KB term, two
spins, an isolated grid, and the Taylor step.  Tolerance 1e-12 relative, as
for the other H psi forms and the density."""
import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_H = 1e-12


def _field(g, seed):
    rng = np.random.default_rng(seed)
    x = [np.arange(n) * 2 * np.pi / n for n in g.shape]
    X, Y, Z = np.meshgrid(*x, indexing="ij")
    amp = rng.uniform(-0.03, 0.03, (3, 3))
    acm = np.stack([amp[d, 0] * np.cos(X + d) + amp[d, 1] * np.sin(2 * Y) + amp[d, 2] * np.cos(Z - d)
                    for d in range(3)])
    div = rng.uniform(-0.05, 0.05) * np.sin(X) * np.cos(Y)
    return np.asfortranarray(acm), np.asfortranarray(div)


@pytest.mark.parametrize("make", [S.periodic_small, lambda: S.no_pp(S.periodic_small()),
                                  lambda: S.periodic_small(nspin=2)], ids=["pp", "no_pp", "two_spins"])
def test_hpsi_micro_ac_against_oracle(make):
    from salmon2_b200.rt import Context
    s = make()
    acm, div = _field(s.grid, 3)
    O = Oracle(s)
    ctx = Context(s)
    ac = (0.01, -0.02, 0.005)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    O.set_micro_ac(acm, div)
    ctx.set_micro_ac(acm, div)
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(s.psi), h)
    assert S.rel_err(ctx.download(h), O.hpsi(s.psi)) < TOL_H
    ctx.close()


def test_taylor_micro_ac_against_oracle():
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s = S.periodic_small()
    acm, div = _field(s.grid, 4)
    O = Oracle(s)
    ctx = Context(s)
    O.set_micro_ac(acm, div)
    ctx.set_micro_ac(acm, div)
    zc = synth.taylor_zc(0.05)
    out, work = ctx.zeros(), ctx.zeros()
    ctx.taylor(ctx.upload(s.psi), out, work, zc)
    assert S.rel_err(ctx.download(out), O.taylor(s.psi, zc)) < TOL_H
    ctx.set_micro_ac(None, None)  # back to the macroscopic stencil
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(s.psi), h)
    O.set_micro_ac(None, None)
    assert S.rel_err(ctx.download(h), O.hpsi(s.psi)) < TOL_H
    ctx.close()


_SYSTEMS = [S.periodic_small, lambda: S.no_pp(S.periodic_small()), lambda: S.periodic_small(nspin=2),
            S.isolated_small]
_IDS = ["pp", "no_pp", "two_spins", "isolated"]


@pytest.mark.parametrize("make", _SYSTEMS, ids=_IDS)
def test_hpsi_symmetrized_micro_ac_against_oracle(make):
    from salmon2_b200.rt import Context
    s = make()
    acm, _ = _field(s.grid, 5)
    O = Oracle(s)
    ctx = Context(s)
    ac = (0.01, -0.02, 0.005)
    O.set_vec_Ac(ac)
    ctx.set_vec_Ac(ac)
    O.set_micro_ac(acm, None, symmetrized=True)
    ctx.set_micro_ac(acm, None, symmetrized=True)
    h = ctx.zeros()
    ctx.hpsi(ctx.upload(s.psi), h)
    assert S.rel_err(ctx.download(h), O.hpsi(s.psi)) < TOL_H
    ctx.close()


def test_taylor_symmetrized_micro_ac_against_oracle():
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s = S.periodic_small(nspin=2)
    acm, _ = _field(s.grid, 6)
    O = Oracle(s)
    ctx = Context(s)
    O.set_micro_ac(acm, None, symmetrized=True)
    ctx.set_micro_ac(acm, None, symmetrized=True)
    zc = synth.taylor_zc(0.05)
    out, work = ctx.zeros(), ctx.zeros()
    ctx.taylor(ctx.upload(s.psi), out, work, zc)
    assert S.rel_err(ctx.download(out), O.taylor(s.psi, zc)) < TOL_H
    ctx.close()


@pytest.mark.parametrize("make", [S.periodic_small, lambda: S.periodic_small(nspin=2), S.isolated_small,
                                  S.periodic_c2_like], ids=["periodic", "two_spins", "isolated", "c2_like"])
def test_microscopic_current_against_oracle(make):
    from salmon2_b200.rt import Context
    s = make()
    ctx = Context(s)
    cur = ctx.calc_microscopic_current(ctx.upload(s.psi))
    ref = Oracle(s).microscopic_current(s.psi)
    assert np.max(np.abs(ref)) > 0
    assert S.rel_err(cur, ref) < TOL_H
    ctx.close()
