"""Batched propagation of independent isolated systems (sb200_batch_*).

Every system of a batch must reproduce its own sb200_rt_propagate exactly
(same device functions and summation order, whatever the tile shape and z
chunk), and the oracle's time loop within the FP64 tolerances.
"""
import functools

import numpy as np
import pytest

import _systems as S
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_OBS = 1e-10


@functools.lru_cache(maxsize=None)
def _systems():
    from salmon2_b200 import synth
    return [
        synth.isolated_system(num=24, no=3, natom=2, seed=31, name="b24"),
        synth.isolated_system(num=(36, 20, 28), no=5, natom=3, seed=32, name="b36x20x28"),
        synth.isolated_system(num=(16, 22, 17), no=2, natom=2, seed=33, name="b16x22x17"),
        S.no_pp(synth.isolated_system(num=(19, 18, 20), no=4, natom=1, seed=34, name="b19_nopp")),
    ]


def _setup(precision="fp64"):
    from salmon2_b200 import synth
    from salmon2_b200.rt import Batch, Context
    systems = _systems()
    ctxs = [Context(s, device=0, precision=precision) for s in systems]
    psi0 = [synth.impulse_kick(s.grid, s.psi, 1e-3) for s in systems]
    return systems, ctxs, psi0, Batch(ctxs)


def _run_batch(ctxs, batch, psi0, nt, dt, zc):
    a = [c.upload(p) for c, p in zip(ctxs, psi0)]
    b = [c.zeros() for c in ctxs]
    w = [c.zeros() for c in ctxs]
    res = batch.propagate(a, b, w, nt, dt, zc)
    return [c.download(p) for c, p in zip(ctxs, res["psi"])], res["rbox"]


def _run_solo(ctxs, psi0, nt, dt, zc):
    psis, boxes = [], []
    for c, p in zip(ctxs, psi0):
        a, b, w = c.upload(p), c.zeros(), c.zeros()
        r = c.rt_propagate(a, b, w, nt, dt, zc)
        psis.append(c.download(r["psi"]))
        boxes.append(r["rbox"])
    return psis, boxes


@pytest.mark.parametrize("nt", [6, 5])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_solo(nt, precision):
    from salmon2_b200 import synth
    systems, ctxs, psi0, batch = _setup(precision)
    dt = 0.05
    zc = synth.taylor_zc(dt)
    pb, rb = _run_batch(ctxs, batch, psi0, nt, dt, zc)
    ps, rs = _run_solo(ctxs, psi0, nt, dt, zc)
    for i in range(len(systems)):
        assert np.array_equal(pb[i], ps[i]), systems[i].name
        assert np.array_equal(rb[i], rs[i]), systems[i].name
    batch.close()


def test_batch_tiles_do_not_change_results():
    from salmon2_b200 import synth
    systems, ctxs, psi0, batch = _setup()
    dt = 0.05
    zc = synth.taylor_zc(dt)
    p0, r0 = _run_batch(ctxs, batch, psi0, 4, dt, zc)
    n = len(systems)
    batch.set_tiles([1] * n, [8] * n)  # 16x16 tiles, 8-plane chunks everywhere
    p1, r1 = _run_batch(ctxs, batch, psi0, 4, dt, zc)
    work = [c.zeros() for c in ctxs]
    psi = [c.upload(p) for c, p in zip(ctxs, psi0)]
    sh, zch = batch.autotune(psi, work, reps=2)
    assert all(s in (0, 1) for s in sh)  # the register-sweep family stays in it
    assert all(1 <= z <= s.grid.num[2] for z, s in zip(zch, systems))
    p2, r2 = _run_batch(ctxs, batch, psi0, 4, dt, zc)
    batch.set_tiles([2] * n, [s.grid.num[2] for s in systems])  # tensor-copy sweep, whole z columns
    sh3, zch3 = batch.autotune(psi, work, reps=2)
    assert all(s == 2 for s in sh3)
    p3, r3 = _run_batch(ctxs, batch, psi0, 4, dt, zc)
    for i in range(n):
        for p_, r_ in ((p1, r1), (p2, r2), (p3, r3)):
            assert np.array_equal(p0[i], p_[i]) and np.array_equal(r0[i], r_[i])
    batch.close()


def test_batch_matches_oracle():
    from salmon2_b200 import synth
    systems, ctxs, psi0, batch = _setup()
    nt, dt = 8, 0.05
    zc = synth.taylor_zc(dt)
    pb, rb = _run_batch(ctxs, batch, psi0, nt, dt, zc)
    for i, s in enumerate(systems):
        ref = Oracle(s).rt_run(psi0[i], nt, dt, zc)
        assert S.rel_err(pb[i], ref["psi"]) < 1e-11, s.name
        d_ref = ref["rbox"][:3] - ref["rbox"][:3, :1]
        d_got = rb[i][:3] - rb[i][:3, :1]
        assert np.max(np.abs(d_got - d_ref)) <= TOL_OBS * np.max(np.abs(ref["rbox"][:3])), s.name
        assert np.max(np.abs(rb[i][3] - ref["rbox"][3])) <= 1e-12 * ref["rbox"][3, 0], s.name
    batch.close()


def test_batch_errors():
    from salmon2_b200 import synth
    from salmon2_b200.rt import Batch, Context, SB200Error
    systems, ctxs, psi0, batch = _setup()
    n = len(systems)
    with pytest.raises(SB200Error) as e:
        batch.set_tiles([3] * n, [8] * n)
    assert e.value.code == 1
    with pytest.raises(SB200Error) as e:
        batch.set_tiles([2] + [0] * (n - 1), [8] * n)  # tensor copies for all systems or none
    assert e.value.code == 1
    with pytest.raises(SB200Error) as e:
        batch.set_tiles([0] * n, [10 ** 6] * n)
    assert e.value.code == 1
    periodic = Context(S.periodic_small(), device=0)
    with pytest.raises(SB200Error) as e:
        Batch([ctxs[0], periodic])
    assert e.value.code == 3  # SB200_ERR_UNSUPPORTED
    with pytest.raises(SB200Error):
        Batch([ctxs[0], ctxs[0]])
    a = [c.upload(p) for c, p in zip(ctxs, psi0)]
    with pytest.raises(SB200Error) as e:
        batch.propagate(a, a, a, 2, 0.05, synth.taylor_zc(0.05))
    assert e.value.code == 1
    batch.close()
