"""The k-point sharding of the multi-GPU path, run as two gloo ranks on the
CPU with the oracle as the per-rank propagator: the all-reduced current of
the shards equals the current of one run over the merged, denser k-mesh."""
import dataclasses
import os

import numpy as np
import pytest

NT, DT = 3, 0.08


def _system():
    from salmon2_b200 import synth
    return synth.periodic_system(a=10.26, num=12, nkgrid=1, no=2, seed=41, name="shard12")


def _field():
    from salmon2_b200 import synth
    return synth.asin2cos(NT, DT, omega=0.05696, f0=0.05696 * 2e-2, tw=NT * DT), synth.taylor_zc(DT)


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import Oracle
    from salmon2_b200 import synth
    s = synth.kpoint_shard(_system(), rank, world, 10.26, 1)
    Ac, zc = _field()
    cur = Oracle(s, threads=1).rt_run(s.psi, NT, DT, zc, Ac_ext=Ac)["curr"]
    t = torch.from_numpy(np.ascontiguousarray(cur))
    dist.all_reduce(t)
    if rank == 0:
        np.save(out, t.numpy())
    dist.destroy_process_group()


def test_two_rank_current_equals_merged_kmesh(tmp_path):
    import socket

    import torch.multiprocessing as mp
    from oracle import Oracle
    from salmon2_b200 import synth
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "j.npy")
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    j_ranks = np.load(out)
    # one process over the merged mesh: both shards' k-points, orbitals and weights
    base = _system()
    sh = [synth.kpoint_shard(base, r, 2, 10.26, 1) for r in range(2)]
    merged = dataclasses.replace(
        base, nk=2, vec_k=np.asfortranarray(np.concatenate([x.vec_k for x in sh], axis=1)),
        wtk=np.concatenate([x.wtk for x in sh]),
        rocc=np.asfortranarray(np.concatenate([x.rocc for x in sh], axis=1)),
        psi=np.asfortranarray(np.concatenate([x.psi for x in sh], axis=5)))
    assert abs(np.sum(merged.wtk) - 1.0) < 1e-15
    Ac, zc = _field()
    j_merged = Oracle(merged, threads=1).rt_run(merged.psi, NT, DT, zc, Ac_ext=Ac)["curr"]
    assert np.max(np.abs(j_ranks - j_merged)) <= 1e-12 * np.max(np.abs(j_merged))


def _scf_rank_main(rank, world, port, out):
    """One k-point shard of the self-consistent loop: per step the Taylor step
    of the shard's orbitals, the shard densities summed over the ranks (the
    all-reduce the library issues with sb200_set_density_comm), then the
    Hartree, PZ-LDA and V_local of the summed density."""
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle as OR
    from oracle import Oracle
    from salmon2_b200 import synth
    s = synth.kpoint_shard(_system(), rank, world, 10.26, 1)
    s = dataclasses.replace(s, V_local=np.array(s.V_local, order="F"))
    O = Oracle(s, threads=1)
    _, zc = _field()
    g = s.grid
    brl = OR.primitive_b_orthogonal([n * h for n, h in zip(g.shape, g.hgs)])
    vpsl = np.array(s.V_local[..., 0])

    def summed_density(psi):
        t = torch.from_numpy(np.ascontiguousarray(O.density(psi)[..., 0]))
        dist.all_reduce(t)
        return t.numpy()

    def set_potential(rho):
        vxc, _ = OR.exc_cor_pz(rho, g.hvol)
        O.V[...] = OR.update_vlocal(vpsl, OR.poisson_ft(rho, brl), vxc[..., None])

    psi = s.psi
    set_potential(summed_density(psi))
    for _ in range(NT):
        psi = O.taylor(psi, zc)
        rho = summed_density(psi)
        set_potential(rho)
    if rank == 0:
        np.save(out, rho)
    dist.destroy_process_group()


def test_two_rank_self_consistent_density_equals_merged_kmesh(tmp_path):
    """The self-consistent loop over two k-point shards, each with the
    all-reduced density, equals one loop over the merged k-mesh (the oracle's
    sbo_rt_run_scf): the density after the last step."""
    import socket

    import torch.multiprocessing as mp
    import oracle as OR
    from oracle import Oracle
    from salmon2_b200 import synth
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "rho.npy")
    mp.start_processes(_scf_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    rho_ranks = np.load(out)
    base = _system()
    sh = [synth.kpoint_shard(base, r, 2, 10.26, 1) for r in range(2)]
    merged = dataclasses.replace(
        base, nk=2, vec_k=np.asfortranarray(np.concatenate([x.vec_k for x in sh], axis=1)),
        wtk=np.concatenate([x.wtk for x in sh]),
        rocc=np.asfortranarray(np.concatenate([x.rocc for x in sh], axis=1)),
        psi=np.asfortranarray(np.concatenate([x.psi for x in sh], axis=5)))
    O = Oracle(merged, threads=1)
    g = merged.grid
    brl = OR.primitive_b_orthogonal([n * h for n, h in zip(g.shape, g.hgs)])
    vpsl = np.array(merged.V_local[..., 0])
    rho0 = O.density(merged.psi)[..., 0]
    v0 = OR.update_vlocal(vpsl, OR.poisson_ft(rho0, brl), OR.exc_cor_pz(rho0, g.hvol)[0][..., None])[..., 0]
    _, zc = _field()
    ref = O.rt_run_scf(merged.psi, NT, DT, zc, vpsl, brl, v0)
    assert np.max(np.abs(rho_ranks - ref["rho"][..., 0])) <= 1e-12 * np.max(np.abs(ref["rho"]))


def _lo_rank_main(rank, world, port, out):
    """One k-point shard of the induced-field ('lo') loop: per step the Taylor
    step at the midpoint A, the shard's current at A(t), the currents summed
    over the ranks (the all-reduce the library issues inside its loop when a
    shard communicator is set), then calc_emfields with the summed current
    (em_field.f90:24-70): the order of the oracle's own loop."""
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import Oracle
    s = _shard_lo(rank, world)
    O = Oracle(s, threads=1)
    Ac_ext, zc = _field()
    Ac_ind = np.zeros_like(Ac_ext)
    Ac_tot = Ac_ext.copy()
    curr = np.zeros((3, NT))
    psi = s.psi
    for itt in range(1, NT + 1):
        O.set_vec_Ac(0.5 * (Ac_tot[:, itt] + Ac_tot[:, itt - 1]))
        psi = O.taylor(psi, zc)
        O.set_vec_Ac_local_only(Ac_tot[:, itt])
        j = torch.from_numpy(np.ascontiguousarray(O.current(psi).sum(axis=1)))
        dist.all_reduce(j)
        j = j.numpy()
        curr[:, itt - 1] = j
        Ac_ind[:, itt + 1] = 2.0 * Ac_ind[:, itt] - Ac_ind[:, itt - 1] - 4.0 * np.pi * j * DT * DT
        Ac_tot[:, itt + 1] = Ac_ext[:, itt + 1] + Ac_ind[:, itt + 1]
    if rank == 0:
        np.save(out, np.concatenate([curr.ravel(), Ac_tot.ravel()]))
    dist.destroy_process_group()


def _shard_lo(rank, world):
    from salmon2_b200 import synth
    return synth.kpoint_shard(_system(), rank, world, 10.26, 1)


def test_two_rank_induced_field_equals_merged_kmesh(tmp_path):
    """'lo' mode over two k-point shards with the current summed every step
    before the induced field is updated: J(t) and A_tot equal one loop over the
    merged k-mesh (the oracle's sbo_rt_run with trans_longi = 'lo').  Without
    the per-step sum each shard's A_ind would follow its own partial current."""
    import socket

    import torch.multiprocessing as mp
    from oracle import Oracle
    from salmon2_b200 import synth
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    out = str(tmp_path / "lo.npy")
    mp.start_processes(_lo_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    base = _system()
    sh = [synth.kpoint_shard(base, r, 2, 10.26, 1) for r in range(2)]
    merged = dataclasses.replace(
        base, nk=2, vec_k=np.asfortranarray(np.concatenate([x.vec_k for x in sh], axis=1)),
        wtk=np.concatenate([x.wtk for x in sh]),
        rocc=np.asfortranarray(np.concatenate([x.rocc for x in sh], axis=1)),
        psi=np.asfortranarray(np.concatenate([x.psi for x in sh], axis=5)))
    Ac, zc = _field()
    ref = Oracle(merged, threads=1).rt_run(merged.psi, NT, DT, zc, Ac_ext=Ac, trans_longi=1)
    j_ref = ref["curr"]
    j_got = got[: 3 * NT].reshape(3, NT)
    a_got = got[3 * NT:].reshape(Ac.shape)
    assert np.max(np.abs(j_got - j_ref)) <= 1e-12 * np.max(np.abs(j_ref))
    assert np.max(np.abs(a_got - ref["Ac_tot"])) <= 1e-12 * np.max(np.abs(ref["Ac_tot"]))
