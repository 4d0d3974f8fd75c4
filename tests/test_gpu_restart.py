"""Restart data in the reference's file layouts (sb200_write_restart /
sb200_read_restart; write_bin / read_bin, write_wavefunction /
read_wavefunction, write_Vh_stock, write_rtdata / read_rtdata of
checkpoint_restart.f90) and the continuation of the time loop
(sb200_rt_set_start / sb200_rt_get_state; restart_rt's Mit):

* files the library writes, parsed here as the reference's records and streams;
* ground-state data written here in the reference's layout (real orbitals,
  more orbitals than the context takes) read into a propagation context;
* the 'slice' layout round trip;
* the reference's checkpoint test (a run restarted from its step-12
  checkpoint repeats the uninterrupted run's later steps): bit for bit for
  the fixed-potential loop in 'tr' and 'lo' (J(t), A(t), orbitals), and for
  the isolated self-consistent CG loop to the CG threshold (the restart solves
  the Hartree potential again from the extrapolated one, as
  initialization_rt.f90:268-283 does).
"""
import os
import struct

import numpy as np
import pytest

import _systems as S

pytestmark = pytest.mark.gpu


def _records(path):
    """the records of a Fortran sequential unformatted file (4-byte markers)"""
    out = []
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        n = struct.unpack("<i", data[i:i + 4])[0]
        out.append(data[i + 4:i + 4 + n])
        assert struct.unpack("<i", data[i + 4 + n:i + 8 + n])[0] == n
        i += 8 + n
    return out


def _put_records(path, recs):
    with open(path, "wb") as f:
        for r in recs:
            f.write(struct.pack("<i", len(r)) + r + struct.pack("<i", len(r)))


def _interior(s):
    """psi (nx, ny, nz, nspin, no, nk) of the interior points"""
    return s.psi[s.grid.interior_slices()]


def test_written_files_follow_the_reference_layout(tmp_path):
    from salmon2_b200.rt import Context
    s = S.periodic_small(nspin=2)
    ctx = Context(s)
    d = tmp_path / "ckpt"
    ctx.write_restart(d, ctx.upload(s.psi), iter=37)
    info = _records(d / "info.bin")
    assert [struct.unpack("<i", r)[0] for r in info] == [s.nk, s.no, 37, 1, 0]
    occ = np.frombuffer(_records(d / "occupation.bin")[0], dtype="<f8")
    assert np.array_equal(occ, np.asarray(s.rocc, order="F").ravel(order="F"))
    wfn = np.fromfile(d / "wfn.bin", dtype="<c16")
    g = s.grid
    n = int(np.prod(g.shape))
    want = _interior(s)
    k = 0
    for ik in range(s.nk):
        for io in range(s.no):
            for isp in range(s.nspin):
                assert np.array_equal(wfn[k * n:(k + 1) * n], want[..., isp, io, ik].ravel(order="F"))
                k += 1
    assert k * n == wfn.size
    assert not os.path.exists(d / "rtdata.bin") and not os.path.exists(d / "Vh_stock.bin")
    ctx.close()


def test_ground_state_data_in_the_reference_layout_start_a_propagation(tmp_path):
    """read_bin of GS data (if_real_orbital = .true., mo = 5 orbitals on file,
    the context takes 3): orbitals widened to complex, the first three
    occupations taken, Mit = 0 without yn_restart."""
    from salmon2_b200.rt import Context
    s = S.isolated_small()
    g = s.grid
    n = int(np.prod(g.shape))
    mo = 5
    rng = np.random.default_rng(31)
    orbs = rng.standard_normal((mo, n))
    occ = np.array([2.0, 2.0, 1.5, 0.5, 0.0])
    d = tmp_path / "gs"
    d.mkdir()
    _put_records(d / "info.bin", [struct.pack("<i", v) for v in (1, mo, 17, 4, 1)])
    _put_records(d / "occupation.bin", [occ.astype("<f8").tobytes()])
    orbs.astype("<f8").tofile(d / "wfn.bin")
    ctx = Context(s)
    psi = ctx.zeros()
    it, rocc = ctx.read_restart(d, psi, yn_restart=False)
    assert it == 0
    assert np.array_equal(rocc[:, 0, 0], occ[: s.no])
    got = ctx.download(psi)[g.interior_slices()]
    for io in range(s.no):
        assert np.array_equal(got[..., 0, io, 0].ravel(order="F"), orbs[io].astype(np.complex128))
    ctx.close()


def test_slice_layout_round_trip(tmp_path):
    from salmon2_b200.rt import Context
    s = S.periodic_small(nspin=2)
    ctx = Context(s)
    d = tmp_path / "sl"
    ctx.write_restart(d, ctx.upload(s.psi), iter=5, method="slice", nblock=3)
    assert os.path.exists(d / "k_000002_ob_000004" / "wfn_ob_000004.dat")
    one = np.fromfile(d / "k_000001_ob_000001" / "wfn_ob_000002.dat", dtype="<c16")
    assert np.array_equal(one[: int(np.prod(s.grid.shape))], _interior(s)[..., 0, 1, 0].ravel(order="F"))
    psi = ctx.zeros()
    it, _ = ctx.read_restart(d, psi, method="slice", nblock=3)
    assert it == 5
    assert np.array_equal(ctx.download(psi), ctx.download(ctx.upload(s.psi)))
    ctx.close()


def _pulse(nt, dt):
    from salmon2_b200 import synth
    return synth.asin2cos(nt, dt, omega=0.05696, f0=0.05696 * 2e-2, tw=nt * dt)


@pytest.mark.parametrize("trans", ["tr", "lo"])
@pytest.mark.parametrize("via_files", [True, False], ids=["files", "set_start"])
def test_restart_repeats_the_uninterrupted_run(tmp_path, trans, via_files):
    """The reference's checkpoint test: steps 13..24 of a run restarted at its
    step-12 checkpoint equal those of the run that went on (bit for bit)."""
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    s = S.periodic_small()
    nt, nc, dt = 24, 12, 0.02
    Ac = _pulse(nt, dt)
    zc = synth.taylor_zc(dt)
    A = Context(s)
    full = A.rt_propagate(A.upload(s.psi), A.zeros(), A.zeros(), nt, dt, zc, Ac_ext=Ac, trans_longi=trans)
    B = Context(s)
    first = B.rt_propagate(B.upload(s.psi), B.zeros(), B.zeros(), nc, dt, zc, Ac_ext=Ac[:, : nc + 2],
                           trans_longi=trans)
    if via_files:
        B.write_restart(tmp_path / "ck", first["psi"], iter=nc, trans_longi=trans)
        assert os.path.exists(tmp_path / "ck" / "rtdata.bin") == (trans == "lo")
        C = Context(s)
        psi = C.zeros()
        it, _ = C.read_restart(tmp_path / "ck", psi, yn_restart=True)
        assert it == nc
    else:
        mit, tot, ind = B.rt_get_state()
        assert mit == nc
        C = B
        psi = first["psi"]
        C.rt_set_start(mit, tot, ind)
    b, w = (C.zeros(), C.zeros())
    rest = C.rt_propagate(psi, b, w, nt - nc, dt, zc, Ac_ext=Ac[:, nc:], trans_longi=trans)
    assert np.array_equal(rest["curr"], full["curr"][:, nc:])
    assert np.array_equal(rest["Ac_tot"][:, 1:], full["Ac_tot"][:, nc + 1:])
    assert np.array_equal(C.download(rest["psi"]), A.download(full["psi"]))
    assert C.rt_get_state()[0] == nt
    for x in {id(A): A, id(B): B, id(C): C}.values():
        x.close()


def test_restart_of_the_isolated_self_consistent_cg_loop(tmp_path):
    """Isolated molecule, Hartree by CG every step: the checkpoint carries
    Vh_stock1 / Vh_stock2; the restarted run's dipole follows the
    uninterrupted one to the CG threshold."""
    import dataclasses as dc
    import oracle as OR
    from salmon2_b200 import synth
    from salmon2_b200.rt import Context
    from test_gpu_scf import _brl, _oracle
    s0 = S.isolated_small()
    s = dc.replace(s0, psi=synth.impulse_kick(s0.grid, s0.psi, 1e-3))
    nt, nc, dt = 12, 6, 0.05
    zc = synth.taylor_zc(dt)
    vpsl = np.array(s.V_local[..., 0])
    O = _oracle(s)
    rho0 = O.density(s.psi)[..., 0]
    vh0, _ = O.poisson_isolated_cg(rho0)
    vxc0 = OR.exc_cor_pz(rho0, s.grid.hvol)[0]

    def fresh():
        ctx = Context(s)
        ctx.update_vlocal(vpsl, vh0, vxc0)
        ctx.set_hartree_cg(vh0)
        ctx.set_self_consistent(True, vpsl, _brl(s))
        return ctx

    A = fresh()
    full = A.rt_propagate(A.upload(s.psi), A.zeros(), A.zeros(), nt, dt, zc)
    B = fresh()
    first = B.rt_propagate(B.upload(s.psi), B.zeros(), B.zeros(), nc, dt, zc)
    B.write_restart(tmp_path / "ck", first["psi"], iter=nc)
    assert os.path.exists(tmp_path / "ck" / "Vh_stock.bin")
    assert np.array_equal(first["rbox"], full["rbox"][:, :nc])
    C = fresh()
    psi = C.zeros()
    it, _ = C.read_restart(tmp_path / "ck", psi, yn_restart=True)
    assert it == nc
    rest = C.rt_propagate(psi, C.zeros(), C.zeros(), nt - nc, dt, zc)
    ref = full["rbox"][:3, nc:] - full["rbox"][:3, :1]
    got = rest["rbox"][:3] - full["rbox"][:3, :1]
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    print(f"restarted CG loop: dipole response relative difference {err:.2e}")
    assert err < 1e-7
    for x in (A, B, C):
        x.close()
