"""Host-side set-up from the other pseudopotential formats with one projector
per angular momentum (sb200_init_ps, the format chosen by the file name as
init_pp does: `.pspnc` ABINIT, `.fhi` ABINITFHI, `.cpi` FHI98PP) against the
oracle's restatement of read_ps_abinit / read_ps_abinitfhi / read_ps_fhi
(oracle/pseudo_ky.py), and across formats: the same radial data written as
`.fhi` and as `.cpi` give bit-identical tables, and written as ABINIT and as
FHI (on ABINIT's grid, the cut-off radius the FHI reader finds given to the
ABINIT file) the same tables to 1e-13.  On CPU: the builder has no device
code."""
import numpy as np
import pytest

import _systems as S
import pseudo_ky as PK


def _grid(periodic):
    from salmon2_b200 import synth
    if periodic:
        return synth.make_grid([12, 12, 12], 6.0 / 12, periodic=True)
    return synth.make_grid([24, 24, 24], 0.25 / synth.AU_LENGTH_AA, periodic=False)


def _rion(periodic):
    if periodic:
        return np.array([[0.2, 5.9, 3.0], [3.1, 0.1, 5.8]]).T
    return np.array([[0.3, -0.2, 1.1], [-1.4, 0.5, -0.7]]).T


def _write(tmp_path, fmt, name="A", **kw):
    if fmt == "pspnc":
        return S.write_abinit_file(str(tmp_path / f"{name}.pspnc"), **kw)
    return S.write_fhi_file(str(tmp_path / f"{name}.{fmt}"), abinit=fmt == "fhi", **kw)


def _lib(files, lloc, grid, rion, kion, lmax=None, vpsl=True):
    from salmon2_b200 import pseudo
    return pseudo.init_ps(files, lloc, grid, rion, kion, lmax_ps=lmax, vpsl=vpsl)


@pytest.mark.parametrize("periodic", [False, True], ids=["isolated", "periodic"])
@pytest.mark.parametrize("fmt", ["pspnc", "fhi", "cpi"])
def test_tables_equal_oracle(tmp_path, fmt, periodic):
    g = _grid(periodic)
    f = _write(tmp_path, fmt, zps=4.0, mlps=2, seed=5)
    pp, v = _lib([f], [2], g, _rion(periodic), [1, 1])
    mps, jxyz, rxyz, uv, ia, rinv, vref = PK.init_ps_ky([f], [2], g, _rion(periodic), [1, 1], by_name=True)
    assert pp.nlma == 2 * (1 + 3) and pp.mps.min() > 0
    assert np.array_equal(pp.mps, mps) and np.array_equal(pp.jxyz, jxyz)
    assert np.array_equal(pp.ia_tbl, ia) and np.array_equal(pp.rinv_uvu, rinv)
    assert np.max(np.abs(pp.rxyz - rxyz)) <= 1e-14 * max(1.0, np.max(np.abs(rxyz)))
    assert np.max(np.abs(pp.uv - uv)) <= 1e-12 * np.max(np.abs(uv))
    assert np.max(np.abs(v - vref)) <= 1e-11 * np.max(np.abs(vref))


def test_fhi_and_cpi_forms_give_identical_tables(tmp_path):
    """read_ps_abinitfhi and read_ps_fhi differ in the header, the optional
    core-correction block and the last grid point of the continuation."""
    g = _grid(False)
    a = S.write_fhi_file(str(tmp_path / "A.fhi"), abinit=True, nlcc=True, seed=6)
    b = S.write_fhi_file(str(tmp_path / "A.cpi"), abinit=False, seed=6)
    pa, va = _lib([a], [1], g, _rion(False), [1, 1])
    pb, vb = _lib([b], [1], g, _rion(False), [1, 1])
    for x, y in ((pa.mps, pb.mps), (pa.jxyz, pb.jxyz), (pa.rxyz, pb.rxyz), (pa.uv, pb.uv),
                 (pa.rinv_uvu, pb.rinv_uvu), (va, vb)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("periodic", [False, True], ids=["isolated", "periodic"])
def test_abinit_and_fhi_forms_give_the_same_tables(tmp_path, periodic):
    mmax, mlps, zps = 600, 2, 4.0
    rad = np.array([1.0e2 * (i / (mmax - 1) + 1.0e-2) ** 5 - 1.0e-8 for i in range(mmax)])
    rng = np.random.default_rng(8)
    amp = rng.uniform(-0.3, 0.3, mlps + 1)
    upp = np.zeros((mmax, mlps + 1))
    vpp = np.zeros((mmax, mlps + 1))
    for i in range(1, mmax):
        for l in range(mlps + 1):
            vpp[i, l], upp[i, l] = S._au_channels(rad[i], zps, amp, l)
    # FHI: upp(i), vpp(i) at rad(i + 1), i = 1..mr; rad(1) = 0, upp(0) = 0, vpp(0) extrapolated
    mr = mmax - 1
    fhi = S.write_fhi_file(str(tmp_path / "A.cpi"), abinit=False, zps=zps, mlps=mlps, radii=rad[1:],
                           values=(upp[1:], vpp[1:]), ratio=float(rad[-1] / rad[-2]))
    for l in range(mlps + 1):
        vpp[0, l] = vpp[1, l] - (vpp[2, l] - vpp[1, l]) / (rad[2] - rad[1]) * rad[1]
    assert PK.KyElement(fhi, None, 0, 20000, fmt="FHI").mr == mr
    _, rrc = PK._read_fhi(PK.KyElement.__new__(PK.KyElement), fhi, 20000, False)
    ab = S.write_abinit_file(str(tmp_path / "A.pspnc"), zps=zps, mlps=mlps, mmax=mmax, rc=list(rrc),
                             values=(upp, vpp))
    g = _grid(periodic)
    pa, va = _lib([ab], [0], g, _rion(periodic), [1, 1])
    pf, vf = _lib([fhi], [0], g, _rion(periodic), [1, 1])
    assert pa.nlma == pf.nlma == 2 * (3 + 5)
    assert np.array_equal(pa.mps, pf.mps) and np.array_equal(pa.jxyz, pf.jxyz)
    assert np.array_equal(pa.rinv_uvu, pf.rinv_uvu)
    assert np.max(np.abs(pa.uv - pf.uv)) <= 1e-13 * np.max(np.abs(pf.uv))
    if periodic:  # the isolated Vpsl reaches the grid continuation, which differs beyond the file
        assert np.max(np.abs(va - vf)) <= 1e-13 * np.max(np.abs(vf))


@pytest.mark.parametrize("name,code", [("A.psp8", 3), ("A.upf", 3), ("A.vps", 3), ("A.dat", 1)])
def test_unsupported_and_unknown_formats_are_refused(tmp_path, name, code):
    from salmon2_b200 import _lib as L
    p = tmp_path / name
    p.write_text("0\n")
    with pytest.raises(L.SB200Error) as e:
        _lib([str(p)], [0], _grid(False), _rion(False), [1, 1])
    assert e.value.code == code


def test_ky_file_through_the_general_entry_equals_the_ky_entry(tmp_path):
    from salmon2_b200 import pseudo
    f = S.write_ky_file(str(tmp_path / "A_rps.dat"), seed=9)
    g = _grid(True)
    pa, va = pseudo.init_ps([f], [1], g, _rion(True), [1, 1])
    pb, vb = pseudo.init_ps_ky([f], [1], g, _rion(True), [1, 1])
    assert np.array_equal(pa.uv, pb.uv) and np.array_equal(va, vb) and np.array_equal(pa.jxyz, pb.jxyz)
