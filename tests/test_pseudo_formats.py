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


@pytest.fixture
def psmask():
    from salmon2_b200 import pseudo
    yield pseudo.set_psmask
    pseudo.set_psmask(False)


@pytest.mark.parametrize("periodic", [False, True], ids=["isolated", "periodic"])
def test_masked_tables_equal_oracle(tmp_path, psmask, periodic):
    """yn_psmask = 'y' (making_ps_with_masking, ps_masking, make_mask_function)
    with the reference's default alpha_mask, gamma_mask, eta_mask.  Tolerance
    1e-9 relative: the mask is the lowest eigenvector of a 200 x 200 matrix of
    norm 628 whose two lowest eigenvalues are 1.6e-7 and 3.0e-4, so any two
    symmetric eigensolvers (the library's Jacobi, numpy's, the reference's
    LAPACK dsyev) agree on it only to about eps * 628 / 3e-4 = 2e-10."""
    f = S.write_ky_file(str(tmp_path / "A_rps.dat"), zps=4.0, mlps=2, seed=14, compact=True, mr=500)
    g = _grid(periodic)
    psmask(True, 0.8, 1.8, 15.0)
    pp, v = _lib([f], [2], g, _rion(periodic), [1, 1])
    mps, jxyz, rxyz, uv, ia, rinv, vref = PK.init_ps_ky([f], [2], g, _rion(periodic), [1, 1], mask=(0.8, 1.8, 15.0))
    assert np.array_equal(pp.mps, mps) and np.array_equal(pp.jxyz, jxyz)
    assert np.array_equal(pp.rinv_uvu, rinv)
    assert np.max(np.abs(pp.uv - uv)) <= 1e-9 * np.max(np.abs(uv))
    assert np.max(np.abs(v - vref)) <= 1e-11 * np.max(np.abs(vref))


def test_masking_widens_the_sphere_and_keeps_the_smooth_projector(tmp_path, psmask):
    """The masked tables reach gamma_mask rps (more sphere points), and for a
    smooth projector the filtered, masked function stays close to the
    unmasked one inside the file's cut-off (the filter passes |k| below
    alpha_mask pi / h; the mask is near 1 at small r / rps)."""
    f = S.write_ky_file(str(tmp_path / "A_rps.dat"), zps=4.0, mlps=1, seed=15, compact=True, rc=1.3, mr=500)
    g = _grid(False)
    rion = np.array([[0.3, -0.2, 1.1]]).T
    p0, _ = _lib([f], [1], g, rion, [1])
    psmask(True)
    p1, _ = _lib([f], [1], g, rion, [1])
    assert p1.mps[0] > 2 * p0.mps[0]
    # the sphere points of the unmasked table, looked up in the masked one
    r0 = np.linalg.norm(p0.rxyz[:, : p0.mps[0], 0], axis=0)
    idx1 = {tuple(p1.jxyz[:, j, 0]): j for j in range(p1.mps[0])}
    sel = [j for j in range(p0.mps[0]) if r0[j] < 0.5 * 1.3 / 0.52917721067]
    a = p0.uv[sel, 0]
    b = p1.uv[[idx1[tuple(p0.jxyz[:, j, 0])] for j in sel], 0]
    assert np.max(np.abs(a - b)) < 0.05 * np.max(np.abs(a))


def test_mask_function_is_normalized_and_vanishes_at_the_cut_off():
    """make_mask_function: 1 at r = 0 (its normalization), decreasing to about
    zero at rps."""
    rad = np.linspace(0.0, 3.0, 301)
    m = PK.make_mask(rad, 201, rad[200], 15.0)
    assert abs(m[0] - 1.0) < 1e-3
    assert abs(m[-1]) < 2e-2 and np.all(np.diff(m[1:-1]) < 1e-12)


def test_masked_tables_from_the_reference_files(psmask):
    """The reference's own C and H files with yn_psmask = 'y', library
    against oracle (1e-9, as above)."""
    import os
    from test_pseudo_ky import REF_PSEUDO
    if not os.path.exists(os.path.join(REF_PSEUDO, "C_rps.dat")):
        pytest.skip("reference pseudopotential files not present")
    from salmon2_b200 import synth
    files = [os.path.join(REF_PSEUDO, "C_rps.dat"), os.path.join(REF_PSEUDO, "H_rps.dat")]
    g = synth.make_grid([48, 48, 48], 0.25 / synth.AU_LENGTH_AA, periodic=False)
    rion = np.array([[0.0, 0.0, 1.13], [0.0, 0.0, 3.14], [0.0, 0.0, -1.13], [0.0, 0.0, -3.14]]).T
    psmask(True)
    pp, v = _lib(files, [1, 0], g, rion, [1, 2, 1, 2], lmax=[1, 0])
    mps, jxyz, rxyz, uv, ia, rinv, vref = PK.init_ps_ky(files, [1, 0], g, rion, [1, 2, 1, 2], lmax_ps=[1, 0],
                                                        by_name=True, mask=(0.8, 1.8, 15.0))
    assert pp.nlma == 2 and np.array_equal(pp.jxyz, jxyz)
    assert np.max(np.abs(pp.uv - uv)) <= 1e-9 * np.max(np.abs(uv))
    assert np.max(np.abs(v - vref)) <= 1e-11 * np.max(np.abs(vref))
