"""Host-side set-up of the Kleinman-Bylander tables from Yabana-Bertsch
pseudopotential files (sb200_init_ps_ky; read_ps_KY, input_pp,
making_ps_without_masking, init_ps, calc_Vpsl_isolated) against the oracle's
numpy restatement (oracle/pseudo_ky.py), on CPU (the builder has no device
code): the sphere tables bit for bit, uV and rinv_uvu to 1e-12, Vpsl (isolated
by interpolation, periodic by form factors and transforms) to 1e-11, on
isolated grids of odd and even extent and on a periodic cell whose spheres
cross the boundary; the reference's own C and H files when the reference tree
is present; known answers of the spline."""
import os

import numpy as np
import pytest

import _systems as S
import pseudo_ky as PK

REF_PSEUDO = os.path.join(os.environ.get("SALMON_REFERENCE", os.path.join(os.path.dirname(__file__), "..", "..",
                                                                          "reference")), "testsuites", "pseudo")


def _compare(files, lloc, grid, rion, kion, lmax=None):
    from salmon2_b200 import pseudo
    pp, v = pseudo.init_ps_ky(files, lloc, grid, rion, kion, lmax_ps=lmax)
    mps, jxyz, rxyz, uv, ia, rinv, vref = PK.init_ps_ky(files, lloc, grid, rion, kion, lmax_ps=lmax)
    assert np.array_equal(pp.mps, mps)
    assert pp.nps == jxyz.shape[1] and pp.nlma == uv.shape[1]
    assert np.array_equal(pp.jxyz, jxyz)
    assert np.max(np.abs(pp.rxyz - rxyz)) <= 1e-14 * max(1.0, np.max(np.abs(rxyz)))
    assert np.array_equal(pp.ia_tbl, ia) and np.array_equal(pp.rinv_uvu, rinv)
    if uv.size:
        assert np.max(np.abs(pp.uv - uv)) <= 1e-12 * np.max(np.abs(uv))
    if vref is not None:
        assert np.max(np.abs(v - vref)) <= 1e-11 * np.max(np.abs(vref))
    return pp, v


@pytest.mark.parametrize("num", [24, 25])
def test_isolated_tables_equal_oracle(tmp_path, num):
    from salmon2_b200 import synth
    fa = S.write_ky_file(str(tmp_path / "A_rps.dat"), zps=4.0, mlps=2, seed=1)
    fb = S.write_ky_file(str(tmp_path / "B_rps.dat"), zps=1.0, mlps=1, rc=0.9, seed=2)
    g = synth.make_grid([num, num, num], 0.25 / synth.AU_LENGTH_AA, periodic=False)
    rion = np.array([[0.3, -0.2, 1.1], [-1.4, 0.5, -0.7], [2.0, 1.7, 0.1]]).T
    pp, v = _compare([fa, fb], [2, 0], g, rion, [1, 2, 1])
    assert pp.nlma == 2 * (1 + 3) + 3  # l = 0, 1 on the two A atoms (l = 2 local), l = 1 on B (l = 0 local)
    assert np.all(np.isfinite(v))


def test_periodic_tables_equal_oracle(tmp_path):
    """Atoms near the cell faces: spheres reach through the periodic images."""
    from salmon2_b200 import synth
    fa = S.write_ky_file(str(tmp_path / "A_rps.dat"), zps=4.0, mlps=1, seed=3)
    g = synth.make_grid([12, 12, 12], 6.0 / 12, periodic=True)
    rion = np.array([[0.2, 5.9, 3.0], [3.1, 0.1, 5.8]]).T
    pp, v = _compare([fa], [1], g, rion, [1, 1])
    assert pp.nlma == 2
    assert pp.mps.min() > 0
    assert np.all(np.isfinite(v)) and abs(np.mean(v)) < np.max(np.abs(v))


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_PSEUDO, "C_rps.dat")),
                    reason="reference pseudopotential files not present")
def test_reference_carbon_and_hydrogen_files(tmp_path):
    """The reference's own C and H files (testsuites/pseudo) on a 16 A box of
    h = 0.25 A with four atoms on the z axis (Lmax_ps = 1 / 0, Lloc_ps = 1 / 0):
    one s projector per C atom, none on H; Vpsl's far field ~ -Z_total / r."""
    from salmon2_b200 import synth
    files = [os.path.join(REF_PSEUDO, "C_rps.dat"), os.path.join(REF_PSEUDO, "H_rps.dat")]
    g = synth.make_grid([64, 64, 64], 0.25 / synth.AU_LENGTH_AA, periodic=False)
    z = np.array([1.13, 3.14, -1.13, -3.14])
    rion = np.stack([np.zeros(4), np.zeros(4), z])
    pp, v = _compare(files, [1, 0], g, rion, [1, 2, 1, 2], lmax=[1, 0])
    assert pp.nlma == 2 and list(pp.ia_tbl) == [1, 3]
    corner = np.linalg.norm([31.5 * g.hgs[0]] * 3)
    assert abs(v[0, 0, 0] - (-10.0 / corner)) < 0.05 * 10.0 / corner


def test_spline_interpolates_and_is_twice_continuous():
    """The natural cubic spline of salmon_math.f90 passes through the nodes,
    keeps first and second derivatives continuous at interior nodes, has zero
    curvature at both ends, and reproduces a straight line exactly."""
    rng = np.random.default_rng(5)
    x = np.cumsum(rng.uniform(0.05, 0.2, 30))
    y = np.sin(3 * x) + 0.1 * x
    a, b, c, d = PK.spline(x, y)
    h = np.diff(x)
    assert np.allclose(d, y[:-1], rtol=0, atol=1e-14)
    assert np.allclose(a * h ** 3 + b * h ** 2 + c * h + d, y[1:], rtol=0, atol=1e-12)
    assert np.allclose((3 * a * h ** 2 + 2 * b * h + c)[:-1], c[1:], atol=1e-10)
    assert np.allclose((6 * a * h + 2 * b)[:-1], 2 * b[1:], atol=1e-9)
    assert abs(b[0]) < 1e-15 and abs(6 * a[-1] * h[-1] + 2 * b[-1]) < 1e-9
    a, b, c, d = PK.spline(x, 2.5 * x - 1.0)
    assert np.allclose(c, 2.5, atol=1e-12) and np.allclose(a, 0, atol=1e-10) and np.allclose(b, 0, atol=1e-10)
