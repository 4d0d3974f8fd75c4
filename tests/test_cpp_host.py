"""The C++ host mirror (include/salmon_b200.hpp): SALMON's hpsi / taylor call
surface in a compiled language, driven by tests/cpp/host_mirror.cpp.

CPU: the driver compiles and links against the library.  GPU: on a periodic
system with two k-points the driver's H psi, kinetic part T psi, eigen
energies, current, density and Taylor step match the oracle, and an invalid
(aliased) hpsi call raises salmon_b200::error with SB200_ERR_INVALID_ARG.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

import _systems as S
from oracle import Oracle
from salmon2_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"
TOL = 1e-12


def build(tmp_path):
    exe = str(tmp_path / "host_mirror")
    libdir = os.path.join(ROOT, "salmon2_b200")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", f"{CUDA}/include",
           os.path.join(ROOT, "tests", "cpp", "host_mirror.cpp"), "-o", exe, "-L", libdir, "-lsalmon_b200",
           f"-Wl,-rpath,{libdir}", "-L", f"{CUDA}/lib64", "-lcudart", f"-Wl,-rpath,{CUDA}/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def write_records(path, recs):
    with open(path, "wb") as f:
        for name, arr in recs.items():
            a = np.asarray(arr)
            kind = 0 if a.dtype.kind in "iu" else 1
            data = np.ascontiguousarray(a.ravel(order="F"), dtype=np.int32 if kind == 0 else np.float64)
            f.write(struct.pack("<I", len(name)) + name.encode() + struct.pack("<IQ", kind, data.size))
            f.write(data.tobytes())


def read_records(path):
    out = {}
    with open(path, "rb") as f:
        while True:
            h = f.read(4)
            if not h:
                break
            n = struct.unpack("<I", h)[0]
            name = f.read(n).decode()
            kind, count = struct.unpack("<IQ", f.read(12))
            dt = np.int32 if kind == 0 else np.float64
            out[name] = np.frombuffer(f.read(count * np.dtype(dt).itemsize), dtype=dt)
    return out


def system_records(s, vec_Ac, zc):
    g, pp = s.grid, s.pp
    zwf = np.asfortranarray(s.psi)
    return {
        "is": np.asarray(g.is_, np.int32), "ie": np.asarray(g.ie, np.int32),
        "is_array": np.asarray(g.is_array, np.int32), "ie_array": np.asarray(g.ie_array, np.int32),
        "lg_num": np.asarray(g.num, np.int32),
        "idx": np.asarray(g.idx, np.int32), "idy": np.asarray(g.idy, np.int32), "idz": np.asarray(g.idz, np.int32),
        "coef_lap0": np.array([g.coef_lap0]), "coef_lap": np.asarray(g.coef_lap), "coef_nab": np.asarray(g.coef_nab),
        "nspin_no_nk": np.array([s.nspin, s.no, s.nk], np.int32),
        "hgs": np.asarray(g.hgs, np.float64), "hvol": np.array([g.hvol]),
        "vec_k": np.asarray(s.vec_k, np.float64), "rocc": np.asarray(s.rocc, np.float64),
        "wtk": np.asarray(s.wtk, np.float64), "vec_Ac": np.asarray(vec_Ac, np.float64),
        "V_local": np.asarray(s.V_local, np.float64),
        "natom_nps_nlma": np.array([pp.natom, pp.nps, pp.nlma], np.int32),
        "mps": np.asarray(pp.mps, np.int32), "jxyz": np.asarray(pp.jxyz, np.int32),
        "rxyz": np.asarray(pp.rxyz, np.float64), "uv": np.asarray(pp.uv, np.float64),
        "ia_tbl": np.asarray(pp.ia_tbl, np.int32), "rinv_uvu": np.asarray(pp.rinv_uvu, np.float64),
        "zc": np.asarray(zc, np.complex128).view(np.float64),
        "zwf": zwf.ravel(order="F").view(np.float64),
        "primitive_b": np.diag([2 * np.pi / (n * h) for n, h in zip(g.shape, g.hgs)]),
    }


def test_host_mirror_builds(tmp_path):
    build(tmp_path)


@pytest.mark.gpu
def test_host_mirror_parity(tmp_path):
    s = S.periodic_small()
    ac = (0.012, -0.006, 0.018)
    zc = synth.taylor_zc(0.08)
    exe = build(tmp_path)
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    write_records(fin, system_records(s, ac, zc))
    r = subprocess.run([exe, fin, fout], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    res = read_records(fout)
    O = Oracle(s)
    O.set_vec_Ac(ac)
    shape = s.psi.shape

    def orb(name):
        return res[name].view(np.complex128).reshape(shape, order="F")

    ref_h, ref_tt = O.hpsi_tt(s.psi)
    assert S.rel_err(orb("htpsi"), ref_h) < TOL
    assert S.rel_err(orb("ttpsi"), ref_tt) < TOL
    esp, ek, en = O.calc_eigen_energy(s.psi)
    assert np.max(np.abs(res["esp"].reshape(esp.shape, order="F") - esp)) <= TOL * np.max(np.abs(esp))
    assert abs(res["ekin"][0] - ek) <= TOL * abs(ek)
    assert abs(res["enl"][0] - en) <= TOL * max(abs(en), np.max(np.abs(esp)))
    curr = O.current(s.psi)
    assert np.max(np.abs(res["curr"].reshape(curr.shape, order="F") - curr)) <= 1e-10 * np.max(np.abs(curr)) + 1e-16
    rho = O.density(s.psi)
    assert S.rel_err(res["rho0"].reshape(rho[..., 0].shape, order="F"), rho[..., 0]) < TOL
    assert S.rel_err(orb("taylor"), O.taylor(s.psi, zc)) < TOL
    assert res["alias_code"][0] == 1.0  # SB200_ERR_INVALID_ARG
    # hartree / exchange_correlation / update_vlocal of that density, then H psi with the new V_local
    import oracle as OR
    g = s.grid
    brl = np.diag([2 * np.pi / (n * h) for n, h in zip(g.shape, g.hgs)])
    r0 = rho[..., 0]
    vh = OR.poisson_ft(r0, brl)
    vxc, exc = OR.exc_cor_pz(r0, g.hvol)
    assert S.rel_err(res["Vh"].reshape(r0.shape, order="F"), vh) < TOL
    assert S.rel_err(res["Vxc"].reshape(r0.shape, order="F"), vxc) < TOL
    assert abs(res["E_xc"][0] - exc) <= TOL * abs(exc)
    import dataclasses
    O2 = Oracle(dataclasses.replace(s, V_local=OR.update_vlocal(s.V_local[..., 0], vh, vxc[..., None])))
    O2.set_vec_Ac(ac)
    assert S.rel_err(orb("htpsi_scf"), O2.hpsi(s.psi)) < TOL
