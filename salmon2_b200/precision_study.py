"""Error of the mixed-precision form against the FP64 form on the GPU.

Runs the same real-time propagation twice through ``sb200_rt_propagate`` --
SB200_PREC_FP64 and SB200_PREC_MIXED (FP32 stencil and Taylor terms n >= 2,
FP64 first term, psi accumulation, density and current) -- and reports:

* ``J_rel_err``: max_t |J_mixed(t) - J_fp64(t)| / max_t |J_fp64(t)| (the
  current of calc_current, src/common/density_matrix.f90:240-463);
* ``spectrum_rel_err``: the same for |FFT(J(t))| with a Hann window, the
  quantity a response spectrum is computed from;
* ``norm_drift``: max_t |N_mixed(t) - N_fp64(t)| / N_fp64(0) with N the
  electron count of calc_dip (src/rt/dip.f90:114-225);
* ``energy_rel_err``: relative difference of the band energy
  sum_o w_o <psi_o|H|psi_o> hvol of the final orbitals (esp of
  sb200_calc_eigen_energy, calc_eigen_energy in src/common/total_energy.f90:505-775).

Usage: ``python -m salmon2_b200.precision_study --nt 4000`` (the 2x2x2
supercell workload: 32^3 grid, 64 atoms, 8 k-points, 256 orbitals per k).

The initial orbitals are band-limited plane-wave sums (kinetic energy
|k+G|^2/2 <= ``--ecut`` Hartree, 2.0 by default), a stand-in for occupied
states; ``--white`` uses white-noise fields instead, whose spectral weight sits
near the grid cutoff (mean kinetic energy about 12 Hartree at h = 0.64 bohr),
where the Taylor terms n >= 2 are of the order of psi itself and the FP32
rounding of those terms is largest.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def band_energy(ctx, psi):
    """sum_o rocc wtk esp_o with esp from sb200_calc_eigen_energy."""
    esp, _, _ = ctx.calc_eigen_energy(psi)
    s = ctx.sys
    occ = np.asarray(s.rocc, dtype=np.float64)  # (no, nk, nspin)
    return float(np.sum(occ * esp * np.asarray(s.wtk)[None, :, None]))


def run(system, nt, dt, Ac, zc, precision):
    from .rt import Context
    ctx = Context(system, precision=precision)
    a, b, w = ctx.upload(system.psi), ctx.zeros(), ctx.zeros()
    t0 = time.perf_counter()
    res = ctx.rt_propagate(a, b, w, nt, dt, zc, Ac_ext=Ac)
    ctx.sync()
    el = time.perf_counter() - t0
    ctx.set_vec_Ac(Ac[:, nt])
    e = band_energy(ctx, res["psi"])
    out = dict(curr=res["curr"].copy(), rbox=res["rbox"].copy(), energy=e, seconds=el)
    ctx.close()
    return out


def compare(r64, rmx):
    J64, Jmx = r64["curr"], rmx["curr"]
    jmax = np.max(np.abs(J64))
    win = np.hanning(J64.shape[1])
    S64 = np.abs(np.fft.rfft(J64 * win, axis=1))
    Smx = np.abs(np.fft.rfft(Jmx * win, axis=1))
    n64, nmx = r64["rbox"][3], rmx["rbox"][3]
    return {
        "J_rel_err": float(np.max(np.abs(Jmx - J64)) / jmax),
        "spectrum_rel_err": float(np.max(np.abs(Smx - S64)) / np.max(S64)),
        "norm_drift": float(np.max(np.abs(nmx - n64)) / n64[0]),
        "energy_rel_err": float(abs(rmx["energy"] - r64["energy"]) / abs(r64["energy"])),
        "fp64_seconds": r64["seconds"], "mixed_seconds": rmx["seconds"],
        "speedup": r64["seconds"] / rmx["seconds"],
    }


def main():
    from . import synth
    ap = argparse.ArgumentParser()
    ap.add_argument("--nt", type=int, default=4000)
    ap.add_argument("--nkgrid", type=int, default=2)
    ap.add_argument("--ecut", type=float, default=2.0)
    ap.add_argument("--white", action="store_true")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    ecut = None if args.white else args.ecut
    s = synth.periodic_system(a=10.26, num=16, nkgrid=args.nkgrid, no=256, supercell=2, seed=3,
                              name="periodic_supercell", ecut=ecut)
    dt = 0.08
    omega = 1.55 / synth.AU_ENERGY_EV
    Ac = synth.asin2cos(args.nt, dt, omega=omega, f0=omega * 1e-3, tw=args.nt * dt)
    zc = synth.taylor_zc(dt)
    r64 = run(s, args.nt, dt, Ac, zc, "fp64")
    rmx = run(s, args.nt, dt, Ac, zc, "mixed")
    res = compare(r64, rmx)
    res.update(workload=f"periodic supercell 32^3, {s.pp.natom} atoms, {s.nk} k, {s.no} orbitals/k, "
                        f"{args.nt} steps dt={dt}", nt=args.nt,
               orbitals="white noise" if ecut is None else f"band-limited, |k+G|^2/2 <= {ecut} Ha")
    print(json.dumps(res), flush=True)
    if args.out:
        json.dump(res, open(args.out, "w"))


if __name__ == "__main__":
    main()
