"""Small seeded systems shared by the parity tests (sizes the oracle finishes
in seconds).  Shapes cover periodic / isolated grids, odd and even extents,
non-cubic boxes, several k-points and both spins."""
import functools

import numpy as np

from salmon2_b200 import synth


@functools.lru_cache(maxsize=None)
def periodic_small(nspin=1):
    # 12^3 diamond cell, 2^3 k-points, 4 orbitals per k
    return synth.periodic_system(a=10.26, num=12, nkgrid=2, no=4, seed=11, nspin=nspin, name="periodic12")


@functools.lru_cache(maxsize=None)
def periodic_c2_like():
    # the C2 cell at full grid resolution (16^3) with one k-point
    return synth.periodic_system(a=10.26, num=16, nkgrid=1, no=3, seed=12, name="periodic16")


@functools.lru_cache(maxsize=None)
def isolated_small():
    return synth.isolated_system(num=24, no=3, natom=2, seed=13, name="isolated24")


@functools.lru_cache(maxsize=None)
def isolated_odd():
    # odd and unequal extents exercise the coordinate shift and the halo
    return synth.isolated_system(num=(21, 19, 17), no=2, natom=2, seed=14, name="isolated_odd")


def no_pp(system):
    pp = synth.PPGrid(0, 0, 0, np.zeros(0, np.int32), np.zeros((3, 0, 0), np.int32, order="F"),
                      np.zeros((3, 0, 0), order="F"), np.zeros((0, 0), order="F"), np.zeros(0, np.int32),
                      np.zeros(0))
    import dataclasses
    return dataclasses.replace(system, pp=pp)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0))


def write_ky_file(path, zps=4.0, mlps=2, mr=400, step=0.01, rc=1.1, seed=0):
    """A Yabana-Bertsch (`_rps.dat`, ps_format 'KY') file with smooth analytic
    channels (angstrom / eV, the format's units): v_l(r) = -zps e^2 erf(r/0.4)/r
    + A_l exp(-(r/0.5)^2), u_l(r) = r^(l+1) exp(-r^2 / 0.72); cut-off radii rc."""
    from math import erf
    rng = np.random.default_rng(seed)
    e2 = 14.399645  # eV * angstrom
    amp = rng.uniform(-8.0, 8.0, mlps + 1)
    lines = [f"{mr:12d} {step:11.5f} {mlps:11d} {zps:11.5f}",
             f"{0:12d} " + " ".join(f"{rc:11.5f}" for _ in range(mlps + 1))]
    rs = [i * step for i in range(mr + 1)]
    for r in rs:
        vs = []
        for l in range(mlps + 1):
            vc = -zps * e2 * (erf(r / 0.4) / r if r > 0 else 2.0 / (0.4 * np.sqrt(np.pi)))
            vs.append(vc + amp[l] * np.exp(-(r / 0.5) ** 2))
        lines.append(f"{r:11.4f} {0.0:11.5f} " + " ".join(f"{v:14.7f}" for v in vs))
    for r in rs:
        us = [r ** (l + 1) * np.exp(-r * r / 0.72) for l in range(mlps + 1)]
        lines.append(f"{r:11.4f} " + " ".join(f"{u:14.9f}" for u in us))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
