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


def write_ky_file(path, zps=4.0, mlps=2, mr=400, step=0.01, rc=1.1, seed=0, compact=False):
    """A Yabana-Bertsch (`_rps.dat`, ps_format 'KY') file with smooth analytic
    channels (angstrom / eV, the format's units): v_l(r) = -zps e^2 erf(r/0.4)/r
    + A_l exp(-(r/0.5)^2), u_l(r) = r^(l+1) exp(-r^2 / 0.72); cut-off radii rc.
    compact: the channels differ by A_l (1 - (r/rc)^2)^3 inside rc only, so
    they are equal beyond it as in real files."""
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
            if compact:
                vs.append(vc + (amp[l] * (1.0 - (r / rc) ** 2) ** 3 if r < rc else 0.0))
            else:
                vs.append(vc + amp[l] * np.exp(-(r / 0.5) ** 2))
        lines.append(f"{r:11.4f} {0.0:11.5f} " + " ".join(f"{v:14.7f}" for v in vs))
    for r in rs:
        us = [r ** (l + 1) * np.exp(-r * r / 0.72) for l in range(mlps + 1)]
        lines.append(f"{r:11.4f} " + " ".join(f"{u:14.9f}" for u in us))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def _au_channels(r, zps, amp, l):
    """Smooth analytic channels in Hartree atomic units for the non-KY
    fixtures: v_l(r) = -zps erf(r/0.75)/r + A_l exp(-(r/0.5)^4), u_l(r) =
    r^(l+1) exp(-r^2/2.6) (the channels differ only inside r ~ 1.1 bohr)."""
    from math import erf
    vc = -zps * (erf(r / 0.75) / r if r > 0 else 2.0 / (0.75 * np.sqrt(np.pi)))
    return vc + amp[l] * np.exp(-(r / 0.5) ** 4), r ** (l + 1) * np.exp(-r * r / 2.6)


def write_fhi_file(path, zps=4.0, mlps=2, mr=420, r1=0.0005, ratio=1.0247, seed=0, abinit=True, radii=None,
                   values=None, nlcc=False):
    """An FHI pseudopotential file: with abinit, the `.fhi` form of the ABINIT
    tables (seven header lines first); else FHI98PP `.cpi`.  radii: the
    mr grid radii rad(2..mr+1) (default r1 ratio^(i-1)); values: optional
    (upp, vpp) arrays (mr, mlps + 1) at those radii instead of the analytic
    channels.  nlcc: append a core-correction block on the same radii."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(-0.3, 0.3, mlps + 1)
    rs = np.asarray(radii, dtype=np.float64) if radii is not None else r1 * ratio ** np.arange(mr)
    mr = len(rs)
    lines = []
    if abinit:
        lines += ["synthetic FHI pseudopotential (ABINIT table form)",
                  f"  {float(zps):.4f}  {float(zps):.4f}    000101              zatom,zion,pspdat",
                  "   6   1   2   0   {0}   0.00000  pspcod,pspxc,lmax,lloc,mmax,r2well".format(mr),
                  "  0.00000  -1.00000  0.00000                rchrg,fchrg,qchrg",
                  "5--- reserved for future features", "6--- reserved for future features",
                  "7--- Here follows the cpi file in the fhi98pp format -"]
    lines.append(f"{zps:.4f}  {mlps + 1}")
    R = lambda x: repr(float(x))
    for k in range(10):
        lines.append(f"  0.0000000000E+00  0.0000000000E+00  0.0000000000E+00   # line {k}")
    for l in range(mlps + 1):
        lines.append(f"{mr:5d} {R(ratio)}")
        for i, r in enumerate(rs):
            if values is None:
                v, u = _au_channels(r, zps, amp, l)
            else:
                u, v = values[0][i, l], values[1][i, l]
            lines.append(f"{i + 1:5d} {R(r)} {R(u)} {R(v)}".replace("e", "D"))
    if nlcc:
        for r in rs:
            lines.append(f"{R(r)} {np.exp(-r):.15e} {-np.exp(-r):.15e} {np.exp(-r):.15e}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


def write_abinit_file(path, zps=4.0, mlps=2, mmax=600, lloc=0, rc=None, seed=0, values=None):
    """An ABINIT format-1 (`.pspnc`, Troullier-Martins) file on ABINIT's grid
    rad(i + 1) = 100 (i / (mmax - 1) + 0.01)^5 - 1e-8, Hartree atomic units.
    rc: per-channel cut-off radii (default 1.3 bohr); values: optional (upp,
    vpp) arrays (mmax, mlps + 1) at indices 0..mmax-1."""
    assert mmax % 3 == 0
    rng = np.random.default_rng(seed)
    amp = rng.uniform(-0.3, 0.3, mlps + 1)
    rc = [1.3] * (mlps + 1) if rc is None else list(rc)
    rad = [1.0e2 * (i / (mmax - 1) + 1.0e-2) ** 5 - 1.0e-8 for i in range(mmax)]
    lines = ["synthetic Troullier-Martins pseudopotential",
             f"  {zps:.5f}  {zps:.5f}  000101    zatom, zion, pspdat",
             f"   1   1   {mlps}   {lloc}   {mmax}   0.00000    pspcod,pspxc,lmax,lloc,mmax,r2well"]
    for l in range(mlps + 1):
        lines.append(f"   {l}   0.000   0.000   1   {float(rc[l])!r}   l,e99.0,e99.9,nproj,rcpsp")
        lines.append("   0.00000000   0.00000000   0.00000000   0.00000000   rms,ekb1,ekb2,epsatm")
    lines.append("   0.00000000   0.00000000   0.00000000   rchrg,fchrg,qchrg")
    for which in (1, 0):  # potentials, then wave functions
        for l in range(mlps + 1):
            lines.append(f"{l} = l for {'potential' if which else 'wavefunction'}")
            vals = []
            for i in range(mmax):
                if values is None:
                    v, u = _au_channels(rad[i], zps, amp, l)
                else:
                    u, v = values[0][i, l], values[1][i, l]
                vals.append(v if which else u)
            for i in range(0, mmax, 3):
                lines.append(" ".join(repr(float(x)) for x in vals[i:i + 3]))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
