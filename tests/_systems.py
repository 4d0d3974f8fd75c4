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
