"""Generate the golden fixtures that pin the oracle to the reference.

The reference's own CUDA kernels for the KB nonlocal term (zpseudo_cuda,
src/common/zpseudo.cu) and for the local part of the current
(stencil_current_core_gpu, src/common/stencil_current.cu) are compiled from
the reference sources (``make -C oracle ref``) and run on a GPU on seeded
inputs.  Their outputs are stored here next to checksums of the inputs, so the
CPU test ``tests/test_golden.py`` can check the oracle against the reference
without a GPU.

Run on a machine with a CUDA GPU:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from salmon2_b200 import synth  # noqa: E402

OUT = os.path.join(HERE, "ref_witness.npz")
A_VALUES = [(0.0, 0.0, 0.0), (0.013, -0.021, 0.034)]


def witness_systems():
    per = synth.periodic_system(a=10.26, num=16, nkgrid=2, no=2, seed=101, name="witness_periodic")
    iso = synth.isolated_system(num=24, no=2, natom=2, seed=102, name="witness_isolated")
    return per, iso


def checksum(a):
    a = np.asarray(a)
    flat = a.ravel(order="F")
    w = np.cos(0.37 * np.arange(flat.size))
    return np.array([np.sum(flat).real, np.sum(flat).imag if np.iscomplexobj(flat) else 0.0,
                     np.sum(np.abs(flat) ** 2), np.sum(w * flat).real])


def sphere_sample(system, arr):
    """values of arr at every sphere point of every atom, orbitals 0..1."""
    g, pp = system.grid, system.pp
    out = []
    for ia in range(pp.natom):
        for j in range(pp.mps[ia]):
            ix, iy, iz = (int(pp.jxyz[d, j, ia]) - int(g.is_array[d]) for d in range(3))
            out.append(arr[ix, iy, iz].reshape(-1, order="F")[:2])
    return np.array(out)


def main():
    from oracle import Oracle
    import ref_witness
    if not ref_witness.available():
        raise SystemExit("oracle/_ref/libsalmon_ref_cuda.so missing: run `make -C oracle ref` first")
    per, iso = witness_systems()
    data = {}
    for name, sysm in (("periodic", per), ("isolated", iso)):
        O = Oracle(sysm)
        data[f"{name}_psi_checksum"] = checksum(sysm.psi)
        data[f"{name}_uv_checksum"] = checksum(sysm.pp.uv)
        for ia_, ac in enumerate(A_VALUES if sysm.grid.periodic else A_VALUES[:1]):
            O.set_vec_Ac(ac)
            href = ref_witness.zpseudo(sysm, sysm.psi, O.zekr)
            data[f"{name}_zpseudo{ia_}_checksum"] = checksum(href)
            data[f"{name}_zpseudo{ia_}_sphere"] = sphere_sample(sysm, href)
            if sysm.grid.periodic:
                data[f"{name}_current{ia_}"] = ref_witness.stencil_current(sysm, sysm.psi, ac)
    np.savez_compressed(OUT, **data)
    print("wrote", OUT, {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main()
