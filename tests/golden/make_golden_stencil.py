"""Generate the golden fixture of the reference's AVX-512 stencil.

``oracle/_ref/libsalmon_ref_avx512.so`` is the reference's own hand-vectorised
stencil (src/common/zstencil_core/avx512/seq.c, built by ``make -C oracle
ref``).  This script runs it on seeded periodic inputs (the 25-point Laplacian,
the k+A gradient and V_local of every orbital, at two vector potentials) and
stores checksums and a strided sample of its output, so that
``tests/test_golden.py`` can check the oracle against the reference's stencil
on machines without the library or without AVX-512.

Run on a CPU with AVX-512:  python tests/golden/make_golden_stencil.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle"), HERE):
    sys.path.insert(0, p)

from salmon2_b200 import synth  # noqa: E402
from make_golden import checksum  # noqa: E402

OUT = os.path.join(HERE, "ref_stencil_avx512.npz")
A_VALUES = [(0.0, 0.0, 0.0), (0.013, -0.021, 0.034)]
SAMPLE_STRIDE = 37


def stencil_systems():
    import dataclasses
    # the local part only: no projectors
    def no_pp(s):
        pp = synth.PPGrid(0, 0, 0, np.zeros(0, np.int32), np.zeros((3, 0, 0), np.int32, order="F"),
                          np.zeros((3, 0, 0), order="F"), np.zeros((0, 0), order="F"), np.zeros(0, np.int32),
                          np.zeros(0))
        return dataclasses.replace(s, pp=pp)
    return {
        "p12_two_spins": no_pp(synth.periodic_system(a=10.26, num=12, nkgrid=2, no=2, seed=71, nspin=2,
                                                     name="stencil12")),
        "p16": no_pp(synth.periodic_system(a=10.26, num=16, nkgrid=1, no=3, seed=72, name="stencil16")),
    }


def sample(a):
    flat = np.asarray(a).ravel(order="F")
    return flat[::SAMPLE_STRIDE].copy()


def main():
    import ref_witness
    if not ref_witness.avx512_available():
        raise SystemExit("oracle/_ref/libsalmon_ref_avx512.so missing or no AVX-512 CPU: run `make -C oracle ref`")
    data = {}
    for name, s in stencil_systems().items():
        data[f"{name}_psi_checksum"] = checksum(s.psi)
        for i, ac in enumerate(A_VALUES):
            h = ref_witness.zstencil_avx512(s, s.psi, ac)
            data[f"{name}_h{i}_checksum"] = checksum(h)
            data[f"{name}_h{i}_sample"] = sample(h)
    np.savez_compressed(OUT, **data)
    print("wrote", OUT, {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main()
