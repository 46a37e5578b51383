"""Generates the golden fixtures in this directory from the reference's own C
(so3_core.c / so3_sampling.c compiled unmodified against the checker's SSHT
and FFTW stand-ins: ``make -C oracle ref``).  Needs the reference tree, so it
runs on the build machine only; the .npz files are committed.

Each fixture holds a seeded flmn, the reference's inverse f, and the
reference's forward of f, for one parameter set.

  python tests/golden/gen_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from so3_b200 import synth  # noqa: E402
from so3_b200.api import SO3Parameters  # noqa: E402

CASES = [
    dict(L=8, N=8, method=1, sampling=0),
    dict(L=8, N=8, method=1, sampling=1),
    dict(L=8, N=8, method=0, reality=1),
    dict(L=10, N=4, L0=2, method=0, storage=1, order=0),
    dict(L=12, N=5, method=0, reality=1, sampling=1, storage=1),
    dict(L=16, N=16, method=0),
    dict(L=9, N=6, method=1, mode=3),
]


def main():
    O.build(ref=True)
    assert O.ref() is not None, "reference build failed"
    for i, c in enumerate(CASES):
        op = O.params(**c)
        p = SO3Parameters(L=op.L, N=op.N, L0=op.L0, reality=op.reality, sampling_scheme=op.sampling_scheme,
                          n_order=op.n_order, storage=op.storage, n_mode=op.n_mode, dl_method=op.dl_method)
        fl = synth.gen_flmn(p, 100 + i)
        f = O.ref_inverse(fl, op)
        back = O.ref_forward(f, op)
        cfg = dict(L=op.L, N=op.N, L0=op.L0, reality=op.reality, sampling=op.sampling_scheme, order=op.n_order,
                   storage=op.storage, mode=op.n_mode, method=op.dl_method)
        np.savez_compressed(os.path.join(HERE, f"case{i:02d}.npz"), flmn=fl, f=f, flmn_back=back,
                            config=json.dumps(cfg))
        print(i, cfg, "ok")


if __name__ == "__main__":
    main()
