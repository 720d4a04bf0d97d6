"""Records outputs of the reference's OWN CUDA path (oracle/_ref/libfastcone_ref.so, built
from the unmodified reference sources by oracle/Makefile) on a B200, as fixtures that pin
the CPU oracle without a GPU.

    python tests/golden/make_golden_gpu.py OUTDIR

Inputs are regenerated deterministically from the seeds stored in each fixture
(tests/golden/ref_cases.py), so only outputs (and, for small cases, inputs) are stored.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from tests.golden.ref_cases import CASES, build_case  # noqa: E402


# Large outputs are stored on a regular sub-lattice (every SUB-th element per axis) plus
# full-array checksums, to keep fixtures small.
SUB = 4


def save_fixture(path, out):
    if out.size > 200_000:
        sub = out[::SUB, ::SUB, ::SUB]
        np.savez_compressed(path, output_sub=sub, sub=SUB, shape=np.array(out.shape),
                            sum=np.float64(out.sum(dtype=np.float64)),
                            sumsq=np.float64(np.square(out, dtype=np.float64).sum()))
    else:
        np.savez_compressed(path, output=out)


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    if O.reflib() is None:
        raise SystemExit("oracle/_ref/libfastcone_ref.so is missing")
    for name in CASES:
        pb, proj, vol, kind, mode = build_case(name)
        if kind == "bp":
            out = O.reflib_backproject(pb, proj, kernel_mode=mode)
        else:
            out = O.reflib_project(pb, vol)
        save_fixture(os.path.join(outdir, f"refgpu_{name}.npz"), out)
        print(name, out.shape, float(np.abs(out).max()))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
