"""Generate the golden matvec fixtures in this directory from the CPU oracle.

    python tests/golden/make_golden.py

Each fixture holds a seeded synthetic Fourier kernel in the reference's egoFur
layout (8 branches (tx,ty,tz,6,1,1)), a seeded source current and the FP64
oracle's egoOpr! output (8-branch recursion restating src/glaAct.jl:63-183).
The reference itself (Julia) cannot run on this image, so these vectors pin
the library to the oracle, not to the Julia package.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.matvec import OprMem, ego_opr  # noqa: E402
from oracle.synth import seeded_current, synth_operator  # noqa: E402

CASES = {
    "self_4x4x4": ((4, 4, 4), None, (0, 0, 0), None),
    "self_5x3x6": ((5, 3, 6), None, (0, 0, 0), None),
    "ext_4x4x2_from_6x4x4": ((4, 4, 2), (6, 4, 4), ("9/32", 0, 0), (0, 0, 0)),
}


def main():
    for name, (tc, sc, to, so) in CASES.items():
        mix, fur, _, is_self, trg, src = synth_operator(tc, ("1/32", "1/32", "1/32"), to, sc, so)
        x = seeded_current(mix.src_cel, 2024)
        y = ego_opr(OprMem(mix, fur), x)
        arrs = {f"fur{e}": fur[e] for e in range(8)}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), x=x, y=y,
                            trg_cel=np.array(trg.cel), src_cel=np.array(src.cel),
                            trg_org=np.array([str(o) for o in trg.org]), src_org=np.array([str(o) for o in src.org]),
                            is_self=np.array(is_self), **arrs)
        print(name, y.shape)


if __name__ == "__main__":
    main()
