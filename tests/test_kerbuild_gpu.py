"""GPU FP64 kernel build (GlaOprMem without egoFur) against the C
restatement of the reference's build (oracle/gen.c), through the C ABI.

The adaptive cubature takes the same decisions on both sides except in rare
borderline cases (FP64 rounding of the error estimate), so the stored kernel
must agree to far better than the cubature tolerance (reltol 1e-6); the
tests ask for 1e-9 relative to the largest stored value.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import TOL_F64, load_pkg, rel_l2
from oracle import kerbuild as kb
from oracle.matvec import OprMem, ego_opr
from oracle.synth import seeded_current

pytestmark = pytest.mark.gpu


def _opt(gila, ord_):
    return gila.GlaKerOpt(1.0 + 0j, ord_, False, True, (), ())


CASES = [
    # (trg_cel, scl, trg_org, src_cel, src_org, intOrd)
    ((4, 5, 6), ("1/32", "1/32", "1/32"), (0, 0, 0), None, None, 8),
    ((8, 8, 8), ("1/32", "1/32", "1/32"), (0, 0, 0), None, None, 16),
    ((3, 2, 1), ("1/20", "1/25", "1/30"), (0, 0, 0), None, None, 8),
    ((4, 4, 4), ("1/50", "1/50", "1/50"), (0, "2/50", 0), (4, 4, 4), (0, "-2/50", 0), 8),
    ((4, 4, 2), ("1/32", "1/32", "1/32"), ("9/32", 0, 0), (6, 4, 4), (0, 0, 0), 8),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}<-{c[3]}@{c[1][0]}")
def test_gpu_kernel_build_matches_oracle(case):
    gila = load_pkg()
    tc, scl, to, sc, so, ord_ = case
    mix, fur_ref, _, is_self, trg, src = kb.build_operator(tc, scl, to, sc, so, int_ord=ord_)
    tv = gila.GlaVol(trg.cel, trg.scl, trg.org)
    sv = None if is_self else gila.GlaVol(src.cel, src.scl, src.org)
    mem = gila.GlaOprMem(_opt(gila, ord_), tv, sv, setTyp=np.complex128)
    fur = mem.egoFur
    scale = max(np.abs(f).max() for f in fur_ref)
    err = max(np.abs(a - b).max() for a, b in zip(fur, fur_ref)) / scale
    assert err < 1e-9, err
    x = seeded_current(mix.src_cel, 4)
    y = gila.egoOpr(mem, np.asfortranarray(x))
    assert rel_l2(y, ego_opr(OprMem(mix, fur_ref), x)) < 1e-9


def test_gpu_built_self_external_identity():
    """test/extSlfTest.jl:44-47 with kernels built on the GPU."""
    gila = load_pkg()
    scl = ("1/50", "1/50", "1/50")
    opt = _opt(gila, 8)
    memU = gila.GlaOprMem(opt, gila.GlaVol((4, 8, 4), scl))
    memE = gila.GlaOprMem(opt, gila.GlaVol((4, 4, 4), scl, (0, "2/50", 0)), gila.GlaVol((4, 4, 4), scl, (0, "-2/50", 0)))
    xA = seeded_current((4, 4, 4), 8)
    xU = np.zeros((4, 8, 4, 3), dtype=np.complex128, order="F")
    xU[:, :4] = xA
    yU = gila.egoOpr(memU, xU)
    yE = gila.egoOpr(memE, np.asfortranarray(xA))
    assert rel_l2(yE, yU[:, 4:]) < 1e-12


def test_gpu_build_complex64_and_overlap_error():
    gila = load_pkg()
    scl = ("1/32", "1/32", "1/32")
    m64 = gila.GlaOprMem(_opt(gila, 8), gila.GlaVol((4, 4, 4), scl), setTyp=np.complex128)
    m32 = gila.GlaOprMem(_opt(gila, 8), gila.GlaVol((4, 4, 4), scl), setTyp=np.complex64)
    for a, b in zip(m64.egoFur, m32.egoFur):
        assert np.abs(a.astype(np.complex64) - b).max() == 0  # cast of the same FP64 build
    with pytest.raises(gila.GilaError, match="overlapping"):
        gila.GlaOprMem(_opt(gila, 8), gila.GlaVol((4, 4, 4), scl, ("1/32", 0, 0)), gila.GlaVol((4, 4, 4), scl))
