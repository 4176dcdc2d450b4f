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


PART_CASES = [
    # (trg_cel, trg_scl, trg_org, src_cel): source at the origin, scale 1/32
    ((8, 8, 8), ("1/64", "1/64", "1/64"), ("12/32", 0, 0), (4, 4, 4)),   # 8 target partitions
    ((8, 4, 8), ("1/64", "1/32", "1/64"), (0, 0, "12/32"), (4, 4, 4)),   # 4, divided along x and z
]


@pytest.mark.parametrize("case", PART_CASES, ids=lambda c: f"{c[0]}@{c[1][0]}<-{c[3]}")
def test_gpu_partitioned_build_matches_oracle(case):
    """Mixed cell scales: the kernel of every target partition
    (src/glaMemSup.jl:60-88) built on the GPU against the oracle's loop over
    partition pairs, then the partitioned matvec on it."""
    gila = load_pkg()
    tc, tscl, to, sc = case
    scl = ("1/32", "1/32", "1/32")
    mix, fur_ref, _, is_self, trg, src = kb.build_operator(tc, tscl, to, sc, (0, 0, 0), int_ord=8, src_scl=scl)
    assert not is_self and np.prod(mix.trg_div) > 1 and fur_ref[0].shape[5] == np.prod(mix.trg_div)
    mem = gila.GlaOprMem(_opt(gila, 8), gila.GlaVol(trg.cel, trg.scl, trg.org), gila.GlaVol(src.cel, src.scl, src.org),
                         setTyp=np.complex128)
    fur = mem.egoFur
    assert all(a.shape == b.shape for a, b in zip(fur, fur_ref))
    scale = max(np.abs(f).max() for f in fur_ref)
    err = max(np.abs(a - b).max() for a, b in zip(fur, fur_ref)) / scale
    assert err < 1e-9, err
    x = seeded_current(mix.src_cel, 6)
    y = gila.egoOpr(mem, np.asfortranarray(x))
    assert rel_l2(y, ego_opr(OprMem(mix, fur_ref), x)) < 1e-9


def test_gpu_partitioned_build_errors():
    """A partitioned target touching the source: each partition's cells lie
    strictly inside the source's faces, which genEgoCrcExt! reports as an
    overlap (src/glaGen.jl:66-80) -- on both sides.  A source grid finer
    than the target (source partitions) is refused by the GPU build."""
    gila = load_pkg()
    scl = ("1/32", "1/32", "1/32")
    with pytest.raises(ValueError, match="overlapping"):
        kb.build_operator((8, 8, 8), ("1/64",) * 3, ("4/32", 0, 0), (4, 4, 4), (0, 0, 0), int_ord=8, src_scl=scl)
    with pytest.raises(gila.GilaError, match="overlapping"):
        gila.GlaOprMem(_opt(gila, 8), gila.GlaVol((8, 8, 8), ("1/64",) * 3, ("4/32", 0, 0)), gila.GlaVol((4, 4, 4), scl))
    with pytest.raises(gila.GilaError, match="source partitions"):
        gila.GlaOprMem(_opt(gila, 8), gila.GlaVol((4, 4, 4), scl, ("12/32", 0, 0)), gila.GlaVol((8, 8, 8), ("1/64",) * 3))
