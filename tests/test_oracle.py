"""CPU tests of the oracle and of the host-side logic (no GPU).

The oracle restates the reference's host matvec (egoBrnHst!).  With no golden
vectors in the reference and no Julia on this image, it is pinned by
agreement of three independent formulations and by the reference's own
relational test (test/extSlfTest.jl:44-47), and the committed fixtures under
tests/golden pin it against later edits.
"""
from __future__ import annotations

import glob
import os
from fractions import Fraction

import numpy as np
import pytest

from conftest import ROOT, load_pkg, rel_l2
from oracle.fur import direct_apply, fur_to_full, padfft_apply
from oracle.gla_mem import ExtInf, Vol, mix_for, tru_inf, vol_even
from oracle.matvec import OprMem, ego_opr
from oracle.synth import seeded_current, synth_operator

SCL = ("1/32", "1/32", "1/32")
SHAPES = [
    ((4, 4, 4), None, (0, 0, 0), None),
    ((5, 3, 6), None, (0, 0, 0), None),
    ((2, 2, 2), None, (0, 0, 0), None),
    ((1, 3, 2), None, (0, 0, 0), None),
    ((3, 5, 7), None, (0, 0, 0), None),
    ((4, 4, 4), (4, 4, 4), (0, "4/32", 0), (0, 0, 0)),
    ((4, 4, 2), (6, 4, 4), ("9/32", 0, 0), (0, 0, 0)),
    ((3, 4, 5), (5, 4, 3), ("1/2", "1/3", "1/4"), (0, 0, 0)),
]


@pytest.mark.parametrize("case", SHAPES, ids=lambda c: f"{c[0]}<-{c[1]}")
def test_three_formulations_agree(case):
    tc, sc, to, so = case
    mix, fur, crc, _, _, _ = synth_operator(tc, SCL, to, sc, so)
    x = seeded_current(mix.src_cel, 1)
    y_branch = ego_opr(OprMem(mix, fur), x)
    y_pad = padfft_apply(mix, fur_to_full(mix, fur), x)[..., 0]
    y_dir = direct_apply(crc, mix.src_cel, mix.trg_cel, x)
    assert rel_l2(y_branch, y_pad) < 1e-13
    assert rel_l2(y_branch, y_dir) < 1e-13


def test_self_external_identity_oracle():
    """test/extSlfTest.jl:44-47 on the oracle."""
    celA = (6, 6, 4)
    celU = (6, 12, 4)
    scl = ("1/50", "1/50", "1/50")
    mixU, furU, _, _, _, _ = synth_operator(celU, scl, (0, 0, 0))
    mixE, furE, _, _, _, _ = synth_operator(celA, scl, (0, "3/50", 0), celA, (0, "-3/50", 0))
    xA = seeded_current(celA, 9)
    xU = np.zeros((*celU, 3), dtype=np.complex128)
    xU[:, :6] = xA
    yU = ego_opr(OprMem(mixU, furU), xU)
    yE = ego_opr(OprMem(mixE, furE), xA)
    assert rel_l2(yE, yU[:, 6:]) < 1e-13


def test_golden_fixtures_reproduce():
    files = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
    assert files
    for f in files:
        d = np.load(f)
        trg = Vol.make(tuple(d["trg_cel"]), SCL, tuple(Fraction(s) for s in d["trg_org"]))
        src = Vol.make(tuple(d["src_cel"]), SCL, tuple(Fraction(s) for s in d["src_org"]))
        _, _, mix, _ = mix_for(trg, None if bool(d["is_self"]) else src)
        fur = [d[f"fur{e}"] for e in range(8)]
        y = ego_opr(OprMem(mix, fur), d["x"])
        assert rel_l2(y, d["y"]) < 1e-14, f


def test_volume_rules():
    """glaVolEveGen and GlaExtInf (src/glaMem.jl:152-216)."""
    v = Vol.make((3, 4, 5), ("1/10", "1/10", "1/10"))
    e = vol_even(v)
    assert e.cel == (4, 4, 6)
    assert e.scl[0] == Fraction(3, 40) and e.scl[2] == Fraction(5, 60)
    fine = Vol.make((8, 8, 8), ("1/50", "1/50", "1/50"))
    coarse = Vol.make((4, 4, 4), ("1/25", "1/25", "1/25"), ("1", 0, 0))
    m = ExtInf.make(fine, coarse)  # target fine, source coarse
    assert m.trg_div == (2, 2, 2) and m.src_div == (1, 1, 1)
    assert m.trg_cel == (4, 4, 4) and m.src_cel == (4, 4, 4)
    with pytest.raises(ValueError):
        ExtInf.make(fine, Vol.make((4, 4, 4), ("1/30", "1/30", "1/30")))
    # partial (symmetric) storage only along axes with equal cells and centres
    t = Vol.make((4, 6, 4), SCL, (0, "1/2", 0))
    s = Vol.make((4, 6, 4), SCL, (0, 0, 0))
    _, _, mx, _ = mix_for(t, s)
    assert tru_inf(t, s, mx) == (3, 6, 3)


def test_python_mirror_host_logic():
    gila = load_pkg()
    v = gila.GlaVol((4, 4, 4), ("1/32", "1/32", "1/32"))
    assert v.scl[0] == Fraction(1, 32)
    o = gila.GlaKerOpt(True)
    assert o.intOrd == 32 and o.numTrd == (128, 2, 1) and o.numBlk == (1, 128, 256)
    # GlaOpr with a non-complex setTyp raises ArgumentError (test/oprTest.jl:4-5)
    with pytest.raises(gila.ArgumentError):
        gila.GlaOpr((1, 1, 1), ("1", "1", "1"), (0, 0, 0), setTyp=np.float64)


def test_kernel_build_oracle_relations():
    """C restatement of the kernel build (oracle/gen.c): the reference's
    self-vs-external identity (test/extSlfTest.jl:44-47) with real kernels
    (B touches A: the contact path of genEgoCrcExt!), symmetry of the 3x3
    blocks, and Gauss-Legendre nodes."""
    import numpy.polynomial.legendre as npl
    from oracle import kerbuild as kb
    x, w = kb.gauleg(32)
    xr, wr = npl.leggauss(32)
    assert np.abs(x - xr).max() < 1e-15 and np.abs(w - wr).max() < 1e-14
    scl = ("1/50", "1/50", "1/50")
    weak = kb.weak(scl, int_ord=8)
    mixU, furU, crcU, _, _, _ = kb.build_operator((4, 8, 4), scl, int_ord=8, weak_vals=weak)
    mixE, furE, _, is_self, _, _ = kb.build_operator((4, 4, 4), scl, (0, "2/50", 0), (4, 4, 4), (0, "-2/50", 0),
                                                     int_ord=8)
    assert not is_self
    xA = seeded_current((4, 4, 4), 3)
    xU = np.zeros((4, 8, 4, 3), dtype=np.complex128)
    xU[:, :4] = xA
    yU = ego_opr(OprMem(mixU, furU), xU)
    yE = ego_opr(OprMem(mixE, furE), xA)
    assert rel_l2(yE, yU[:, 4:]) < 1e-12
    assert np.abs(crcU[0, 1] - crcU[1, 0]).max() < 1e-12 * np.abs(crcU[0, 1]).max()


def test_threaded_host_path_matches_sequential():
    """The timed CPU baseline runs the restatement with scipy.fft workers and
    the recursion's branches on threads (as egoBrnHst! spawns them); the
    values must be those of the sequential restatement."""
    import oracle.matvec as om
    from oracle.synth import seeded_current, synth_operator
    mix, fur, _, _, _, _ = synth_operator((10, 8, 6), ("1/32", "1/32", "1/32"))
    mem = om.OprMem(mix, fur)
    x = seeded_current(mix.src_cel, 3)
    seq = om.ego_opr(mem, x)
    saved = (om._fft, om._ifft, om._parallel)
    try:
        om.use_fft_workers(4)
        par = om.ego_opr(mem, x)
    finally:
        om._fft, om._ifft, om._parallel = saved
    assert np.allclose(par, seq, rtol=0, atol=1e-13 * np.abs(seq).max())
