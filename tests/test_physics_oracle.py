"""Physics pins of the CPU oracle's kernel build and matvec (no GPU).

The reference's only absolute checks of its operator are three print-only
scripts (test/anaTest.jl, test/posDefTest.jl, test/intConTest.jl) that its
runner leaves disabled; they are ported here with assertions, on the
reference's own test volume (16^3 cells of 1/50 wavelength, intOrd 32).  They
pin the oracle -- which every GPU parity test compares against -- to the
physics rather than to a second restatement of the same code:
  * dipole: the field of a unit dipole matches the analytic dyadic Green
    function outside the 5x5x5-cell window to 3.6% (maximum of the
    reference's error measure) and 0.3% relative L2; the three orientations
    give the same error (cubic symmetry);
  * passivity: the anti-Hermitian part of the dense operator has no
    eigenvalue below -1e-6, and the operator is reciprocal (M = M^T);
  * quadrature convergence: wekS / wekE / wekV at intOrd 32 and 40 agree to
    1e-8;
  * near field: the operator's 3x3 blocks between a cell and its neighbours
    (self, face, edge and vertex contact, and non-touching pairs) against
    the Galerkin double integral of the analytic Green function by direct
    Gauss-Legendre quadrature -- the imaginary part, smooth everywhere, to
    1e-10 for every pair; the real part, singular at contact, to 5e-5 for
    the non-touching pairs (the weak-form cubature's tolerance is 1e-6).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import analytic as an
from oracle import kerbuild as kb
from oracle.matvec import OprMem, ego_opr

REF_CEL = (16, 16, 16)
REF_SCL = ("1/50", "1/50", "1/50")


@pytest.fixture(scope="module")
def ref_operator():
    mix, fur, _, _, _, _ = kb.build_operator(REF_CEL, REF_SCL, int_ord=32)
    return OprMem(mix, fur)


def dipole_check(apply, cel, scl):
    """Per orientation (max error, relative L2) of test/anaTest.jl's measure."""
    win = an.window_cells(scl, cel)
    out = []
    for d in range(3):
        x, loc, pos, vec = an.dipole_source(cel, scl, d)
        num = apply(x)
        ana = an.ego_ana(cel, scl, (0, 0, 0), pos, vec)
        out.append(an.dipole_errors(num, ana, loc, win))
    return out


def test_oracle_dipole_field_matches_analytic(ref_operator):
    errs = dipole_check(lambda x: ego_opr(ref_operator, x), REF_CEL, REF_SCL)
    mx = [e[0] for e in errs]
    l2 = [e[1] for e in errs]
    assert max(mx) < 0.036, errs
    assert max(l2) < 0.003, errs
    assert max(mx) - min(mx) < 1e-10 * max(mx), errs


def test_oracle_passivity_and_reciprocity():
    cel = (4, 4, 4)
    mix, fur, _, _, _, _ = kb.build_operator(cel, REF_SCL, int_ord=32)
    mem = OprMem(mix, fur)
    n = 3 * int(np.prod(cel))
    M = np.zeros((n, n), dtype=np.complex128)
    for k in range(n):
        e = np.zeros(n, dtype=np.complex128)
        e[k] = 1.0
        M[:, k] = ego_opr(mem, e.reshape((*cel, 3), order="F")).reshape(-1, order="F")
    ev = an.anti_hermitian_eigs(M)
    assert ev.min() > -1e-6, ev.min()
    assert ev.max() > 1e-3  # the radiative part is not trivially zero
    assert np.linalg.norm(M - M.T) <= 1e-13 * np.linalg.norm(M)


def test_oracle_weak_integrals_converge():
    a = kb.weak(REF_SCL, int_ord=32)
    b = kb.weak(REF_SCL, int_ord=40)
    for x, y in zip(a, b):
        assert np.max(np.abs(x - y) / np.abs(y)) < 1e-8


NEAR_CEL = (8, 8, 8)
NEAR_SCL = ("1/32", "1/32", "1/32")
NEAR_SRC = (2, 3, 3)


def near_field_check(apply, cel=NEAR_CEL, scl=NEAR_SCL, src=NEAR_SRC):
    """Per cell offset (Im error, Re error or None for touching pairs), each
    relative to the largest entry of its quadrature block; and the same
    errors relative to the largest entry of all the blocks (the real part of
    the self block), the scale of a rounding error."""
    from fractions import Fraction
    h = float(Fraction(scl[0]))
    blocks = an.operator_blocks(apply, cel, src, an.NEAR_OFFSETS)
    scale = max(np.abs(b).max() for b in blocks.values())
    rel, absl = {}, {}
    for off, blk in blocks.items():
        qi = an.cell_pair_block(off, h, "im")
        di = np.abs(blk.imag - qi).max()
        dr = er = None
        if max(abs(o) for o in off) >= 2:
            qr = an.cell_pair_block(off, h, "re")
            dr = np.abs(blk.real - qr).max()
            er = dr / np.abs(qr).max()
        rel[off] = (di / np.abs(qi).max(), er)
        absl[off] = (di / scale, None if dr is None else dr / scale)
    return rel, absl


def assert_near_field(errs):
    for off, (ei, er) in errs.items():
        assert ei < 1e-10, (off, ei)
        assert er is None or er < 5e-5, (off, er)
    assert sum(er is not None for _, er in errs.values()) >= 4


def test_quadrature_blocks_converged():
    h = 1.0 / 32
    for off in [(0, 0, 0), (1, 1, 0)]:
        a, b = an.cell_pair_block(off, h, "im", 6), an.cell_pair_block(off, h, "im", 8)
        assert np.abs(a - b).max() < 1e-12 * np.abs(b).max()
    a, b = an.cell_pair_block((2, 1, 0), h, "re", 8), an.cell_pair_block((2, 1, 0), h, "re", 10)
    assert np.abs(a - b).max() < 1e-9 * np.abs(b).max()


def test_oracle_near_field_blocks_match_quadrature():
    mix, fur, _, _, _, _ = kb.build_operator(NEAR_CEL, NEAR_SCL, int_ord=32)
    mem = OprMem(mix, fur)
    assert_near_field(near_field_check(lambda x: ego_opr(mem, x))[0])
