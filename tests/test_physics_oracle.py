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
    1e-8.
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
