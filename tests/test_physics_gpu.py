"""Physics pins of the GPU kernel build and matvec, at the default intOrd 32.

Operators are built on the GPU (GlaOprMem without egoFur) and applied through
the C ABI.  The checks are the reference's disabled physics scripts with
assertions (see tests/test_physics_oracle.py for the same checks on the CPU
oracle), plus the exact 32^3 workload end to end against the oracle:
  * test/anaTest.jl:10-106   dipole field vs the analytic Green function;
  * test/posDefTest.jl:10-29 passivity (and reciprocity) of the dense operator;
  * test/intConTest.jl:6-35  wekS / wekE / wekV converged at intOrd 32;
  * the near-field blocks (self and contact pairs included) against direct
    quadrature of the analytic Green function;
  * the 32^3 self operator of 1/32-wavelength cells: GPU build vs the C
    oracle's build, and its matvec on a seeded current vs the oracle's
    matvec, in ComplexF64 and ComplexF32.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import TOL_F32, TOL_F64, load_pkg, rel_l2
from oracle import analytic as an
from oracle import kerbuild as kb
from oracle.matvec import OprMem, ego_opr
from oracle.synth import seeded_current
from test_physics_oracle import assert_near_field, dipole_check, near_field_check

pytestmark = pytest.mark.gpu


def _build(gila, cel, scl, dtype=np.complex128, ord_=32):
    opt = gila.GlaKerOpt(1.0 + 0j, ord_, False, True, (), ())
    return gila.GlaOprMem(opt, gila.GlaVol(cel, scl), setTyp=dtype)


@pytest.mark.parametrize("cel,scl,max_err,max_l2", [
    ((16, 16, 16), ("1/50",) * 3, 0.036, 0.003),   # the reference's test volume
    ((32, 32, 32), ("1/32",) * 3, 0.012, 0.004),   # the 32^3 workload's volume
])
def test_gpu_dipole_field_matches_analytic(cel, scl, max_err, max_l2):
    gila = load_pkg()
    mem = _build(gila, cel, scl)
    errs = dipole_check(lambda x: gila.egoOpr(mem, x), cel, scl)
    mx = [e[0] for e in errs]
    assert max(mx) < max_err, errs
    assert max(e[1] for e in errs) < max_l2, errs
    assert max(mx) - min(mx) < 1e-9 * max(mx), errs


@pytest.mark.parametrize("cel,scl", [((6, 6, 6), ("1/32",) * 3), ((8, 8, 8), ("1/50",) * 3),
                                     ((4, 6, 5), ("1/20", "1/25", "1/30"))])
def test_gpu_passivity_and_reciprocity(cel, scl):
    """The dense operator, one column per unit source (test/posDefTest.jl:
    10-21), as one batched apply of 3V vectors."""
    gila = load_pkg()
    mem = _build(gila, cel, scl)
    n = 3 * int(np.prod(cel))
    eye = np.asfortranarray(np.eye(n, dtype=np.complex128).reshape((*cel, 3, n), order="F"))
    out = np.zeros_like(eye, order="F")
    mem.apply_into(eye, out, nrhs=n)
    M = out.reshape((n, n), order="F")
    ev = an.anti_hermitian_eigs(M)
    assert ev.min() > -1e-6, ev.min()
    assert ev.max() > 1e-3
    assert np.linalg.norm(M - M.T) <= 1e-12 * np.linalg.norm(M)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_gpu_near_field_blocks_match_quadrature(dtype):
    """GPU build and GPU matvec.  In ComplexF32 the imaginary part (about
    1/800 of the self block's real part) is held to FP32 rounding of the
    largest entry, 2e-6 of it, and the far real part to the quadrature's
    5e-5."""
    gila = load_pkg()
    mem = _build(gila, (8, 8, 8), ("1/32",) * 3, dtype)
    rel, absl = near_field_check(lambda x: gila.egoOpr(mem, np.asfortranarray(x.astype(dtype))))
    if dtype == np.complex128:
        assert_near_field(rel)
    else:
        for off in rel:
            assert absl[off][0] < 2e-6, (off, absl[off])
            assert rel[off][1] is None or rel[off][1] < 5e-5, (off, rel[off])


def test_gpu_weak_integrals_converge_and_match_oracle():
    gila = load_pkg()
    for scl in [("1/50",) * 3, ("1/32",) * 3, ("1/20", "1/25", "1/30")]:
        a = gila.weak_integrals(scl, 1.0, 32)
        b = gila.weak_integrals(scl, 1.0, 40)
        for x, y in zip(a, b):
            assert np.max(np.abs(x - y) / np.abs(y)) < 1e-8, scl
    ref = kb.weak(("1/50",) * 3, int_ord=32)
    got = gila.weak_integrals(("1/50",) * 3, 1.0, 32)
    for x, y in zip(got, ref):
        assert np.max(np.abs(x - y) / np.abs(y)) < 1e-12


def test_gpu_32cube_workload_end_to_end():
    """The 32^3 self operator at 1/32 wavelength, intOrd 32: the GPU build
    against the C oracle's build (same cubature decisions: agreement far
    below the cubature tolerance), then the matvec of a seeded N(0,1) current
    on each side."""
    gila = load_pkg()
    cel, scl = (32, 32, 32), ("1/32",) * 3
    mix, fur_ref, _, _, _, _ = kb.build_operator(cel, scl, int_ord=32)
    mem = _build(gila, cel, scl)
    fur = mem.egoFur
    scale = max(np.abs(f).max() for f in fur_ref)
    err = max(np.abs(a - b).max() for a, b in zip(fur, fur_ref)) / scale
    assert err < 1e-9, err
    x = seeded_current(cel, 32)
    want = ego_opr(OprMem(mix, fur_ref), x)
    # the GPU matvec on the oracle's own kernel: rounding only
    mem_ref = gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(cel, scl), egoFur=fur_ref, setTyp=np.complex128)
    assert rel_l2(gila.egoOpr(mem_ref, np.asfortranarray(x)), want) <= TOL_F64
    # GPU build + GPU matvec end to end
    assert rel_l2(gila.egoOpr(mem, np.asfortranarray(x)), want) <= max(TOL_F64, 10 * err)
    # ComplexF32: the same FP64 build cast, FP32 FFT / multiply / accumulate
    mem32 = _build(gila, cel, scl, np.complex64)
    y32 = gila.egoOpr(mem32, np.asfortranarray(x.astype(np.complex64)))
    assert rel_l2(y32, want) <= TOL_F32
