"""CPU checks of the solve oracle (oracle/solve.py): the restated BiCGStab(l)
and refinement loop against a dense direct solve of the LippmannSchwinger
matrix (examples/GilaOperators.jl:89-95) on tiny volumes, and the shadow
generator against the published splitmix64 output."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.matvec import OprMem
from oracle.solve import (GOLDEN, bicgstabl, dense_ls, ls_apply, reliable_solve, shadow,
                          splitmix64_mix)
from oracle.synth import seeded_current, synth_operator


def _slab_chi(cel, lo, hi, val):
    chi = np.zeros(cel, dtype=np.complex128, order="F")
    chi[:, :, lo:hi] = val
    return chi


@pytest.fixture(scope="module")
def tiny():
    cel = (4, 4, 4)
    mix, fur, *_ = synth_operator(cel, ("1/32", "1/32", "1/32"))
    mem = OprMem(mix, fur)
    chi = _slab_chi(cel, 1, 3, 3.0 + 0.1j)
    A = dense_ls(mem, chi)
    return mem, chi, A


def test_splitmix64_known_answer():
    # splitmix64 from state 0: the first output is 0xE220A8397B1DCDAF
    assert int(splitmix64_mix(np.uint64(GOLDEN))) == 0xE220A8397B1DCDAF


def test_shadow_distribution():
    s = shadow(4096)
    assert s.shape == (4096,)
    for part in (s.real, s.imag):
        assert part.min() >= 0.0 and part.max() < 1.0
        assert abs(part.mean() - 0.5) < 0.03
    assert np.array_equal(s, shadow(4096))


def test_dense_matches_apply(tiny):
    mem, chi, A = tiny
    x = np.reshape(seeded_current(mem.mix.src_cel, 3), -1, order="F")
    assert np.linalg.norm(A @ x - ls_apply(mem, chi, x)) < 1e-13 * np.linalg.norm(A @ x)


@pytest.mark.parametrize("ell", [1, 2, 4])
def test_bicgstabl_vs_direct(tiny, ell):
    mem, chi, A = tiny
    b = np.reshape(seeded_current(mem.mix.src_cel, 11), -1, order="F")
    x_ref = np.linalg.solve(A, b)
    x, info = bicgstabl(lambda v: A @ v, b, ell=ell, reltol=1e-10, max_mv=2000)
    assert info["nrm"] <= 1e-10 * np.linalg.norm(b)
    # the recursively updated residual tracks the true residual
    assert np.linalg.norm(b - A @ x) <= 2e-10 * np.linalg.norm(b)
    assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)


def test_reliable_plain_and_low_precision_inner(tiny):
    mem, chi, A = tiny
    b = np.reshape(seeded_current(mem.mix.src_cel, 12), -1, order="F")
    x_ref = np.linalg.solve(A, b)
    x, info = reliable_solve(lambda v: A @ v, b, tol=1e-6)
    assert info["rel_res"] <= 1e-6 and info["updates"] == 1 and info["restarts"] == 1
    assert np.linalg.norm(x - x_ref) <= 1e-4 * np.linalg.norm(x_ref)
    # the plain solve is BiCGStab(l) on b / |b| followed by one FP64 residual
    xb, ib = bicgstabl(lambda v: A @ v, b / np.linalg.norm(b), reltol=0.9e-6)
    assert ib["iters"] == info["iters"]
    assert np.linalg.norm(np.linalg.norm(b) * xb - x) <= 1e-13 * np.linalg.norm(x)
    # single-precision inner operator: reliable updates still reach 1e-10
    A32 = A.astype(np.complex64)

    def inner(v):
        return (A32 @ v.astype(np.complex64)).astype(np.complex128)

    x2, info2 = reliable_solve(lambda v: A @ v, b, tol=1e-10, inner_apply=inner)
    assert info2["rel_res"] <= 1e-10 and info2["updates"] >= 2
    assert np.linalg.norm(x2 - x_ref) <= 1e-7 * np.linalg.norm(x_ref)


def test_identity_medium(tiny):
    mem, _, _ = tiny
    chi = np.zeros(mem.mix.src_cel, dtype=np.complex128)
    b = np.reshape(seeded_current(mem.mix.src_cel, 13), -1, order="F")
    x, info = reliable_solve(lambda v: ls_apply(mem, chi, v), b, tol=1e-6)
    assert np.linalg.norm(x - b) <= 1e-13 * np.linalg.norm(b)
    assert info["iters"] == 1
