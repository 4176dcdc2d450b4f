"""Analytic checks of the Green operator's physics: the point-dipole field,
passivity and reciprocity of the dense operator, and the Galerkin cell-pair
blocks by direct quadrature.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

The reference ships these checks as print-only scripts that its test runner
leaves commented out (test/runtests.jl:103-113):
  * test/anaTest.jl:10-106   the field of a unit dipole from egoOpr! against
                             the analytic dyadic Green function, outside a
                             window of 4 cell widths around the dipole;
  * test/posDefTest.jl:10-29 the smallest eigenvalue of the anti-Hermitian
                             part of the dense operator, "greater than
                             -1.0e-6 is considered normal";
  * test/intConTest.jl:6-35  wekS / wekE / wekV at intOrd and intOrd + 8
                             agreeing to 1e-8 (kerbuild.weak / the GPU
                             entry point do the evaluation).
The functions here restate the arithmetic of the first two so that the tests
can assert on it.  The dipole check leaves out the cells within two of the
dipole; the cell-pair blocks (below) check those near-field entries too.
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np

SEP_TOL = 1.0e-9   # test/anaTest.jl:5
LOW_TOL = 1.0e-12  # test/anaTest.jl:6


def cell_centres(cel, scl, org=(0, 0, 0)):
    """GlaVol.grd (src/glaMem.jl:144-145): per axis the cell-centre
    coordinates org - brd : scl : org + brd, brd = scl*(floor(cel/2) -
    iseven(cel)/2), in wavelengths."""
    out = []
    for c, s, o in zip(cel, scl, org):
        s, o = Fraction(s), Fraction(o)
        brd = s * (Fraction(c // 2) - Fraction(1 if c % 2 == 0 else 0, 2))
        out.append(np.array([float(o - brd + k * s) for k in range(c)]))
    return out


def ego_ana(cel, scl, org, dip_pos, dip_vec) -> np.ndarray:
    """egoAna! (test/anaTest.jl:10-52): the analytic field at every cell
    centre of a point dipole dip_vec at dip_pos, as an (Nx, Ny, Nz, 3) array.
    With s = 2 pi |r| (wavelength 1) and unit vector r^:
        G(r) = 2 pi^2 e^{i s} / s [ (1 + (i s - 1)/s^2) I
                                    - (1 + 3 (i s - 1)/s^2) r^ r^ ],
    and i 4 pi^2/3 I (the limit of the imaginary part) where s < 1e-9."""
    grd = cell_centres(cel, scl, org)
    X, Y, Z = np.meshgrid(*grd, indexing="ij")
    d = (X - dip_pos[0], Y - dip_pos[1], Z - dip_pos[2])
    sep = 2.0 * math.pi * np.sqrt(d[0] ** 2 + d[1] ** 2 + d[2] ** 2)
    small = sep < SEP_TOL
    sp = np.where(small, 1.0, sep)
    sh = [2.0 * math.pi * di / sp for di in d]
    pre = 2.0 * math.pi ** 2 * np.exp(1j * sp) / sp
    a = 1.0 + (1j * sp - 1.0) / sp ** 2
    b = 1.0 + 3.0 * (1j * sp - 1.0) / sp ** 2
    out = np.zeros((*cel, 3), dtype=np.complex128)
    for i in range(3):
        acc = np.zeros(cel, dtype=np.complex128)
        for j in range(3):
            g = pre * ((a if i == j else 0.0) - b * sh[i] * sh[j])
            g = np.where(small, (2.0 * math.pi ** 2 * 2.0j / 3.0) * (1.0 if i == j else 0.0), g)
            acc = acc + g * dip_vec[j]
        out[..., i] = acc
    return out


def dipole_source(cel, scl, direction: int):
    """The source of test/anaTest.jl:68-84: one cell at index div(N, 2)
    (1-based; the reference uses cel[1] for every axis) carrying the current
    1/prod(scl) along `direction`.  Returns (x, loc0, dip_pos, dip_vec) with
    loc0 the 0-based cell index and dip_pos its centre."""
    n = cel[0] // 2
    loc = (n - 1, n - 1, n - 1)
    grd = cell_centres(cel, scl)
    pos = tuple(grd[k][loc[k]] for k in range(3))
    vec = np.zeros(3, dtype=np.complex128)
    vec[direction] = 1.0
    x = np.zeros((*cel, 3), dtype=np.complex128, order="F")
    x[loc[0], loc[1], loc[2], direction] = 1.0 / float(np.prod([Fraction(s) for s in scl]))
    return x, loc, pos, vec


def window_cells(scl, cel) -> int:
    """winInt of test/anaTest.jl:60-67: half-width, in cells, of the window
    of 4 minimum cell widths removed around the dipole."""
    m = min(Fraction(s) for s in scl)
    return min(int((Fraction(1, 2) * 4 * m) // m), min(cel))


def dipole_errors(num, ana, loc, win):
    """difMat of test/anaTest.jl:90-101: per element min(|a - n|,
    |a - n| / max(|n|, 1e-12)), zeroed in the window around the dipole.
    Returns (maximum, relative L2 of ana - num outside the window)."""
    diff = np.abs(ana - num)
    dm = np.minimum(diff, diff / np.maximum(np.abs(num), LOW_TOL))
    sl = tuple(slice(l - win, l + win + 1) for l in loc)
    dm[sl] = 0.0
    mask = np.ones(num.shape, dtype=bool)
    mask[sl] = False
    rl2 = float(np.linalg.norm((ana - num)[mask]) / np.linalg.norm(ana[mask]))
    return float(dm.max()), rl2


def anti_hermitian_eigs(M: np.ndarray, frq: complex = 1.0 + 0j) -> np.ndarray:
    """Eigenvalues of egoDenMatAsm (test/posDefTest.jl:22-27):
    (i/2) conj(f^2) M^H - (i/2) f^2 M, a Hermitian matrix."""
    asm = 0.5j * np.conj(frq ** 2) * M.conj().T - 0.5j * frq ** 2 * M
    return np.linalg.eigvalsh(0.5 * (asm + asm.conj().T))


# --------------------------------------------------------- cell-pair blocks
# The operator's 3x3 block between a source cell and a target cell is the
# Galerkin integral (1/V) int_target int_source G(r - r') dr' dr of the
# dipole field G above (a unit current in the source cell; the dipole test
# feeds 1/V).  Its imaginary part is an entire function of r - r',
#     Im G(r) = 2 pi^2 [ (2 j0(s) - j2(s)) / 3 I + j2(s) r^ r^ ],  s = 2 pi |r|,
# so a tensor Gauss-Legendre rule over both cubes converges to rounding for
# every pair, touching and self pairs included; the real part,
#     Re G(r) = 2 pi^2 [ (y2(s) - 2 y0(s)) / 3 I - y2(s) r^ r^ ],
# is smooth only for cells that do not touch.  (j, y: spherical Bessel
# functions; the two forms restate the bracket of egoAna! split into
# e^{is}/s terms.)

def green_part(d: np.ndarray, part: str) -> np.ndarray:
    """Re or Im of G at separations d[..., 3] (wavelengths): [..., 3, 3]."""
    from scipy.special import spherical_jn, spherical_yn
    r = np.sqrt((d ** 2).sum(-1))
    s = 2.0 * math.pi * r
    out = np.zeros(d.shape[:-1] + (3, 3))
    if part == "im":
        j0 = spherical_jn(0, s)
        small = s < 1e-3
        ss = np.where(small, 1.0, s)
        j2s2 = np.where(small, 1.0 / 15.0 - s ** 2 / 210.0, spherical_jn(2, ss) / ss ** 2)  # j2(s) / s^2
        iso = (2.0 * j0 - j2s2 * s ** 2) / 3.0
        for i in range(3):
            for j in range(3):
                out[..., i, j] = 2.0 * math.pi ** 2 * (iso * (i == j) + j2s2 * (2.0 * math.pi) ** 2 * d[..., i] * d[..., j])
        return out
    y0 = spherical_yn(0, s)
    y2 = spherical_yn(2, s)
    for i in range(3):
        for j in range(3):
            out[..., i, j] = 2.0 * math.pi ** 2 * ((y2 - 2.0 * y0) / 3.0 * (i == j) - y2 * d[..., i] * d[..., j] / r ** 2)
    return out


def cell_pair_block(off, h: float, part: str, n: int = 8) -> np.ndarray:
    """(1/V) int int of Re or Im G over two cubes of side h whose centres are
    off * h apart (target minus source), by an n-point Gauss-Legendre rule
    per coordinate (n^6 point pairs)."""
    x, w = np.polynomial.legendre.leggauss(n)
    x = x * h / 2.0
    w = w * h / 2.0
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    W = (w[:, None, None] * w[None, :, None] * w[None, None, :]).ravel()
    P = np.stack([X.ravel(), Y.ravel(), Z.ravel()], -1)
    d = (np.asarray(off, dtype=float) * h)[None, None, :] + P[:, None, :] - P[None, :, :]
    return np.einsum("a,b,abij->ij", W, W, green_part(d, part)) / h ** 3


# (target - source) cell offsets of the near-field check: self, face, edge
# and vertex contact, and non-touching pairs
NEAR_OFFSETS = [(0, 0, 0), (1, 0, 0), (0, 1, 1), (1, 1, 1), (2, 0, 0), (2, 1, 0), (0, 2, 2), (3, 1, 0), (2, -1, 1)]


def operator_blocks(apply, cel, src_cell, offsets):
    """3x3 blocks of the operator between src_cell and src_cell + off, from
    three matvecs with unit currents (one per component)."""
    cols = []
    for j in range(3):
        x = np.zeros((*cel, 3), dtype=np.complex128, order="F")
        x[tuple(src_cell) + (j,)] = 1.0
        cols.append(np.asarray(apply(x)))
    out = {}
    for off in offsets:
        t = tuple(a + b for a, b in zip(src_cell, off))
        out[off] = np.array([[cols[j][t + (i,)] for j in range(3)] for i in range(3)])
    return out
