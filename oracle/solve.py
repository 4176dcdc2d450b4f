"""Oracle restatement of the scattering solve (I - chi G) x = b.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

* LippmannSchwinger (examples/GilaOperators.jl:57-96): A x = x - chi .* (G x),
  chi per cell broadcast over the three components (:71, :94).
* solve (examples/scattering_film.jl:58-61) calls IterativeSolvers.bicgstabl
  (A, b): BiCGStab(l) of Sleijpen & Fokkema (1993), l = 2, zero initial
  guess, a random shadow residual, stopping when the recursively updated
  residual norm falls to reltol * |b| or the matvec budget is used.
  IterativeSolvers is not vendored or pinned by the reference (it appears in
  the examples only); ``bicgstabl`` below restates the published method.
* ``refine_solve`` is the FP64 iterative-refinement loop the GPU solver wraps
  around BiCGStab(l) (no reference counterpart: the reference solves in one
  precision); with FP64 inner solves it is the plain GPU solve step for step.

Vectors are flat in the reference's memory order: (Nx, Ny, Nz, 3) column-major.
"""
from __future__ import annotations

import numpy as np

from .matvec import OprMem, ego_opr

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
SHADOW_SEED = 0x5EED


def splitmix64_mix(z: np.ndarray) -> np.ndarray:
    """The output function of splitmix64 (Steele, Lea & Flood 2014)."""
    with np.errstate(over="ignore"):
        z = np.asarray(z, dtype=np.uint64)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def shadow(n: int, seed: int = SHADOW_SEED) -> np.ndarray:
    """The GPU solver's shadow residual: element i has real and imaginary
    parts uniform on [0, 1) (the distribution of IterativeSolvers' rand(T, n)),
    from splitmix64 steps 1 and 2 of the state seed + golden * (2 i + 1)."""
    i = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + GOLDEN * (np.uint64(2) * i + np.uint64(1))
        u = []
        for _ in range(2):
            z = z + GOLDEN
            u.append((splitmix64_mix(z) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0))
    return u[0] + 1j * u[1]


def ls_apply(mem: OprMem, chi: np.ndarray, x: np.ndarray) -> np.ndarray:
    """LippmannSchwinger * x (examples/GilaOperators.jl:89-95) on a flat vector."""
    cel = mem.mix.src_cel
    x4 = np.reshape(x, (*cel, 3), order="F")
    g = ego_opr(mem, x4)
    return np.reshape(x4 - chi[..., None] * g, -1, order="F")


def bicgstabl(apply, b: np.ndarray, ell: int = 2, reltol: float = np.sqrt(np.finfo(float).eps),
              max_mv: int | None = None, rs: np.ndarray | None = None):
    """BiCGStab(l) from a zero initial guess.  Returns (x, info) with info
    iters (l-step cycles), mv (operator applications) and nrm (final
    recursively updated residual norm)."""
    n = b.size
    if max_mv is None:
        max_mv = n
    if rs is None:
        rs = shadow(n)
    x = np.zeros(n, dtype=np.complex128)
    R = np.zeros((ell + 1, n), dtype=np.complex128)
    U = np.zeros((ell + 1, n), dtype=np.complex128)
    R[0] = b
    nrm = np.linalg.norm(R[0])
    tolerance = reltol * nrm
    sigma = omega = 1.0 + 0j
    mv = it = 0
    broke = False
    while not (mv >= max_mv or nrm <= tolerance):
        # a zero or non-finite rho, sigma or MR system ends the solve at the
        # current iterate (the GPU solver retires the right-hand side there),
        # and so does a residual that a BiCG step already brought to
        # tolerance (the next step would divide rounding noise by rounding
        # noise: its sigma is rho - beta * rho_prev)
        sigma = -omega * sigma
        for j in range(1, ell + 1):          # BiCG part
            rho = np.vdot(rs, R[j - 1])
            if rho == 0 or not np.isfinite(rho):
                broke = True
                break
            beta = rho / sigma
            U[:j] = R[:j] - beta * U[:j]
            U[j] = apply(U[j - 1])
            sigma = np.vdot(rs, U[j])
            if sigma == 0 or not np.isfinite(sigma):
                broke = True
                break
            alpha = rho / sigma
            R[:j] -= alpha * U[1:j + 1]
            x += alpha * U[0]
            nrm = np.linalg.norm(R[0])
            if nrm <= tolerance:             # converged inside the BiCG part
                break
            R[j] = apply(R[j - 1])
        mv += 2 * ell
        it += 1
        if broke or nrm <= tolerance:
            break
        M = np.conj(R) @ R.T                 # minimal-residual part
        try:
            gamma = np.linalg.solve(M[1:, 1:], M[1:, 0])
        except np.linalg.LinAlgError:
            broke = True
            break
        if not np.all(np.isfinite(gamma)):
            broke = True
            break
        U[0] -= gamma @ U[1:]
        x += gamma @ R[:ell]
        R[0] -= gamma @ R[1:]
        omega = gamma[-1]
        nrm = np.linalg.norm(R[0])
        if omega == 0:
            broke = True
            break
    return x, {"iters": it, "mv": mv, "nrm": nrm, "broke": broke}


def refine_solve(apply64, b: np.ndarray, tol: float = 1e-6, ell: int = 2, inner_apply=None,
                 inner_tol: float = 1e-4, max_outer: int = 20, max_mv: int = 4000):
    """FP64 iterative refinement around BiCGStab(l), the GPU solver's outer
    loop: r = b - A x; the correction equation A d = r / |r| is solved to
    relative residual t = 0.9 tol |b| / |r| (mixed: at least inner_tol) by
    BiCGStab(l) on `inner_apply` (FP64 `apply64` when None); x += |r| d.
    Returns (x, info)."""
    mixed = inner_apply is not None
    inner = inner_apply or apply64
    x = np.zeros_like(b)
    r = b.copy()
    bn = np.linalg.norm(b)
    rn = bn
    info = {"iters": 0, "outer": 0, "mv": 0}
    mv = 0
    for outer in range(max_outer):
        if bn == 0 or rn <= tol * bn:
            break
        if mv + 2 * ell > max_mv:
            break
        t = 0.9 * tol * bn / rn
        if mixed:
            t = max(t, inner_tol)
        d, inf = bicgstabl(inner, r / rn, ell=ell, reltol=t, max_mv=max_mv - mv)
        mv += inf["mv"]
        info["iters"] += inf["iters"]
        x = x + rn * d
        r = b - apply64(x)
        prev, rn = rn, np.linalg.norm(r)
        info["outer"] += 1
        if not rn < 0.5 * prev and rn > tol * bn:
            break
    info["mv"] = mv
    info["rel_res"] = 0.0 if bn == 0 else rn / bn
    return x, info


def dense_ls(mem: OprMem, chi: np.ndarray) -> np.ndarray:
    """The LippmannSchwinger matrix, one column per unit vector (tiny volumes)."""
    n = 3 * int(np.prod(mem.mix.src_cel))
    A = np.empty((n, n), dtype=np.complex128)
    e = np.zeros(n, dtype=np.complex128)
    for k in range(n):
        e[k] = 1.0
        A[:, k] = ls_apply(mem, chi, e)
        e[k] = 0.0
    return A
