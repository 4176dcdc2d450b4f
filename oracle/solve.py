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
* ``reliable_solve`` is the GPU solver's algorithm: BiCGStab(l) with
  reliable updates (FP64 solution and FP64 residual replacement) around a
  Krylov process on the ComplexF32 (mixed) or ComplexF64 (plain) operator
  (no reference counterpart: the reference solves in one precision); with
  the FP64 operator it is the plain GPU solve step for step.

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


class _Krylov:
    """State of one BiCGStab(l) process (Sleijpen & Fokkema 1993) on the
    operator `apply`: residuals R[0..l], search directions U[0..l], the
    iterate x, and the scalars sigma, omega; shadow residual rs."""

    def __init__(self, apply, r0: np.ndarray, ell: int, rs: np.ndarray):
        n = r0.size
        self.apply, self.ell, self.rs = apply, ell, rs
        self.R = np.zeros((ell + 1, n), dtype=np.complex128)
        self.U = np.zeros((ell + 1, n), dtype=np.complex128)
        self.R[0] = r0
        self.x = np.zeros(n, dtype=np.complex128)
        self.sigma = self.omega = 1.0 + 0j

    def cycle(self, tolerance: float):
        """One l-step cycle.  Returns (nrm, state): state "ok", "conv" (the
        residual reached `tolerance` inside the cycle, which then ends) or
        "broke" (a zero or non-finite rho, sigma or MR system, or omega = 0
        after the update)."""
        R, U, rs, ell = self.R, self.U, self.rs, self.ell
        self.sigma = -self.omega * self.sigma
        for j in range(1, ell + 1):          # BiCG part
            rho = np.vdot(rs, R[j - 1])
            if rho == 0 or not np.isfinite(rho):
                return np.linalg.norm(R[0]), "broke"
            beta = rho / self.sigma
            U[:j] = R[:j] - beta * U[:j]
            U[j] = self.apply(U[j - 1])
            self.sigma = np.vdot(rs, U[j])
            if self.sigma == 0 or not np.isfinite(self.sigma):
                return np.linalg.norm(R[0]), "broke"
            alpha = rho / self.sigma
            R[:j] -= alpha * U[1:j + 1]
            self.x += alpha * U[0]
            nrm = np.linalg.norm(R[0])
            # a residual that a BiCG step already brought to tolerance ends
            # the cycle: the next step would divide rounding noise by rounding
            # noise (its sigma is rho - beta * rho_prev)
            if nrm <= tolerance:
                return nrm, "conv"
            R[j] = self.apply(R[j - 1])
        M = np.conj(R) @ R.T                 # minimal-residual part
        try:
            gamma = np.linalg.solve(M[1:, 1:], M[1:, 0])
        except np.linalg.LinAlgError:
            return np.linalg.norm(R[0]), "broke"
        if not np.all(np.isfinite(gamma)):
            return np.linalg.norm(R[0]), "broke"
        U[0] -= gamma @ U[1:]
        self.x += gamma @ R[:ell]
        R[0] -= gamma @ R[1:]
        self.omega = gamma[-1]
        nrm = np.linalg.norm(R[0])
        if self.omega == 0:
            return nrm, "broke"
        return nrm, ("conv" if nrm <= tolerance else "ok")


def bicgstabl(apply, b: np.ndarray, ell: int = 2, reltol: float = np.sqrt(np.finfo(float).eps),
              max_mv: int | None = None, rs: np.ndarray | None = None):
    """BiCGStab(l) from a zero initial guess, stopping on the recursively
    updated residual (IterativeSolvers.bicgstabl's criterion).  Returns
    (x, info) with iters (l-step cycles), mv (operator applications), nrm
    (final recursive residual norm) and broke."""
    n = b.size
    if max_mv is None:
        max_mv = n
    if rs is None:
        rs = shadow(n)
    k = _Krylov(apply, b, ell, rs)
    nrm = np.linalg.norm(b)
    tolerance = reltol * nrm
    mv = it = 0
    state = "ok"
    while not (mv >= max_mv or nrm <= tolerance or state == "broke"):
        nrm, state = k.cycle(tolerance)
        mv += 2 * ell
        it += 1
    return k.x, {"iters": it, "mv": mv, "nrm": nrm, "broke": state == "broke"}


RELIABLE_GAP = 8  # cycles between two updates triggered by the residual drop delta (solver.h kReliableGap)


def reliable_solve(apply64, b: np.ndarray, tol: float = 1e-6, ell: int = 2, inner_apply=None,
                   delta: float = 0.1, max_mv: int = 4000, max_restarts: int = 20, rs=None):
    """The GPU solver's algorithm: BiCGStab(l) on `inner_apply` (FP64
    `apply64` when None) with reliable updates (residual replacement, van der
    Vorst & Ye 2000; its mixed-precision form as in Clark et al. 2010).

    The Krylov process runs on the scaled system A d = r / s (s = |r| at its
    start).  After a cycle whose recursive residual fell below delta times
    its largest value since the last update, at least RELIABLE_GAP cycles
    after that update (mixed only; delta = 0 for the plain solve), claimed
    convergence (0.9 tol |b| / s), or broke down: the
    correction is folded into the FP64 solution, x += s d, d = 0, and the
    recursive residual is replaced by the FP64 one, r = (b - A64 x) / s,
    keeping the search directions.  A breakdown, or claimed convergence that
    the FP64 residual does not confirm, restarts the process from r.
    Returns (x, info): iters, updates (FP64 residuals), mv, rel_res."""
    n = b.size
    if rs is None:
        rs = shadow(n)
    inner = inner_apply or apply64
    d = delta if inner_apply is not None else 0.0
    x = np.zeros_like(b)
    bn = np.linalg.norm(b)
    r = b.copy()
    rn = bn
    info = {"iters": 0, "updates": 0, "mv": 0, "restarts": 0}

    def done():
        return bn == 0 or rn <= tol * bn

    mv = 0
    k = None
    while not done():
        if k is None:
            if info["restarts"] >= max_restarts:
                break
            s = rn
            k = _Krylov(inner, r / s, ell, rs)
            maxr = 1.0
            since = 0
            info["restarts"] += 1
        if mv + 2 * ell > max_mv:
            break
        nrm, state = k.cycle(0.9 * tol * bn / s)
        mv += 2 * ell
        info["iters"] += 1
        since += 1
        if state == "ok" and not (nrm < d * maxr and since >= RELIABLE_GAP):
            maxr = max(maxr, nrm)
            continue
        x = x + s * k.x                      # reliable update
        k.x[:] = 0
        r = b - apply64(x)
        rn = np.linalg.norm(r)
        info["updates"] += 1
        since = 0
        if state == "ok":
            k.R[0] = r / s
            maxr = rn / s
        else:
            k = None                         # restart (from r) unless done
    if k is not None and np.any(k.x):
        x = x + s * k.x
        r = b - apply64(x)
        rn = np.linalg.norm(r)
        info["updates"] += 1
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
