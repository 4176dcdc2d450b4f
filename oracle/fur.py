"""Oracle restatement of the Fourier-kernel assembly of GlaOprMem and two
independent formulations of the matvec used to cross-check the 8-branch
recursion in ``matvec.py``.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

  * toe_to_crc     egoToeCrc! / indSel / indFlp     src/glaGen.jl:143-163,647-662
  * crc_to_fur     FFT of the 6 unique components, parity-branch extraction,
                   symmetric truncation, cast       src/glaMemSup.jl:96-156
  * blk_ego_itr    component map (xx,yy,zz,xy,xz,yz) src/glaMemSup.jl:273-291
  * fur_to_full    re-expansion of the 8 stored branches to the full padded
                   spectrum using the mirror/sign rules of mulBrnHst!
                   (src/glaActSup.jl:697-752)
  * padfft_apply   zero-pad -> 3-D FFT -> 3x3 multiply -> IFFT -> truncate
  * direct_apply   real-space circular convolution with the circulant
                   (the idea of utl/glaEgoMat.jl:15-77)
"""
from __future__ import annotations

import math

import numpy as np

from .gla_mem import ExtInf

# (row, col) of the upper triangle for stored component c = 0..5
COMP_RC = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
OFFDIAG_AXES = {3: (0, 1), 4: (0, 2), 5: (1, 2)}


def blk_ego_itr(crt: int) -> int:
    """blkEgoItr: 1-based Cartesian block index 3*(col-1)+row -> stored
    component (1-based)."""
    return {1: 1, 2: 4, 4: 4, 5: 2, 3: 5, 7: 5, 6: 6, 8: 6, 9: 3}[crt]


def toe_to_crc(toe: np.ndarray) -> np.ndarray:
    """egoToeCrc!: embed a self Toeplitz field toe[3,3,Nx,Ny,Nz] into the
    circulant crc[3,3,2Nx,2Ny,2Nz]; index N is zeroed, the mirrored half
    flips the sign of off-diagonal entries (dipole reflection)."""
    n = toe.shape[2:]
    crc = np.zeros((3, 3, *[2 * v for v in n]), dtype=np.complex128)
    idx = []
    flp = []
    for d in range(3):
        p = np.arange(2 * n[d])
        sel = np.where(p < n[d], p, 2 * n[d] - p)  # 0-based indSel
        f = np.where(p < n[d], 1.0, -1.0)
        idx.append(np.clip(sel, 0, n[d] - 1))
        flp.append(f)
    sub = toe[:, :, idx[0][:, None, None], idx[1][None, :, None], idx[2][None, None, :]]
    fl = [flp[0][:, None, None], flp[1][None, :, None], flp[2][None, None, :]]
    for r in range(3):
        for c in range(3):
            m = np.ones_like(sub[0, 0].real)
            if r != c:
                m = m * fl[r] * fl[c]
            crc[r, c] = sub[r, c] * m
    for d in range(3):
        sl = [slice(None)] * 5
        sl[2 + d] = n[d]
        crc[tuple(sl)] = 0
    return crc


def crc_to_fur(crc: np.ndarray, tru, set_dtype=np.complex128):
    """GlaOprMem kernel section: crc[3,3,Px,Py,Pz,parS,parT] (or without the
    two partition axes) -> list of 8 arrays (tx,ty,tz,6,parS,parT)."""
    if crc.ndim == 5:
        crc = crc[..., None, None]
    P = crc.shape[2:5]
    par_s, par_t = crc.shape[5], crc.shape[6]
    prp = np.empty((*P, 6, par_s, par_t), dtype=np.complex128)
    for t in range(par_t):
        for s in range(par_s):
            for col in range(3):
                for row in range(col + 1):
                    b = blk_ego_itr(3 * col + row + 1) - 1
                    prp[:, :, :, b, s, t] = np.fft.fftn(crc[row, col, :, :, :, s, t])
    if not np.all(np.isfinite(prp)):
        raise ValueError("Fourier transform of circulant contains non-numeric values.")
    half = [max(p // 2, 2) for p in P]
    fur = []
    for eo in range(8):
        px, py, pz = (eo // 4) % 2, (eo // 2) % 2, eo % 2
        sub = prp[px::2, py::2, pz::2]
        full = np.broadcast_to(sub, (*half, 6, par_s, par_t))
        fur.append(np.array(full[:tru[0], :tru[1], :tru[2]], dtype=set_dtype, order="F"))
    return fur


def axis_map(mix: ExtInf, stored: int, d: int):
    """For axis d, map every padded frequency f in [0,P) to
    (branch bit, stored index, mirrored flag) following mulBrnHst!."""
    brn = mix.brn[d]
    P = 2 * brn
    f = np.arange(P)
    p = f % 2
    k = f // 2
    if stored == brn:
        return p, k, np.zeros(P, dtype=bool)
    t = mix.trg_cel[d]
    fwd_even = int(math.ceil(t / 2)) + (1 if t % 2 == 0 else 0)
    fwd_odd = int(math.ceil(t / 2))
    m = np.where(p == 0,
                 np.where(k < fwd_even, k, brn - k),
                 np.where(k < fwd_odd, k, brn - 1 - k))
    mir = np.where(p == 0, k >= fwd_even, k >= fwd_odd)
    return p, m, mir


def fur_to_full(mix: ExtInf, fur) -> np.ndarray:
    """Expand the 8 stored branches to G[c, fx, fy, fz, s, t] over the full
    padded spectrum (P = 2*brn per axis)."""
    st = fur[0].shape[:3]
    maps = [axis_map(mix, st[d], d) for d in range(3)]
    P = [2 * b for b in mix.brn]
    par_s, par_t = fur[0].shape[4], fur[0].shape[5]
    G = np.empty((6, *P, par_s, par_t), dtype=np.complex128)
    (px, mx, rx), (py, my, ry), (pz, mz, rz) = maps
    eo = (4 * px[:, None, None] + 2 * py[None, :, None] + pz[None, None, :])
    rev = [rx[:, None, None], ry[None, :, None], rz[None, None, :]]
    for c in range(6):
        vals = np.empty((*P, par_s, par_t), dtype=np.complex128)
        for b in range(8):
            sel = eo == b
            if not np.any(sel):
                continue
            g = fur[b][:, :, :, c]
            v = g[mx[:, None, None], my[None, :, None], mz[None, None, :]]
            vals[sel] = v[sel]
        if c in OFFDIAG_AXES:
            a, b2 = OFFDIAG_AXES[c]
            sgn = np.where(rev[a] ^ rev[b2], -1.0, 1.0)
            vals = vals * sgn[..., None, None]
        G[c] = vals
    return G


def _sym(Gc, fx):
    """3x3 symmetric matrix rows from the six components."""
    xx, yy, zz, xy, xz, yz = Gc
    return ((xx, xy, xz), (xy, yy, yz), (xz, yz, zz))


def padfft_apply(mix: ExtInf, G: np.ndarray, x: np.ndarray) -> np.ndarray:
    """Zero-padded FFT convolution; x[x,y,z,3,parS] -> y[x,y,z,3,parT] at
    partition size."""
    P = G.shape[1:4]
    par_s, par_t = G.shape[4], G.shape[5]
    if x.ndim == 4:
        x = x[..., None]
    X = np.zeros((*P, 3, par_s), dtype=np.complex128)
    sc = mix.src_cel
    X[:sc[0], :sc[1], :sc[2]] = x
    X = np.fft.fftn(X, axes=(0, 1, 2))
    tc = mix.trg_cel
    out = np.empty((*tc, 3, par_t), dtype=np.complex128)
    for t in range(par_t):
        Y = np.zeros((*P, 3), dtype=np.complex128)
        for s in range(par_s):
            M = _sym([G[c, :, :, :, s, t] for c in range(6)], None)
            for i in range(3):
                for j in range(3):
                    Y[..., i] += M[i][j] * X[..., j, s]
        y = np.fft.ifftn(Y, axes=(0, 1, 2))
        out[..., t] = y[:tc[0], :tc[1], :tc[2]]
    return out


def direct_apply(crc: np.ndarray, src_cel, trg_cel, x: np.ndarray) -> np.ndarray:
    """Real-space circular convolution y[n] = sum_m C[m] x[(n-m) mod P]
    (single partition) with the symmetric 3x3 built from the upper triangle
    of the circulant crc[3,3,Px,Py,Pz]."""
    P = crc.shape[2:5]
    out = np.zeros((*trg_cel, 3), dtype=np.complex128)
    xs = np.nonzero(np.ones(src_cel, dtype=bool))
    pts = list(zip(*xs))
    for i in range(3):
        for j in range(3):
            r, c = (i, j) if i <= j else (j, i)
            C = crc[r, c]
            for (a, b, e) in pts:
                xv = x[a, b, e, j]
                if xv == 0:
                    continue
                ix = (np.arange(trg_cel[0]) - a) % P[0]
                iy = (np.arange(trg_cel[1]) - b) % P[1]
                iz = (np.arange(trg_cel[2]) - e) % P[2]
                out[..., i] += C[np.ix_(ix, iy, iz)] * xv
    return out
