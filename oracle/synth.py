"""Seeded synthetic Green kernels with the reference's symmetries.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

The real-space kernel of the reference comes from face-pair cubature
(src/glaGen.jl).  For matvec parity any kernel with the same symmetry and
storage rules exercises exactly the same code paths, so this module builds the
circulant from a smooth closed-form dyadic field evaluated at the reference's
circulant separations (grdSel / sepGrd, src/glaGen.jl:603-645):
diagonal components are even along every axis, the xy / xz / yz components
are odd along both of their axes -- the properties that make the symmetric
half-storage of GlaOprMem exact.
"""
from __future__ import annotations

import math

import numpy as np

from .gla_mem import Vol, ExtInf, mix_for, tru_inf
from .fur import crc_to_fur, toe_to_crc


def dyadic(r: np.ndarray, vol: float) -> np.ndarray:
    """Free-space dyadic Green function (wavelength 1) times cell volume,
    G[3,3,...] at separation vectors r[3,...]; finite value at r = 0."""
    k = 2 * math.pi
    rr = np.sqrt((r ** 2).sum(axis=0))
    safe = np.where(rr > 0, rr, 1.0)
    g = np.exp(1j * k * safe) / (4 * math.pi * safe)
    kr = k * safe
    a = 1 + (1j * kr - 1) / kr ** 2
    b = (3 - 3j * kr - kr ** 2) / kr ** 2
    out = np.empty((3, 3, *r.shape[1:]), dtype=np.complex128)
    for i in range(3):
        for j in range(3):
            v = g * (b * r[i] * r[j] / safe ** 2 + (a if i == j else 0))
            out[i, j] = np.where(rr > 0, v * vol * k ** 2, (-1.0 / 3.0 if i == j else 0.0))
    return out


def _sep_axis(trg: Vol, src: Vol, d: int) -> np.ndarray:
    """Separations along axis d for every circulant index m in [0, Nt+Ns):
    grdSel over sepGrd(trg,src,0) / sepGrd(trg,src,1); index Nt is unused."""
    nt, ns = trg.cel[d], src.cel[d]
    t0 = float(trg.start()[d])
    s0 = float(src.start()[d])
    s1 = float(src.stop()[d])
    gt = float(trg.grd[d])
    gs = float(src.grd[d])
    out = np.zeros(nt + ns)
    for m in range(nt + ns):
        if m < nt:
            out[m] = (t0 - s0) + m * gt
        elif m > nt:
            out[m] = (t0 - s1) + (m - nt - 1) * gs
    return out


def synth_crc(trg: Vol, src: Vol, is_self: bool) -> np.ndarray:
    """Circulant crc[3,3,P...] of the synthetic dyadic field (1 partition)."""
    vol = float(np.prod([float(s) for s in src.scl]))
    if is_self:
        n = trg.cel
        r = np.stack(np.meshgrid(*[np.arange(v) * float(trg.grd[d])
                                   for d, v in enumerate(n)], indexing="ij"))
        return toe_to_crc(dyadic(r, vol))
    sep = [_sep_axis(trg, src, d) for d in range(3)]
    r = np.stack(np.meshgrid(*sep, indexing="ij"))
    crc = dyadic(r, vol)
    nt = trg.cel
    for d in range(3):
        sl = [slice(None)] * 5
        sl[2 + d] = nt[d]
        crc[tuple(sl)] = 0
    return crc


def synth_operator(trg_cel, scl, trg_org=(0, 0, 0), src_cel=None, src_org=None,
                   set_dtype=np.complex128):
    """Build (mix, fur, crc, is_self, trg, src) for a synthetic operator with
    a single partition (equal cell scales)."""
    trg = Vol.make(trg_cel, scl, trg_org)
    src = None if src_cel is None else Vol.make(src_cel, scl, src_org)
    trg, src, mix, is_self = mix_for(trg, src)
    crc = synth_crc(trg, src, is_self)
    fur = crc_to_fur(crc, tru_inf(trg, src, mix), set_dtype)
    return mix, fur, crc, is_self, trg, src


def seeded_current(cel, seed: int, dtype=np.complex128) -> np.ndarray:
    """Source current [x,y,z,3] with i.i.d. N(0,1) real and imaginary parts."""
    rng = np.random.default_rng(seed)
    shp = (*cel, 3)
    return (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(dtype)
