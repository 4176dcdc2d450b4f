"""ctypes binding of the C restatement of the kernel build (gen.c) and the
GlaOprMem assembly on top of it.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess
from fractions import Fraction

import numpy as np

from .fur import crc_to_fur
from .gla_mem import Vol, mix_for, tru_inf

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libgilaref.so")
_lib = None

I3 = ct.c_int64 * 3


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "gen.c")):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        _lib = ct.CDLL(LIB)
        _lib.gila_ref_weak.restype = ct.c_int
        _lib.gila_ref_self_circulant.restype = ct.c_int
        _lib.gila_ref_ext_circulant.restype = ct.c_int
        _lib.gila_ref_face_pair.restype = ct.c_int
        _lib.gila_ref_max_regions.restype = ct.c_long
        _lib.gila_ref_gauleg.restype = ct.c_int
    return _lib


def _rat3(v):
    n = I3(*[Fraction(x).numerator for x in v])
    d = I3(*[Fraction(x).denominator for x in v])
    return n, d


def gauleg(n):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().gila_ref_gauleg(n, x.ctypes.data_as(ct.POINTER(ct.c_double)), w.ctypes.data_as(ct.POINTER(ct.c_double)))
    return x, w


def weak(scl, frq=1.0 + 0j, int_ord=32):
    """Unscaled (wS[3], wE[9], wV[6]) of wekS / wekE / wekV (src/glaInt.jl:75-262)."""
    out = np.zeros(36)
    n, d = _rat3(scl)
    st = lib().gila_ref_weak(n, d, ct.c_double(frq.real), ct.c_double(frq.imag), int_ord,
                             out.ctypes.data_as(ct.POINTER(ct.c_double)))
    if st:
        raise RuntimeError(f"gila_ref_weak failed ({st})")
    c = out[0::2] + 1j * out[1::2]
    return c[:3], c[3:12], c[12:18]


def face_pair(tscl, sscl, sep, ft, fs, frq=1.0 + 0j):
    """One hcubature face-pair integral (egoSrfAdp!, src/glaGen.jl:559-584),
    unscaled; returns (value, regions)."""
    out = np.zeros(2)
    nr = ct.c_int()
    tn, td = _rat3(tscl)
    sn, sd = _rat3(sscl)
    s = (ct.c_double * 3)(*sep)
    st = lib().gila_ref_face_pair(tn, td, sn, sd, s, ft, fs, ct.c_double(frq.real), ct.c_double(frq.imag),
                                  out.ctypes.data_as(ct.POINTER(ct.c_double)), ct.byref(nr))
    if st:
        raise RuntimeError("face_pair failed")
    return out[0] + 1j * out[1], nr.value


def _crc_to_rc(raw, P):
    """crc[z][y][x][3][3] -> crc[3,3,Px,Py,Pz]."""
    a = raw.reshape(P[2], P[1], P[0], 3, 3)
    return np.ascontiguousarray(a.transpose(3, 4, 2, 1, 0))


def self_circulant(vol: Vol, frq=1.0 + 0j, int_ord=32, weak_vals=None):
    """genEgoSlf! (src/glaGen.jl:38-53): circulant crc[3,3,2Nx,2Ny,2Nz]."""
    P = [2 * c for c in vol.cel]
    raw = np.zeros(int(np.prod(P)) * 9 * 2)
    cel = I3(*vol.cel)
    sn, sd = _rat3(vol.scl)
    gn, gd = _rat3(vol.grd)
    wk = None
    if weak_vals is not None:
        w = np.concatenate([np.asarray(v, dtype=np.complex128) for v in weak_vals])
        wk = np.zeros(36)
        wk[0::2] = w.real
        wk[1::2] = w.imag
    st = lib().gila_ref_self_circulant(cel, sn, sd, gn, gd, ct.c_double(frq.real), ct.c_double(frq.imag), int_ord,
                                       None if wk is None else wk.ctypes.data_as(ct.POINTER(ct.c_double)),
                                       raw.ctypes.data_as(ct.POINTER(ct.c_double)))
    if st:
        raise RuntimeError(f"self circulant failed ({st})")
    return _crc_to_rc(raw[0::2] + 1j * raw[1::2], P)


def ext_circulant(trg: Vol, src: Vol, frq=1.0 + 0j, int_ord=32):
    """genEgoExt! (src/glaGen.jl:17-31): circulant crc[3,3,Nt+Ns...]."""
    P = [t + s for t, s in zip(trg.cel, src.cel)]
    raw = np.zeros(int(np.prod(P)) * 9 * 2)
    args = []
    for v in (trg, src):
        args += [I3(*v.cel), *_rat3(v.scl), *_rat3(v.org), *_rat3(v.grd)]
    st = lib().gila_ref_ext_circulant(*args, ct.c_double(frq.real), ct.c_double(frq.imag), int_ord,
                                      raw.ctypes.data_as(ct.POINTER(ct.c_double)))
    if st == -3:
        raise ValueError("Source and target volumes are overlapping.")
    if st:
        raise RuntimeError(f"external circulant failed ({st})")
    return _crc_to_rc(raw[0::2] + 1j * raw[1::2], P)


def partition_vols(vol: Vol, div, par_cel):
    """The partitions of a volume whose cells sit on a grid `div` times
    coarser than the pair's common grid (src/glaMemSup.jl:60-87): partition
    offsets x fastest, centre ((off - (div - 1) / 2) * scl + org), cell
    scale scl, grid step div * scl."""
    out = []
    for k in range(div[2]):
        for j in range(div[1]):
            for i in range(div[0]):
                off = (i, j, k)
                org = tuple((Fraction(o) - Fraction(d - 1, 2)) * s + g
                            for o, d, s, g in zip(off, div, vol.scl, vol.org))
                grd = tuple(d * s for d, s in zip(div, vol.scl))
                out.append(Vol(tuple(par_cel), vol.scl, org, grd))
    return out


def build_operator_vols(trg: Vol, src: Vol | None, frq=1.0 + 0j, int_ord=32, set_dtype=np.complex128,
                        weak_vals=None):
    """GlaOprMem without egoFur (src/glaMemSup.jl:16-171) for volume pairs of
    any compatible scales: the external circulant of every (source,
    target) partition pair, crc[3,3,P...,parS,parT], then the Fourier
    kernel.  Returns (mix, fur, crc, is_self, trg, src)."""
    trg, src, mix, is_self = mix_for(trg, src)
    if is_self:
        crc = self_circulant(trg, frq, int_ord, weak_vals)
    else:
        tp = partition_vols(trg, mix.trg_div, mix.trg_cel)
        sp = partition_vols(src, mix.src_div, mix.src_cel)
        if len(tp) * len(sp) == 1:
            crc = ext_circulant(trg, src, frq, int_ord)
        else:
            P = [t + s for t, s in zip(mix.trg_cel, mix.src_cel)]
            crc = np.empty((3, 3, *P, len(sp), len(tp)), dtype=np.complex128)
            for ti, tv in enumerate(tp):
                for si, sv in enumerate(sp):
                    crc[..., si, ti] = ext_circulant(tv, sv, frq, int_ord)
    if not np.all(np.isfinite(crc)):
        raise ValueError("Computed circulant contains non-numeric values.")
    fur = crc_to_fur(crc, tru_inf(trg, src, mix), set_dtype)
    return mix, fur, crc, is_self, trg, src


def build_operator(trg_cel, scl, trg_org=(0, 0, 0), src_cel=None, src_org=None, frq=1.0 + 0j, int_ord=32,
                   set_dtype=np.complex128, weak_vals=None, src_scl=None):
    """GlaOprMem without egoFur for a target (and source) given by cells,
    scale and centre; `src_scl` defaults to the target's scale."""
    trg = Vol.make(trg_cel, scl, trg_org)
    src = None if src_cel is None else Vol.make(src_cel, scl if src_scl is None else src_scl, src_org)
    return build_operator_vols(trg, src, frq, int_ord, set_dtype, weak_vals)
