"""Oracle restatement of the volume / partition structures of src/glaMem.jl.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from fractions import Fraction
from typing import Tuple

Int3 = Tuple[int, int, int]
Rat3 = Tuple[Fraction, Fraction, Fraction]


def _rat3(v) -> Rat3:
    return tuple(Fraction(x) for x in v)  # type: ignore[return-value]


@dataclass(frozen=True)
class Vol:
    """GlaVol (src/glaMem.jl:12-19, constructor :136-148).

    ``org`` is the centre of the volume; cell centres are
    ``org - brd + k*grd`` with ``brd = grd*(floor(cel/2) - iseven(cel)/2)``.
    """
    cel: Int3
    scl: Rat3
    org: Rat3
    grd: Rat3  # grid step (cell pitch); equals scl unless partitioned

    @staticmethod
    def make(cel, scl, org=(0, 0, 0), grd=None) -> "Vol":
        scl = _rat3(scl)
        org = _rat3(org)
        grd = scl if grd is None else _rat3(grd)
        if not all(s <= g for s, g in zip(scl, grd)):
            raise ValueError("cell scale must be smaller than the grid scale")
        return Vol(tuple(int(c) for c in cel), scl, org, grd)

    def brd(self) -> Rat3:
        return tuple(g * (Fraction(c // 2) - Fraction(1 if c % 2 == 0 else 0, 2))
                     for g, c in zip(self.grd, self.cel))

    def start(self) -> Rat3:
        return tuple(o - b for o, b in zip(self.org, self.brd()))

    def stop(self) -> Rat3:
        return tuple(o + b for o, b in zip(self.org, self.brd()))


def vol_even(v: Vol) -> Vol:
    """glaVolEveGen (src/glaMem.jl:152-175): make every cell count even by
    adding one cell along odd axes and shrinking the cell to keep the extent."""
    if all(c % 2 == 0 for c in v.cel):
        return v
    par = [c % 2 for c in v.cel]
    new_cel = tuple(c + p for c, p in zip(v.cel, par))
    new_scl = tuple(Fraction(s.numerator * c, s.denominator * n)
                    for s, c, n in zip(v.scl, v.cel, new_cel))
    new_grd = tuple(Fraction(g.numerator * c, g.denominator * n)
                    for g, c, n in zip(v.grd, v.cel, new_cel))
    return Vol(new_cel, new_scl, v.org, new_grd)


def _rgcd(a: Fraction, b: Fraction) -> Fraction:
    return Fraction(math.gcd(a.numerator, b.numerator),
                    math.lcm(a.denominator, b.denominator))


def _rlcm(a: Fraction, b: Fraction) -> Fraction:
    return Fraction(math.lcm(a.numerator, b.numerator),
                    math.gcd(a.denominator, b.denominator))


@dataclass(frozen=True)
class ExtInf:
    """GlaExtInf (src/glaMem.jl:39-47, constructor :190-216)."""
    min_scl: Rat3
    trg_div: Int3
    src_div: Int3
    trg_cel: Int3
    src_cel: Int3

    @staticmethod
    def make(trg: Vol, src: Vol) -> "ExtInf":
        ok = 1
        for a, b in zip(src.scl, trg.scl):
            ok *= int((a / b).denominator == 1) + int((b / a).denominator == 1)
        if ok == 0:
            raise ValueError("Volume pair must share a common scale grid.")
        min_scl = tuple(_rgcd(a, b) for a, b in zip(src.scl, trg.scl))
        max_scl = tuple(_rlcm(a, b) for a, b in zip(src.scl, trg.scl))
        trg_div = tuple(int(m // s) for m, s in zip(max_scl, trg.scl))
        src_div = tuple(int(m // s) for m, s in zip(max_scl, src.scl))
        trg_cel = tuple(c // d for c, d in zip(trg.cel, trg_div))
        src_cel = tuple(c // d for c, d in zip(src.cel, src_div))
        if math.prod(trg_cel) == 0 or math.prod(src_cel) == 0:
            raise ValueError("Volume sizes are incompatible---volume smaller than cell.")
        return ExtInf(min_scl, trg_div, src_div, trg_cel, src_cel)

    def par_offsets(self, which: str):
        """trgPar / srcPar: partition grid offsets, x fastest (Julia
        CartesianIndices order)."""
        div = self.trg_div if which == "trg" else self.src_div
        out = []
        for k in range(div[2]):
            for j in range(div[1]):
                for i in range(div[0]):
                    out.append((i, j, k))
        return out

    @property
    def brn(self) -> Int3:
        return tuple((t + s) // 2 for t, s in zip(self.trg_cel, self.src_cel))


def mix_for(trg: Vol, src: Vol | None):
    """Self / external detection and even-cell regeneration as done at the
    top of GlaOprMem (src/glaMemSup.jl:26-43).  Returns (trg, src, mix, self)."""
    if src is None or src == trg:
        return trg, trg, ExtInf.make(trg, trg), True
    if sum((t + s) % 2 for t, s in zip(trg.cel, src.cel)) != 0:
        trg = vol_even(trg)
        src = vol_even(src)
    return trg, src, ExtInf.make(trg, src), False


def tru_inf(trg: Vol, src: Vol, mix: ExtInf) -> Int3:
    """Stored kernel extent per axis (src/glaMemSup.jl:121-136)."""
    tot = tuple(t + s for t, s in zip(mix.trg_cel, mix.src_cel))
    out = []
    for d in range(3):
        if (mix.trg_cel[d] == mix.src_cel[d] and math.prod(mix.src_div) == 1
                and math.prod(mix.trg_div) == 1 and trg.org[d] == src.org[d]):
            n = mix.trg_cel[d]
            out.append(max(int(math.ceil(n / 2)) + (1 if n % 2 == 0 else 0), 2))
        else:
            out.append(tot[d] // 2)
    return tuple(out)
