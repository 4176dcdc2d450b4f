"""The on-disk kernel cache (gila_opr_save / gila_opr_load, GILAFUR1).

The reference keeps egoFur between sessions with Serialization in a Scratch
space (test/runtests.jl:38-98) or with JLD2 keyed by type, cells and scale
(examples/GilaOperators.jl:28-55).  Here an operator saved and loaded again
must hold the same egoFur bit for bit and give a bit-identical matvec; the
header is parsed independently with numpy against the documented layout; a
ComplexF64 file loads as ComplexF32 by a cast.
"""
from __future__ import annotations

from fractions import Fraction

import numpy as np
import pytest

from conftest import load_pkg
from oracle.synth import seeded_current, synth_operator

pytestmark = pytest.mark.gpu

SCL = ("1/32", "1/32", "1/32")
CASES = [((12, 10, 8), None, (0, 0, 0), None),
         ((8, 6, 4), (6, 10, 8), ("13/32", 0, 0), (0, 0, 0))]


def _mem(gila, case, dtype):
    tc, sc, to, so = case
    mix, fur, _, is_self, trg, src = synth_operator(tc, SCL, to, sc, so)
    tv = gila.GlaVol(trg.cel, trg.scl, trg.org)
    sv = None if is_self else gila.GlaVol(src.cel, src.scl, src.org)
    opt = gila.GlaKerOpt(1.0 + 0.25j, 24, False, True, (), ())
    return mix, gila.GlaOprMem(opt, tv, sv, egoFur=[f.astype(dtype) for f in fur], setTyp=dtype), is_self


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
@pytest.mark.parametrize("case", CASES, ids=["self", "external"])
def test_save_load_round_trip_is_bit_identical(tmp_path, case, dtype):
    gila = load_pkg()
    mix, mem, is_self = _mem(gila, case, dtype)
    path = tmp_path / "op.gilafur"
    mem.save(path)
    back = gila.GlaOprMem.load(path, setTyp=dtype)
    for a, b in zip(mem.egoFur, back.egoFur):
        assert a.dtype == b.dtype and np.array_equal(a, b)
    assert back.trgVol == mem.trgVol and back.srcVol == mem.srcVol
    assert back.cmpInf.frqPhz == 1.0 + 0.25j and back.cmpInf.intOrd == 24
    x = np.asfortranarray(seeded_current(mix.src_cel, 9).astype(dtype))
    assert np.array_equal(gila.egoOpr(mem, x), gila.egoOpr(back, x))
    # the header, read with numpy against the documented layout
    raw = path.read_bytes()
    assert raw[:8] == b"GILAFUR1"
    i32 = np.frombuffer(raw, "<i4", 6, 8)
    assert list(i32) == [1, 1 if dtype == np.complex128 else 0, 1 if is_self else 0, 0, 24, 0]
    assert tuple(np.frombuffer(raw, "<f8", 2, 32)) == (1.0, 0.25)
    vols = np.frombuffer(raw, "<i8", 42, 48).reshape(2, 7, 3)
    assert tuple(vols[0, 0]) == tuple(mem.trgVol.cel)
    assert tuple(Fraction(int(n), int(d)) for n, d in zip(vols[1, 1], vols[1, 2])) == tuple(mem.srcVol.scl)
    dims = np.frombuffer(raw, "<i8", 48, 384).reshape(8, 6)
    fur = mem.egoFur
    assert all(tuple(dims[e]) == fur[e].shape for e in range(8))
    cs = np.dtype(dtype).itemsize
    assert len(raw) == 768 + cs * sum(f.size for f in fur)
    first = np.frombuffer(raw, dtype, fur[0].size, 768).reshape(fur[0].shape, order="F")
    assert np.array_equal(first, fur[0])


def test_load_casts_and_rejects_bad_files(tmp_path):
    gila = load_pkg()
    _, mem, _ = _mem(gila, CASES[0], np.complex128)
    path = tmp_path / "op.gilafur"
    mem.save(path)
    m32 = gila.GlaOprMem.load(path, setTyp=np.complex64)
    for a, b in zip(mem.egoFur, m32.egoFur):
        assert np.array_equal(a.astype(np.complex64), b)
    bad = tmp_path / "bad.gilafur"
    bad.write_bytes(b"NOTAFUR1" + path.read_bytes()[8:])
    with pytest.raises(gila.GilaError, match="not a GILAFUR1"):
        gila.GlaOprMem.load(bad)
    short = tmp_path / "short.gilafur"
    short.write_bytes(path.read_bytes()[:-16])
    with pytest.raises(gila.GilaError, match="ends inside"):
        gila.GlaOprMem.load(short)
