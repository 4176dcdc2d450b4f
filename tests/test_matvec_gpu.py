"""GPU parity of the matvec against the FP64 CPU oracle (egoBrnHst!
restatement), through the C-ABI.

Tolerances (relative L2 over the whole output): ComplexF64 <= 1e-12,
ComplexF32 <= 1e-5.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import TOL_F32, TOL_F64, load_pkg, rel_l2
from oracle.matvec import OprMem, ego_opr
from oracle.synth import seeded_current, synth_operator

pytestmark = pytest.mark.gpu

SCL = ("1/32", "1/32", "1/32")

# (trg_cel, src_cel, trg_org, src_org): self when src_cel is None
CASES = [
    ((8, 8, 8), None, (0, 0, 0), None),
    ((5, 3, 6), None, (0, 0, 0), None),
    ((2, 2, 2), None, (0, 0, 0), None),
    ((1, 3, 2), None, (0, 0, 0), None),
    ((16, 12, 10), None, (0, 0, 0), None),
    ((7, 9, 5), None, (0, 0, 0), None),
    ((4, 4, 4), (4, 4, 4), (0, "4/32", 0), (0, 0, 0)),
    ((4, 4, 2), (6, 4, 4), ("9/32", 0, 0), (0, 0, 0)),
    ((3, 4, 5), (5, 4, 3), ("1/2", "1/3", "1/4"), (0, 0, 0)),
    ((8, 8, 4), (8, 8, 8), ("10/32", 0, 0), (0, 0, 0)),
]


def _build(gila, case, dtype):
    tc, sc, to, so = case
    mix, fur, crc, is_self, trg, src = synth_operator(tc, SCL, to, sc, so, set_dtype=np.complex128)
    tv = gila.GlaVol(trg.cel, trg.scl, trg.org)
    sv = None if is_self else gila.GlaVol(src.cel, src.scl, src.org)
    mem = gila.GlaOprMem(gila.GlaKerOpt(True), tv, sv, egoFur=[f.astype(dtype) for f in fur], setTyp=dtype)
    return mix, fur, mem


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}<-{c[1]}")
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_matvec_parity(case, dtype):
    gila = load_pkg()
    mix, fur, mem = _build(gila, case, dtype)
    x = seeded_current(mix.src_cel, 7)
    xin = np.asfortranarray(x.astype(dtype))
    y = gila.egoOpr(mem, xin)
    # oracle on the same (possibly rounded) kernel, in FP64
    ref = ego_opr(OprMem(mix, [f.astype(dtype).astype(np.complex128) for f in fur]), xin.astype(np.complex128))
    tol = TOL_F64 if dtype == np.complex128 else TOL_F32
    assert rel_l2(y, ref) <= tol
    # input untouched
    assert np.array_equal(xin, np.asfortranarray(x.astype(dtype)))


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_multi_rhs_and_axpby(dtype):
    gila = load_pkg()
    mix, fur, mem = _build(gila, ((6, 10, 8), None, (0, 0, 0), None), dtype)
    n = 5
    xs = [seeded_current(mix.src_cel, 100 + k).astype(dtype) for k in range(n)]
    X = np.stack([np.asfortranarray(x) for x in xs], axis=-1)
    X = np.asfortranarray(X)
    Y = np.empty_like(X)
    mem.apply_into(X, Y, nrhs=n)
    tol = TOL_F64 if dtype == np.complex128 else TOL_F32
    om = OprMem(mix, [f.astype(dtype).astype(np.complex128) for f in fur])
    for k in range(n):
        assert rel_l2(Y[..., k], ego_opr(om, xs[k].astype(np.complex128))) <= tol
    # mul!(out, G, x, alpha, beta)
    a, b = 0.5 - 2j, 1.5 + 0.25j
    out0 = np.asfortranarray(seeded_current(mix.trg_cel, 3).astype(dtype))
    out = out0.copy(order="F")
    G = gila.GlaOpr(mem)
    gila.mul(out, G, xs[0], a, b)
    ref = a * ego_opr(om, xs[0].astype(np.complex128)) + b * out0.astype(np.complex128)
    assert rel_l2(out, ref) <= tol


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_host_batches_pipelined(dtype):
    """Several vectors in host memory go through the device one at a time
    with overlapped copies: the same values as the batched device call,
    for pinned and pageable host memory, host input or host output only,
    and the fused axpby (whose old host output is uploaded per vector)."""
    import torch
    gila = load_pkg()
    mix, fur, mem = _build(gila, ((64, 64, 8), None, (0, 0, 0), None), dtype)
    n = 4
    tdt = torch.complex128 if dtype == np.complex128 else torch.complex64
    xs = [np.asfortranarray(seeded_current(mix.src_cel, 200 + k).astype(dtype)) for k in range(n)]
    X = np.asfortranarray(np.stack(xs, axis=-1))
    Xt = torch.from_numpy(np.ascontiguousarray(X.transpose(4, 3, 2, 1, 0)))
    Xd = Xt.cuda()
    Yd = torch.empty_like(Xd)
    mem.apply_into(Xd, Yd, nrhs=n)
    ref = Yd.cpu()
    Yp = torch.empty_like(Xt).pin_memory()
    mem.apply_into(Xt.pin_memory(), Yp, nrhs=n)                 # pinned host -> pinned host
    assert torch.equal(Yp, ref)
    Yh = torch.empty_like(Xt)
    mem.apply_into(Xt, Yh, nrhs=n)                              # pageable host
    assert torch.equal(Yh, ref)
    Ym = torch.empty_like(Xt).pin_memory()
    mem.apply_into(Xd, Ym, nrhs=n)                              # device in, host out
    assert torch.equal(Ym, ref)
    Yd2 = torch.empty_like(Xd)
    mem.apply_into(Xt.pin_memory(), Yd2, nrhs=n)                # host in, device out
    assert torch.equal(Yd2.cpu(), ref)
    # axpby with host output: out = a G x + b out
    a, b = 0.5 - 2j, 1.5 + 0.25j
    O0 = torch.from_numpy(np.ascontiguousarray(
        np.stack([seeded_current(mix.trg_cel, 300 + k).astype(dtype) for k in range(n)], axis=-1)
        .transpose(4, 3, 2, 1, 0)))
    Od = O0.cuda()
    mem.axpby_into(a, Xd, b, Od, nrhs=n)
    Oh = O0.clone().pin_memory()
    mem.axpby_into(a, Xt.pin_memory(), b, Oh, nrhs=n)
    assert torch.equal(Oh, Od.cpu())
    assert Yp.dtype == tdt
    tol = TOL_F64 if dtype == np.complex128 else TOL_F32
    om = OprMem(mix, [f.astype(dtype).astype(np.complex128) for f in fur])
    got = Yp.numpy().transpose(4, 3, 2, 1, 0)
    for k in range(n):
        assert rel_l2(got[..., k], ego_opr(om, xs[k].astype(np.complex128))) <= tol


def test_device_tensors_and_determinism():
    import torch
    gila = load_pkg()
    mix, fur, mem = _build(gila, ((12, 8, 10), None, (0, 0, 0), None), np.complex128)
    x = seeded_current(mix.src_cel, 11)
    xt = torch.from_numpy(np.ascontiguousarray(x.transpose(3, 2, 1, 0))).cuda()
    y1 = gila.egoOpr(mem, xt)
    y2 = gila.egoOpr(mem, xt)
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)  # bit-identical on repeat
    ref = ego_opr(OprMem(mix, fur), x)
    got = y1.cpu().numpy().transpose(3, 2, 1, 0)
    assert rel_l2(got, ref) <= TOL_F64


def test_self_external_identity():
    """test/extSlfTest.jl:44-47: G_U(x_A) restricted to B equals
    G_ext(B<-A)(x_A) for A, B touching halves of U."""
    gila = load_pkg()
    celA = (8, 8, 8)
    celU = (8, 16, 8)
    scl = ("1/50", "1/50", "1/50")
    # U centred at 0 spans y in [-8,8)/50; A = lower half centred at -4/50,
    # B = upper half centred at +4/50
    mixU, furU, _, _, trgU, _ = synth_operator(celU, scl, (0, 0, 0))
    mixE, furE, _, _, trgB, srcA = synth_operator(celA, scl, (0, "4/50", 0), celA, (0, "-4/50", 0))
    opt = gila.GlaKerOpt(True)
    memU = gila.GlaOprMem(opt, gila.GlaVol(celU, scl, (0, 0, 0)), egoFur=furU)
    memE = gila.GlaOprMem(opt, gila.GlaVol(celA, scl, (0, "4/50", 0)), gila.GlaVol(celA, scl, (0, "-4/50", 0)),
                          egoFur=furE)
    xU = np.zeros((*celU, 3), dtype=np.complex128, order="F")
    xA = seeded_current(celA, 5)
    xU[:, :8, :, :] = xA
    yU = gila.egoOpr(memU, xU)
    yE = gila.egoOpr(memE, np.asfortranarray(xA))
    assert rel_l2(yE, yU[:, 8:, :, :]) <= 1e-12


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_multi_slab_path(dtype, monkeypatch):
    """x/y passes split into many L2 slabs (tiny slab size) and several rhs,
    on a non-cubic external operator."""
    monkeypatch.setenv("GILA_SLAB_BYTES", "2048")
    gila = load_pkg()
    case = ((8, 6, 4), (6, 10, 8), ("13/32", 0, 0), (0, 0, 0))
    mix, fur, mem = _build(gila, case, dtype)
    n = 3
    xs = [seeded_current(mix.src_cel, 40 + k).astype(dtype) for k in range(n)]
    X = np.asfortranarray(np.stack(xs, axis=-1))
    Y = np.empty((*mix.trg_cel, 3, n), dtype=dtype, order="F")
    mem.apply_into(X, Y, nrhs=n)
    tol = TOL_F64 if dtype == np.complex128 else TOL_F32
    om = OprMem(mix, [f.astype(dtype).astype(np.complex128) for f in fur])
    for k in range(n):
        assert rel_l2(Y[..., k], ego_opr(om, xs[k].astype(np.complex128))) <= tol


def test_golden_fixtures_gpu():
    """The committed oracle fixtures (tests/golden) through the C ABI."""
    import glob
    import os
    from fractions import Fraction
    from conftest import ROOT
    gila = load_pkg()
    files = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))
    assert files
    for f in files:
        d = np.load(f)
        trg = gila.GlaVol(tuple(int(v) for v in d["trg_cel"]), SCL, tuple(Fraction(s) for s in d["trg_org"]))
        src = None if bool(d["is_self"]) else gila.GlaVol(tuple(int(v) for v in d["src_cel"]), SCL,
                                                          tuple(Fraction(s) for s in d["src_org"]))
        for dtype, tol in ((np.complex128, TOL_F64), (np.complex64, TOL_F32)):
            mem = gila.GlaOprMem(gila.GlaKerOpt(True), trg, src, egoFur=[d[f"fur{e}"].astype(dtype) for e in range(8)],
                                 setTyp=dtype)
            y = gila.egoOpr(mem, np.asfortranarray(d["x"].astype(dtype)))
            assert rel_l2(y, d["y"]) <= tol, (f, dtype)


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
@pytest.mark.parametrize("cels", [((8, 8, 8), (4, 4, 4)), ((8, 4, 8), (4, 4, 4)), ((4, 8, 8), (4, 4, 4)),
                                  ((64, 64, 64), (32, 32, 32))],
                         ids=lambda c: f"{c[0]}<-{c[1]}")
def test_target_partitions(dtype, cels):
    """Mixed cell scales (src/glaMem.jl:190-216): a target grid finer than
    the source splits into target partitions (genPrt / mrgPrt,
    src/glaActSup.jl:4-68, 939-1004); egoOpr! takes a source-partition-sized
    input and scatters each target partition back into the full target.
    External operators store the full spectrum, so any seeded kernel values
    exercise the same code paths."""
    from oracle.gla_mem import Vol, mix_for, tru_inf
    gila = load_pkg()
    tcel, scel = cels
    tscl = tuple(f"1/{64 if t == 2 * s else 32}" for t, s in zip(tcel, scel))
    trg = Vol.make(tcel, tscl, ("12/32", 0, 0))
    src = Vol.make(scel, SCL, (0, 0, 0))
    trg, src, mix, is_self = mix_for(trg, src)
    assert not is_self and np.prod(mix.trg_div) > 1
    tru = tru_inf(trg, src, mix)
    par_t = int(np.prod(mix.trg_div))
    rng = np.random.default_rng(5)
    fur = [np.asfortranarray(rng.standard_normal((*tru, 6, 1, par_t)) + 1j * rng.standard_normal((*tru, 6, 1, par_t)))
           for _ in range(8)]
    mem = gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(tcel, tscl, ("12/32", 0, 0)), gila.GlaVol(scel, SCL),
                         egoFur=[f.astype(dtype) for f in fur], setTyp=dtype)
    x = np.asfortranarray(seeded_current(mix.src_cel, 9).astype(dtype))
    y = gila.egoOpr(mem, x)
    assert tuple(y.shape) == (*tcel, 3)
    ref = ego_opr(OprMem(mix, [f.astype(dtype).astype(np.complex128) for f in fur]), x.astype(np.complex128))
    tol = TOL_F64 if dtype == np.complex128 else TOL_F32
    assert rel_l2(y, ref) <= tol


def test_source_partitions_rejected():
    """A source grid finer than the target (several source partitions):
    egoOpr! checks the input against the partition size and then cannot
    split it into partitions (src/glaAct.jl:37-49 with the reshape of
    egoBrnHst!), so the reference errors; the library reports GILA_ERR_SIZE."""
    from oracle.gla_mem import Vol, mix_for, tru_inf
    gila = load_pkg()
    tcel, scel = (4, 4, 4), (8, 8, 8)
    sscl = ("1/64", "1/64", "1/64")
    trg, src, mix, _ = mix_for(Vol.make(tcel, SCL, ("12/32", 0, 0)), Vol.make(scel, sscl, (0, 0, 0)))
    par_s = int(np.prod(mix.src_div))
    assert par_s > 1
    tru = tru_inf(trg, src, mix)
    rng = np.random.default_rng(6)
    fur = [np.asfortranarray(rng.standard_normal((*tru, 6, par_s, 1)) + 0j) for _ in range(8)]
    x = np.asfortranarray(seeded_current(mix.src_cel, 3))
    with pytest.raises(ValueError):
        ego_opr(OprMem(mix, fur), x)
    mem = gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(tcel, SCL, ("12/32", 0, 0)), gila.GlaVol(scel, sscl),
                         egoFur=fur)
    with pytest.raises(gila.GilaError):
        gila.egoOpr(mem, x)
