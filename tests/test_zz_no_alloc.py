"""The allocation-free matvec entry point, gila_opr_apply_noalloc.

It serves callers that cannot let the library allocate device memory while a
matvec runs -- hosts whose memory pool owns the whole device, loops that forbid
allocation after start-up -- by keeping the scratch between the passes in a
fixed 64 MiB device array.  These tests call it through the C ABI and compare
its output, on two calls in a row, with the regular entry point
gila_opr_apply on the same operator and input: the two run the same kernels on
the same lines, so the results must be bit-identical; the first call is also
checked against the FP64 oracle.  The file is named to be collected last, and
passes both on its own in a fresh process and after the other tests.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import pytest

from conftest import TOL_F32, TOL_F64, load_pkg, rel_l2
from oracle.matvec import OprMem, ego_opr
from oracle.synth import seeded_current, synth_operator

pytestmark = pytest.mark.gpu

SCL = ("1/32", "1/32", "1/32")


def _opr(gila, case, dtype):
    tc, sc, to, so = case
    mix, fur, _, is_self, trg, src = synth_operator(tc, SCL, to, sc, so)
    tv = gila.GlaVol(trg.cel, trg.scl, trg.org)
    sv = None if is_self else gila.GlaVol(src.cel, src.scl, src.org)
    mem = gila.GlaOprMem(gila.GlaKerOpt(True), tv, sv, egoFur=[f.astype(dtype) for f in fur], setTyp=dtype)
    return mix, mem, fur


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
@pytest.mark.parametrize("case", [((12, 10, 8), None, (0, 0, 0), None),
                                  ((8, 6, 4), (6, 10, 8), ("13/32", 0, 0), (0, 0, 0))],
                         ids=["self", "external"])
def test_noalloc_matches_apply_twice(case, dtype):
    import torch
    gila = load_pkg()
    lib = gila._lib.lib()
    mix, mem, fur = _opr(gila, case, dtype)
    tdt = torch.complex128 if dtype == np.complex128 else torch.complex64
    code = gila._lib.GILA_C128 if dtype == np.complex128 else gila._lib.GILA_C64
    x = seeded_current(mix.src_cel, 21).astype(dtype)
    xt = torch.from_numpy(np.ascontiguousarray(x.transpose(3, 2, 1, 0))).cuda()
    tc = mix.trg_cel
    ref = torch.empty((3, tc[2], tc[1], tc[0]), dtype=tdt, device="cuda")
    st = lib.gila_opr_apply(mem._h, code, ct.c_void_p(xt.data_ptr()), xt.numel(), ct.c_void_p(ref.data_ptr()),
                            ref.numel(), 1, None)
    assert st == 0, gila._lib.last_error()
    tol = TOL_F64 if dtype == np.complex128 else TOL_F32
    want = ego_opr(OprMem(mix, [f.astype(dtype).astype(np.complex128) for f in fur]), x.astype(np.complex128))
    for k in range(2):
        out = torch.full_like(ref, float("nan"))
        st = lib.gila_opr_apply_noalloc(mem._h, code, ct.c_void_p(xt.data_ptr()), xt.numel(),
                                        ct.c_void_p(out.data_ptr()), out.numel(), None)
        assert st == 0, gila._lib.last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref), f"call {k}: differs from gila_opr_apply"
        if k == 0:
            got = out.cpu().numpy().reshape(-1).reshape((*tc, 3), order="F")
            assert rel_l2(got, want) <= tol
    # on a caller's stream: enqueued there, the caller synchronises
    side = torch.cuda.Stream()
    out = torch.full_like(ref, float("nan"))
    torch.cuda.synchronize()
    st = lib.gila_opr_apply_noalloc(mem._h, code, ct.c_void_p(xt.data_ptr()), xt.numel(),
                                    ct.c_void_p(out.data_ptr()), out.numel(), ct.c_void_p(side.cuda_stream))
    assert st == 0, gila._lib.last_error()
    side.synchronize()
    assert torch.equal(out, ref)


def test_noalloc_rejects_oversize_and_host_vectors():
    import torch
    gila = load_pkg()
    lib = gila._lib.lib()
    # a 96^3 ComplexF64 self operator needs 3*96*192*192 complex doubles
    # (170 MiB) for its padded spectrum alone: more than the 64 MiB scratch
    cel = (96, 96, 96)
    tru = [49, 49, 49]
    rng = np.random.default_rng(0)
    fur = [np.asfortranarray(rng.standard_normal((*tru, 6, 1, 1)) + 0j) for _ in range(8)]
    mem = gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(cel, SCL), egoFur=fur, setTyp=np.complex128)
    x = torch.zeros((3, *cel), dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    st = lib.gila_opr_apply_noalloc(mem._h, gila._lib.GILA_C128, ct.c_void_p(x.data_ptr()), x.numel(),
                                    ct.c_void_p(y.data_ptr()), y.numel(), None)
    assert st == gila._lib.GILA_ERR_SIZE
    assert "too large" in gila._lib.last_error()
    # host vectors are refused (staging them would need device buffers)
    mix, small, _ = _opr(gila, ((4, 4, 4), None, (0, 0, 0), None), np.complex128)
    xh = np.zeros((4, 4, 4, 3), dtype=np.complex128, order="F")
    yh = np.zeros_like(xh)
    st = lib.gila_opr_apply_noalloc(small._h, gila._lib.GILA_C128, ct.c_void_p(xh.ctypes.data), xh.size,
                                    ct.c_void_p(yh.ctypes.data), yh.size, None)
    assert st == gila._lib.GILA_ERR_ARG
