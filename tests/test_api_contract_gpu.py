"""The operator API contract of test/oprTest.jl, through the C ABI.

The reference's generic_tests (test/oprTest.jl:15-55) run on its self,
external and merged operators (test/oprTest.jl:57-99; volumes of
test/runtests.jl:8-29: 16^3 cells of 1/50 wavelength, the external pair
touching along y, the merged volume 16x32x16).  Here the same operators are
built on the GPU, in both precisions, and every assertion of generic_tests and
of the per-operator testsets is made:
  * eltype is complex; G * x on the 4-D and on the flat input equals egoOpr!
    on a copy (same kernels, so bit-identical here, where the reference asks
    for isapprox); neither input is mutated;
  * a vector of the other complex type raises AssertionError, a vector one
    element too long raises DimensionMismatch;
  * adjoint(adjoint(G)) has the same egoFur and the same action, isadjoint
    flips; issymmetric / isposdef / ishermitian / isdiag are false;
  * size, glaSze, isselfoperator, isexternaloperator per operator;
  * a non-complex setTyp raises ArgumentError (test/oprTest.jl:4-5).
Device (CUDA tensor) inputs are checked against the host result as the
reference's device testsets do (test/oprTest.jl:81-99).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_pkg

pytestmark = pytest.mark.gpu

SCL = ("1/50", "1/50", "1/50")
CEL = (16, 16, 16)
CEL_U = (16, 32, 16)


def _ops(gila, dtype):
    return {
        "self": gila.GlaOpr(CEL, SCL, (0, 0, 0), setTyp=dtype),
        # GlaOprMem(cmpInf, volB, volA): target volB at y = 16/50, source volA
        "external": gila.GlaOpr(CEL, SCL, (0, 0, 0), CEL, SCL, (0, "16/50", 0), setTyp=dtype),
        "merge": gila.GlaOpr(CEL_U, SCL, (0, 0, 0), setTyp=dtype),
    }


EXPECT = {
    "self": ((16 * 16 * 16 * 3, 16 * 16 * 16 * 3), ((16, 16, 16, 3), (16, 16, 16, 3)), True),
    "external": ((16 * 16 * 16 * 3, 16 * 16 * 16 * 3), ((16, 16, 16, 3), (16, 16, 16, 3)), False),
    "merge": ((16 * 32 * 16 * 3, 16 * 32 * 16 * 3), ((16, 32, 16, 3), (16, 32, 16, 3)), True),
}


@pytest.fixture(scope="module", params=[np.complex64, np.complex128], ids=["c64", "c128"])
def operators(request):
    gila = load_pkg()
    return gila, request.param, _ops(gila, request.param)


def test_non_complex_settyp_is_argument_error():
    gila = load_pkg()
    with pytest.raises(gila.ArgumentError):
        gila.GlaOpr((1, 1, 1), (1, 1, 1), (0, 0, 0), setTyp=np.float64)


@pytest.mark.parametrize("name", ["self", "external", "merge"])
def test_operator_testset(operators, name):
    gila, dtype, ops = operators
    opr = ops[name]
    size, sze, is_self = EXPECT[name]
    assert gila.size(opr) == size
    assert gila.glaSze(opr) == sze
    assert gila.isselfoperator(opr) is is_self
    assert gila.isexternaloperator(opr) is (not is_self)
    assert np.dtype(gila.eltype(opr)) == np.dtype(dtype)


@pytest.mark.parametrize("name", ["self", "external", "merge"])
def test_generic_tests(operators, name):
    gila, dtype, ops = operators
    opr = ops[name]
    assert np.dtype(gila.eltype(opr)).kind == "c"
    x = np.ones(gila.size(opr, 2), dtype=dtype)
    x4 = np.reshape(x, gila.glaSze(opr, 2), order="F")
    ref = gila.egoOpr(opr.mem, np.array(x4, order="F", copy=True))
    acted4 = opr * x4
    assert acted4.shape == gila.glaSze(opr, 1)
    assert np.array_equal(acted4, ref)
    assert np.array_equal(x4, np.reshape(np.ones(gila.size(opr, 2), dtype=dtype), gila.glaSze(opr, 2), order="F"))
    acted = opr * x
    assert acted.ndim == 1 and np.array_equal(acted, np.reshape(ref, -1, order="F"))
    assert np.array_equal(x, np.ones(gila.size(opr, 2), dtype=dtype))
    other = np.complex128 if dtype == np.complex64 else np.complex64
    with pytest.raises(AssertionError):
        opr * np.ones(gila.size(opr, 2), dtype=other)
    with pytest.raises(gila.DimensionMismatch):
        opr * np.ones(gila.size(opr, 2) + 1, dtype=dtype)
    adj = gila.adjoint(opr)
    adj_adj = gila.adjoint(adj)
    for a, b in zip(adj_adj.mem.egoFur, opr.mem.egoFur):
        assert np.array_equal(a, b)
    assert np.array_equal(adj_adj * x, opr * x)
    assert gila.isadjoint(opr) is False
    assert gila.isadjoint(adj) is True
    assert gila.issymmetric(opr) is False
    assert gila.isposdef(opr) is False
    assert gila.ishermitian(opr) is False
    assert gila.isdiag(opr) is False


@pytest.mark.parametrize("name", ["external", "merge"])
def test_device_inputs_match_host(operators, name):
    import torch
    gila, dtype, ops = operators
    opr = ops[name]
    rng = np.random.default_rng(5)
    cel = gila.glaSze(opr, 2)[:3]
    x4 = np.asfortranarray((rng.standard_normal((*cel, 3)) + 1j * rng.standard_normal((*cel, 3))).astype(dtype))
    host = opr * x4
    xt = torch.from_numpy(np.ascontiguousarray(x4.reshape(-1, order="F"))).cuda()
    keep = xt.clone()
    dev = opr * xt
    assert dev.is_cuda and torch.equal(xt, keep)
    assert np.array_equal(dev.cpu().numpy(), np.reshape(host, -1, order="F"))
