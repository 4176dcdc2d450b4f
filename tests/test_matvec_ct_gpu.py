"""GPU matvec parity at the transform lengths with compile-time specialised
kernels (P = Nsrc + Ntrg in {64, 96, 128, 192, 256, 384, 512} per axis):
the fused z pass, the tile-width variants the autotuner picks among and the
FP32 line-pair / row-pair kernels, against the FP64 oracle on the same
kernel values."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import TOL_F32, TOL_F64, load_pkg, rel_l2
from oracle.matvec import OprMem, ego_opr
from oracle.synth import seeded_current, synth_operator

pytestmark = pytest.mark.gpu

SCL = ("1/32", "1/32", "1/32")

# (trg_cel, src_cel, trg_org): self when src_cel is None
CT_CASES = [
    ((32, 48, 32), None, (0, 0, 0)),        # P = 64, 96, 64
    ((64, 96, 48), None, (0, 0, 0)),        # 128, 192, 96
    ((128, 32, 64), None, (0, 0, 0)),       # 256, 64, 128
    ((192, 8, 24), None, (0, 0, 0)),        # 384, 16, 48
    ((256, 8, 16), None, (0, 0, 0)),        # 512, 16, 32
    ((8, 16, 256), None, (0, 0, 0)),        # z = 512
    ((16, 8, 192), None, (0, 0, 0)),        # z = 384
    ((16, 256, 8), None, (0, 0, 0)),        # y = 512
    ((64, 64, 32), (64, 64, 64), ("80/32", 0, 0)),  # external: 128, 128, 96
    ((16, 8, 128), None, (0, 0, 0)),        # z = 256
    ((16, 16, 48), (16, 16, 80), (0, 0, "100/32")),  # external z = 128, 80 source planes
    # equal x and y lengths: the fused x / y cluster pass
    ((32, 32, 16), None, (0, 0, 0)),        # 64, 64
    ((48, 48, 8), None, (0, 0, 0)),         # 96, 96
    ((96, 96, 8), None, (0, 0, 0)),         # 192, 192
    ((128, 128, 8), None, (0, 0, 0)),       # 256, 256
    ((192, 192, 4), None, (0, 0, 0)),       # 384, 384
    ((256, 256, 4), None, (0, 0, 0)),       # 512, 512
    ((40, 64, 8), (24, 64, 8), ("50/32", 0, 0)),  # external 64, 128 ... x != y
]


def _build(gila, case, dtype):
    tc, sc, to = case
    so = None if sc is None else (0, 0, 0)
    mix, fur, *_ = synth_operator(tc, SCL, to, sc, so, set_dtype=np.complex128)
    sv = None if sc is None else gila.GlaVol(sc, SCL, so)
    mem = gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(tc, SCL, to), sv,
                         egoFur=[f.astype(dtype) for f in fur], setTyp=dtype)
    ref = OprMem(mix, [f.astype(dtype).astype(np.complex128) for f in fur])
    return mix, mem, ref


@pytest.mark.parametrize("case", CT_CASES, ids=lambda c: f"{c[0]}<-{c[1]}")
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_ct_matvec_parity_all_tiles(case, dtype):
    gila = load_pkg()
    mix, mem, ref = _build(gila, case, dtype)
    x = np.asfortranarray(seeded_current(mix.src_cel, 17).astype(dtype))
    y_ref = ego_opr(ref, x.astype(np.complex128))
    tol = TOL_F64 if dtype == np.complex128 else TOL_F32
    # the autotuned launch, then every compiled y / z tile width
    outs = [gila.egoOpr(mem, x)]
    for z in (4, 8, 16):
        for yt in (4, 8, 16):
            mem.tiles = (0, 0, yt, z)
            if mem.tiles[2:] != (yt, z):
                continue
            outs.append(gila.egoOpr(mem, x))
    for y in outs:
        assert rel_l2(y, y_ref) <= tol
    # tiles change the launch shape only: bit-identical results
    for y in outs[1:]:
        assert np.array_equal(y, outs[0])


@pytest.mark.parametrize("case", [CT_CASES[1], ((64, 64, 8), None, (0, 0, 0))], ids=["xy-separate", "xy-fused"])
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_ct_multi_rhs(dtype, case):
    gila = load_pkg()
    mix, mem, ref = _build(gila, case, dtype)
    xs = [np.asfortranarray(seeded_current(mix.src_cel, 20 + k).astype(dtype)) for k in range(3)]
    X = np.asfortranarray(np.stack(xs, axis=-1))
    Y = mem.new_output(X[..., 0], nrhs=3)
    mem.apply_into(X, Y, nrhs=3)
    for k in range(3):
        assert np.array_equal(Y[..., k], gila.egoOpr(mem, xs[k]))


@pytest.mark.parametrize("case", [CT_CASES[1], CT_CASES[2], CT_CASES[6], CT_CASES[7], CT_CASES[14], CT_CASES[15],
                                  CT_CASES[8]], ids=lambda c: f"{c[0]}<-{c[1]}")
@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_ct_radix_orders(case, dtype):
    """Both radix orders of the x and y transforms (greedy, reversed): the
    same transform, so every combination matches the oracle."""
    gila = load_pkg()
    mix, mem, ref = _build(gila, case, dtype)
    x = np.asfortranarray(seeded_current(mix.src_cel, 23).astype(dtype))
    y_ref = ego_opr(ref, x.astype(np.complex128))
    tol = TOL_F64 if dtype == np.complex128 else TOL_F32
    for xr in (0, 1):
        for yr in (0, 1):
            mem.schedule = (xr, yr)
            assert mem.schedule == (xr, yr)
            assert rel_l2(gila.egoOpr(mem, x), y_ref) <= tol
    with pytest.raises(gila.GilaError):
        mem.schedule = (2, 0)


@pytest.mark.parametrize("case", [CT_CASES[1], CT_CASES[2], CT_CASES[10], ((64, 64, 64), None, (0, 0, 0))],
                         ids=lambda c: f"{c[0]}<-{c[1]}")
def test_ct_z_mirror_pairs(case, monkeypatch):
    """The fused z pass with one task per mirror pair of z frequencies (one
    kernel load for kz and P - kz) against one task per frequency, at every
    z tile: the same arithmetic, so bit-identical, and both on the oracle."""
    gila = load_pkg()
    mix, mem, ref = _build(gila, case, np.complex128)
    x = np.asfortranarray(seeded_current(mix.src_cel, 29).astype(np.complex128))
    y_ref = ego_opr(ref, x.astype(np.complex128))
    for z in (4, 8, 16):
        mem.tiles = (0, 0, 0, z)
        if mem.tiles[3] != z:
            continue
        outs = []
        for mode in ("0", "2"):
            monkeypatch.setenv("GILA_ZMIRROR", mode)
            outs.append(gila.egoOpr(mem, x))
        assert rel_l2(outs[1], y_ref) <= TOL_F64
        assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
def test_ct_batch_sizes_keep_results(dtype):
    """Launch shapes are re-picked per batch size of device-resident
    vectors, the radix schedule is not: an operator first used on one
    vector, then on batches of 4 and 2, keeps its schedule and gives every
    vector bit-identical results."""
    import torch

    gila = load_pkg()
    mix, mem, ref = _build(gila, CT_CASES[1], dtype)
    n = mix.src_cel
    xs = [np.asfortranarray(seeded_current(n, 40 + k).astype(dtype)) for k in range(4)]
    xd = torch.stack([torch.from_numpy(x.ravel(order="F").copy()).reshape(3, n[2], n[1], n[0]) for x in xs]).cuda()
    singles = []
    for k in range(4):
        y = torch.empty_like(xd[k])
        mem.apply_into(xd[k], y)
        singles.append(y)
    sched = mem.schedule
    for nb in (4, 2):
        Y = torch.empty_like(xd[:nb])
        mem.apply_into(xd[:nb].contiguous(), Y, nrhs=nb)
        assert mem.schedule == sched
        for k in range(nb):
            assert torch.equal(Y[k], singles[k])
    y0 = singles[0].cpu().numpy().reshape(-1)
    y_ref = ego_opr(ref, xs[0].astype(np.complex128)).ravel(order="F")
    assert rel_l2(y0, y_ref) <= (TOL_F64 if dtype == np.complex128 else TOL_F32)
