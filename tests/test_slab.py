"""Slab-decomposed matvec (SlabOpr): the plan and the two all-to-all
exchanges, run as real torch.distributed ranks (gloo, world size 2 and 3) on
the CPU.

The three per-rank pieces are the GPU library's on a GPU; here numpy
stand-ins with the same data contract (x/y spectra of source planes, the z
pass of a row range with the operator's kernel at the global row, inverse
x/y of target planes) compute a generic circulant operator y =
crop(IFFT3(K . FFT3(pad(x)))), so that what is checked is the slab
bookkeeping: every rank's target planes equal those of the whole-volume
computation, with uneven slabs and ranks that hold no planes.  The GPU
pieces themselves are checked against the single-GPU matvec in
tests/test_slab_gpu.py."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from conftest import load_pkg


class NumpyPieces:
    """CPU stand-ins for gila_opr_slab_fwd / _z / _inv."""

    def __init__(self, src_cel, trg_cel, K):
        self.src_cel, self.trg_cel, self.K = tuple(src_cel), tuple(trg_cel), K
        Pz, Py, Px = K.shape[:3]
        self.dims = (Px, Py, Pz, src_cel[2], trg_cel[2])

    def fwd(self, x, B):
        a = x.numpy()
        pad = np.zeros(a.shape[:2] + B.shape[2:], dtype=a.dtype)
        pad[:, :, :a.shape[2], :a.shape[3]] = a
        B.copy_(torch.from_numpy(np.fft.fft2(pad, axes=(2, 3)).astype(a.dtype)))

    def z(self, Bz, ky0, nky):
        Px, Py, Pz, nin, nout = self.dims
        b = Bz.numpy()
        src = b[:3 * nin * nky * Px].reshape(3, nin, nky, Px).copy()
        pad = np.zeros((3, Pz, nky, Px), dtype=b.dtype)
        pad[:, :nin] = src
        f = np.fft.fft(pad, axis=1)
        k = self.K[:, ky0:ky0 + nky]  # [Pz, nky, Px, 3, 3]
        g = np.einsum("zyxij,jzyx->izyx", k, f)
        out = np.fft.ifft(g, axis=1)[:, :nout]
        b[:3 * nout * nky * Px] = out.astype(b.dtype).reshape(-1)

    def inv(self, B, y):
        a = np.fft.ifft2(B.numpy(), axes=(2, 3))
        y.copy_(torch.from_numpy(a[:, :, :y.shape[2], :y.shape[3]].astype(y.numpy().dtype)))


def make_case(src_cel, trg_cel, seed):
    P = [s + t for s, t in zip(src_cel, trg_cel)]
    rng = np.random.default_rng(seed)
    K = rng.standard_normal((P[2], P[1], P[0], 3, 3)) + 1j * rng.standard_normal((P[2], P[1], P[0], 3, 3))
    K = K + np.swapaxes(K, -1, -2)
    x = rng.standard_normal((3, src_cel[2], src_cel[1], src_cel[0])) + \
        1j * rng.standard_normal((3, src_cel[2], src_cel[1], src_cel[0]))
    return K, x


def whole_volume(K, x, trg_cel):
    P = K.shape[:3]
    pad = np.zeros((3,) + P, dtype=complex)
    pad[:, :x.shape[1], :x.shape[2], :x.shape[3]] = x
    f = np.fft.fftn(pad, axes=(1, 2, 3))
    g = np.einsum("zyxij,jzyx->izyx", K, f)
    y = np.fft.ifftn(g, axes=(1, 2, 3))
    return y[:, :trg_cel[2], :trg_cel[1], :trg_cel[0]]


CASES = [((5, 4, 7), (5, 4, 7)),   # self-like, 7 planes over 2 or 3 ranks
         ((4, 3, 5), (3, 4, 6)),   # external-like, source and target differ
         ((3, 3, 2), (4, 2, 1))]   # fewer planes than ranks


def _rank(rank, world, port, src_cel, trg_cel):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        gila = load_pkg()
        K, x = make_case(src_cel, trg_cel, 7)
        pieces = NumpyPieces(src_cel, trg_cel, K)
        op = gila.SlabOpr(None, pieces=pieces)
        z0, nz = op.source_planes
        y = op.apply(torch.from_numpy(np.ascontiguousarray(x[:, z0:z0 + nz])))
        t0, nt = op.target_planes
        want = whole_volume(K, x, trg_cel)[:, t0:t0 + nt]
        assert tuple(y.shape) == (3, nt, trg_cel[1], trg_cel[0])
        err = np.abs(y.numpy() - want).max() / np.abs(want).max() if nt else 0.0
        assert err < 1e-12, (rank, err)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", CASES, ids=["self", "external", "few-planes"])
def test_slab_exchange_matches_whole_volume(world, case):
    mp.spawn(_rank, args=(world, _free_port(), case[0], case[1]), nprocs=world, join=True)


def test_slab_ranges_and_plan():
    gila = load_pkg()
    assert gila.slab_ranges(7, 3) == [(0, 3), (3, 2), (5, 2)]
    assert gila.slab_ranges(2, 3) == [(0, 1), (1, 1), (2, 0)]
    assert gila.slab_ranges(8, 1) == [(0, 8)]
    with pytest.raises(ValueError):
        gila.slab_ranges(4, 0)
    pl = gila.SlabPlan((10, 8, 14, 7, 6), 3)
    assert sum(n for _, n in pl.zs) == 7 and sum(n for _, n in pl.zt) == 6 and sum(n for _, n in pl.ky) == 8
    assert pl.row_buffer_len(0) == 3 * 7 * 3 * 10


def test_in_process_decomposition_matches_whole_volume():
    """slab_apply_local (the single-device form the GPU test uses) with the
    numpy pieces, 1 to 4 ranks."""
    gila = load_pkg()
    for src_cel, trg_cel in CASES:
        K, x = make_case(src_cel, trg_cel, 3)
        want = whole_volume(K, x, trg_cel)
        for world in (1, 2, 3, 4):
            y = gila.slab_apply_local(NumpyPieces(src_cel, trg_cel, K), torch.from_numpy(x), world)
            assert np.abs(y.numpy() - want).max() <= 1e-12 * np.abs(want).max()
