"""Slab pieces of the matvec on the GPU (gila_opr_slab_fwd / _z / _inv).

The decomposition of 1 to 5 ranks runs in one process on the one GPU
(slab_apply_local: every rank's pieces in turn, the exchanges as device
copies with SlabOpr's chunk layout), and must give the single-GPU matvec's
result bit for bit: the pieces run the same per-line arithmetic with the
operator's launch choices.  A one-rank NCCL process group runs SlabOpr's
own all-to-all path.  Bad arguments come back as errors."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, TOL_F32, TOL_F64, load_pkg, rel_l2
from oracle.matvec import OprMem, ego_opr
from oracle.synth import seeded_current, synth_operator

pytestmark = pytest.mark.gpu

SCL = ("1/32", "1/32", "1/32")
CASES = [((24, 20, 16), None, (0, 0, 0)),                 # self, generic lengths
         ((32, 32, 64), None, (0, 0, 0)),                 # self, specialised z = 128 (fused z kernel)
         ((16, 12, 10), (12, 16, 8), ("20/32", 0, 0)),    # external
         ((12, 10, 3), None, (0, 0, 0))]                  # fewer planes than ranks


def build_case(case, dtype, seed=5):
    import torch
    gila = load_pkg()
    tc, sc, to = case
    so = None if sc is None else (0, 0, 0)
    mix, fur, *_ = synth_operator(tc, SCL, to, sc, so, set_dtype=np.complex128)
    sv = None if sc is None else gila.GlaVol(sc, SCL, so)
    mem = gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(tc, SCL, to), sv,
                         egoFur=[f.astype(dtype) for f in fur], setTyp=dtype)
    x = seeded_current(mix.src_cel, seed).astype(dtype)
    xd = torch.from_numpy(np.ascontiguousarray(x.transpose(3, 2, 1, 0))).cuda()
    no = mem.outSze
    y_ref = torch.empty((3, no[2], no[1], no[0]), dtype=xd.dtype, device=xd.device)
    mem.apply_into(xd, y_ref)
    ref = OprMem(mix, [f.astype(dtype).astype(np.complex128) for f in fur])
    return mem, x, xd, y_ref, ref


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64], ids=["c128", "c64"])
@pytest.mark.parametrize("case", CASES, ids=["self", "self-z128", "external", "few-planes"])
def test_slab_decomposition_bit_identical(case, dtype):
    import torch
    gila = load_pkg()
    mem, x, xd, y_ref, ref = build_case(case, dtype)
    want = ego_opr(ref, x.astype(np.complex128))
    got = y_ref.cpu().numpy().transpose(3, 2, 1, 0)
    assert rel_l2(got, want) <= (TOL_F64 if dtype == np.complex128 else TOL_F32)
    pieces = gila.SlabPieces(mem)
    assert pieces.dims[3] == mem.inSze[2] and pieces.dims[4] == mem.outSze[2]
    for world in (1, 2, 3, 5):
        y = gila.slab_apply_local(pieces, xd, world)
        torch.cuda.synchronize()
        assert torch.equal(y, y_ref), world


CHILD = r"""
import json, os, sys
import torch, torch.distributed as dist
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np
from conftest import load_pkg
from test_slab_gpu import CASES, build_case
os.environ["MASTER_ADDR"] = "127.0.0.1"
os.environ["MASTER_PORT"] = "{port}"
torch.cuda.set_device(0)
dist.init_process_group("nccl", rank=0, world_size=1)
gila = load_pkg()
out = []
for dt in (np.complex128, np.complex64):
    mem, x, xd, y_ref, ref = build_case(CASES[0], dt)
    op = gila.SlabOpr(mem)
    y = op.apply(xd)
    torch.cuda.synchronize()
    out.append(bool(torch.equal(y, y_ref)))
dist.destroy_process_group()
print(json.dumps({{"equal": out}}))
"""


def test_slab_opr_nccl_one_rank():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    src = CHILD.format(root=ROOT, tests=os.path.join(ROOT, "tests"), port=port)
    r = subprocess.run([sys.executable, "-c", src], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, NCCL_NVLS_ENABLE="0"))
    assert r.returncode == 0, r.stderr[-3000:]
    assert json.loads(r.stdout.strip().splitlines()[-1])["equal"] == [True, True]


def test_slab_pieces_reject_bad_arguments():
    import torch
    gila = load_pkg()
    mem, x, xd, y_ref, ref = build_case(CASES[0], np.complex128)
    pieces = gila.SlabPieces(mem)
    Px, Py, Pz, nin, nout = pieces.dims
    lib = gila._lib.lib()
    B = torch.empty((3, 2, Py, Px), dtype=torch.complex128, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    import ctypes as ct
    # element type
    assert lib.gila_opr_slab_fwd(mem._h, gila._lib.GILA_C64, ct.c_void_p(xd.data_ptr()), 2,
                                 ct.c_void_p(B.data_ptr()), ct.c_void_p(st)) == gila._lib.GILA_ERR_TYPE
    # plane count and row range
    assert lib.gila_opr_slab_fwd(mem._h, gila._lib.GILA_C128, ct.c_void_p(xd.data_ptr()), nin + 1,
                                 ct.c_void_p(B.data_ptr()), ct.c_void_p(st)) == gila._lib.GILA_ERR_SIZE
    Bz = torch.empty(3 * max(nin, nout) * 4 * Px, dtype=torch.complex128, device="cuda")
    assert lib.gila_opr_slab_z(mem._h, gila._lib.GILA_C128, ct.c_void_p(Bz.data_ptr()), Py - 2, 4,
                               ct.c_void_p(st)) == gila._lib.GILA_ERR_SIZE
    # host memory
    h = np.zeros(3 * 2 * Py * Px, dtype=np.complex128)
    assert lib.gila_opr_slab_fwd(mem._h, gila._lib.GILA_C128, ct.c_void_p(xd.data_ptr()), 2,
                                 ct.c_void_p(h.ctypes.data), ct.c_void_p(st)) == gila._lib.GILA_ERR_ARG
    torch.cuda.synchronize()
