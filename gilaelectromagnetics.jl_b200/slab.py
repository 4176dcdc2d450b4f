"""Slab-decomposed matvec: one Green operator applied across the GPUs of a
process group (one process per GPU), for volumes whose vectors and padded
spectrum do not fit one GPU.

The reference runs a volume on one device (src/glaAct.jl:191-321) and has no
counterpart.  Each rank builds the same operator (GlaOprMem: the whole
Fourier kernel) on its own GPU and keeps

  * source z planes  zs[r] of the input vector,
  * target z planes  zt[r] of the output vector,
  * spectrum rows    ky[r] between the passes,

contiguous near-equal ranges in rank order (slab_ranges).  One matvec is the
library's three slab pieces with two all-to-all exchanges between them
(NCCL over NVLink through torch.distributed; every remote chunk lands in the
receiving GPU's own memory before the next piece reads it):

  1. gila_opr_slab_fwd   x and y passes of the rank's source planes;
  2. all-to-all          rank s receives rows ky[s] of every rank's planes,
                         i.e. the whole source z extent of its rows;
  3. gila_opr_slab_z     the fused z pass of the rank's rows;
  4. all-to-all          rank r receives target planes zt[r] of every rank's
                         rows;
  5. gila_opr_slab_inv   inverse y and x passes of the rank's target planes.

The pieces run gila_opr_apply's per-line arithmetic with the operator's
launch choices, so the result equals the single-GPU matvec bit for bit once
the operator has been applied (or autotuned) on each rank.  One exchange per
component and direction keeps every received chunk in place: the chunks of a
component arrive in rank order, which is z order (forward) or row order
(inverse).
"""
from __future__ import annotations

import ctypes as ct
from typing import List, Optional, Sequence, Tuple

from . import _lib as L

__all__ = ["slab_ranges", "SlabPlan", "SlabPieces", "SlabOpr", "slab_apply_local"]


def slab_ranges(n: int, parts: int) -> List[Tuple[int, int]]:
    """(start, count) of `parts` contiguous ranges covering range(n), the
    first n % parts one longer (ranges may be empty when parts > n)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    base, extra = divmod(int(n), int(parts))
    out, s = [], 0
    for r in range(parts):
        k = base + (1 if r < extra else 0)
        out.append((s, k))
        s += k
    return out


class SlabPlan:
    """Which planes and rows each of `world` ranks holds, for an operator
    with padded lengths (Px, Py, Pz), nin source and nout target z planes."""

    def __init__(self, dims: Sequence[int], world: int):
        self.Px, self.Py, self.Pz, self.nin, self.nout = (int(d) for d in dims)
        self.world = int(world)
        self.zs = slab_ranges(self.nin, world)
        self.zt = slab_ranges(self.nout, world)
        self.ky = slab_ranges(self.Py, world)
        self.nzmax = max(self.nin, self.nout)

    # -- chunk layout shared by the distributed and the in-process exchange --
    def fwd_chunks(self, B, c: int):
        """Chunks of component c of a rank's forward spectra B [3, nz, Py,
        Px] for each destination rank s: rows ky[s] of every plane."""
        return [B[c, :, k0:k0 + nk, :] for (k0, nk) in self.ky]

    def z_input(self, Bz, c: int, s: int):
        """Component c's source planes in rank s's row buffer, as [nin, nky,
        Px]; rank r's chunk fills planes zs[r]."""
        nky = self.ky[s][1]
        n = self.nin * nky * self.Px
        return Bz[c * n:(c + 1) * n].view(self.nin, nky, self.Px)

    def z_output(self, Bz, c: int, s: int):
        """Component c's target planes in rank s's row buffer, [nout, nky,
        Px]; planes zt[r] go to rank r."""
        nky = self.ky[s][1]
        n = self.nout * nky * self.Px
        return Bz[c * n:(c + 1) * n].view(self.nout, nky, self.Px)

    def row_buffer_len(self, s: int) -> int:
        return 3 * self.nzmax * self.ky[s][1] * self.Px


class SlabPieces:
    """The three slab pieces of one operator on this process's GPU (the C
    ABI's gila_opr_slab_fwd / _z / _inv on the current torch stream)."""

    def __init__(self, mem):
        self.mem = mem
        d = (ct.c_int64 * 5)()
        _check(L.lib().gila_opr_slab_dims(mem._h, d))
        self.dims = tuple(int(v) for v in d)
        self.src_cel = tuple(mem.inSze[:3])
        self.trg_cel = tuple(mem.outSze[:3])
        self.code = mem._code

    def _stream(self, t):
        import torch
        return ct.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)

    def fwd(self, x, B):
        """x: [3, nz, Ny, Nx] source planes; B: [3, nz, Py, Px] out."""
        _check(L.lib().gila_opr_slab_fwd(self.mem._h, self.code, ct.c_void_p(x.data_ptr()), int(x.shape[1]),
                                         ct.c_void_p(B.data_ptr()), self._stream(x)))

    def z(self, Bz, ky0: int, nky: int):
        _check(L.lib().gila_opr_slab_z(self.mem._h, self.code, ct.c_void_p(Bz.data_ptr()), int(ky0), int(nky),
                                       self._stream(Bz)))

    def inv(self, B, y):
        """B: [3, nz, Py, Px] target-plane spectra; y: [3, nz, Nyt, Nxt] out."""
        _check(L.lib().gila_opr_slab_inv(self.mem._h, self.code, ct.c_void_p(B.data_ptr()), int(B.shape[1]),
                                         ct.c_void_p(y.data_ptr()), self._stream(B)))


def _check(status: int):
    from . import _check as chk
    chk(status)


def _real(t):
    import torch
    return torch.view_as_real(t).reshape(-1)


class SlabOpr:
    """One operator's matvec split over the ranks of a torch.distributed
    process group (NCCL for GPUs; any backend with all_to_all_single).

    SlabOpr(mem, group=None): `mem` is this rank's GlaOprMem (the same
    operator on every rank).  apply(x) takes this rank's source planes,
    x[:, k] = z plane source_planes[0] + k of the reference layout, as a
    contiguous [3, nz, Ny, Nx] complex tensor on this rank's GPU, and returns
    this rank's target planes [3, nzt, Nyt, Nxt].  Every rank calls apply
    with the same sequence of operators (two collectives per component)."""

    def __init__(self, mem, group=None, pieces=None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.pieces = pieces if pieces is not None else SlabPieces(mem)
        self.plan = SlabPlan(self.pieces.dims, self.world)

    @property
    def source_planes(self) -> Tuple[int, int]:
        return self.plan.zs[self.rank]

    @property
    def target_planes(self) -> Tuple[int, int]:
        return self.plan.zt[self.rank]

    @property
    def rows(self) -> Tuple[int, int]:
        return self.plan.ky[self.rank]

    def apply(self, x):
        import torch
        import torch.distributed as dist
        pl, r, pc = self.plan, self.rank, self.pieces
        Px, Py = pl.Px, pl.Py
        nzs, nzt, (ky0, nky) = pl.zs[r][1], pl.zt[r][1], pl.ky[r]
        Nx, Ny = pc.src_cel[0], pc.src_cel[1]
        Nxt, Nyt = pc.trg_cel[0], pc.trg_cel[1]
        if tuple(x.shape) != (3, nzs, Ny, Nx) or not x.is_contiguous():
            raise ValueError(f"rank {r}: source planes must be a contiguous [3, {nzs}, {Ny}, {Nx}] tensor")
        opts = dict(dtype=x.dtype, device=x.device)
        B = torch.empty((3, nzs, Py, Px), **opts)
        if nzs:
            pc.fwd(x, B)
        Bz = torch.empty(pl.row_buffer_len(r), **opts)
        for c in range(3):
            send = torch.cat([ch.reshape(-1) for ch in pl.fwd_chunks(B, c)])
            recv = pl.z_input(Bz, c, r)
            dist.all_to_all_single(_real(recv), _real(send),
                                   output_split_sizes=[2 * n * nky * Px for (_, n) in pl.zs],
                                   input_split_sizes=[2 * nzs * nk * Px for (_, nk) in pl.ky], group=self.group)
        if nky:
            pc.z(Bz, ky0, nky)
        Bt = torch.empty((3, nzt, Py, Px), **opts)
        for c in range(3):
            send = pl.z_output(Bz, c, r)
            recv = torch.empty(nzt * Py * Px, **opts)
            dist.all_to_all_single(_real(recv), _real(send),
                                   output_split_sizes=[2 * nzt * nk * Px for (_, nk) in pl.ky],
                                   input_split_sizes=[2 * n * nky * Px for (_, n) in pl.zt], group=self.group)
            off = 0
            for (k0, nk) in pl.ky:
                Bt[c, :, k0:k0 + nk, :] = recv[off:off + nzt * nk * Px].view(nzt, nk, Px)
                off += nzt * nk * Px
        y = torch.empty((3, nzt, Nyt, Nxt), **opts)
        if nzt:
            pc.inv(Bt, y)
        return y


def slab_apply_local(pieces, x, world: int):
    """The slab decomposition of `world` ranks run in one process on one
    device: every rank's pieces in turn, the exchanges as copies between the
    ranks' buffers with the chunk layout SlabOpr sends.  x: the whole source
    vector [3, Nz, Ny, Nx]; returns the whole target vector [3, Nzt, Nyt,
    Nxt].  It checks the decomposition on a single GPU (no kernel of one
    rank waits for another's)."""
    import torch
    pl = SlabPlan(pieces.dims, world)
    Px, Py = pl.Px, pl.Py
    Nxt, Nyt = pieces.trg_cel[0], pieces.trg_cel[1]
    opts = dict(dtype=x.dtype, device=x.device)
    Bs = []
    for r in range(world):
        z0, nz = pl.zs[r]
        B = torch.empty((3, nz, Py, Px), **opts)
        if nz:
            pieces.fwd(x[:, z0:z0 + nz].contiguous(), B)
        Bs.append(B)
    Bz = [torch.empty(pl.row_buffer_len(s), **opts) for s in range(world)]
    for c in range(3):
        for r in range(world):
            chunks = pl.fwd_chunks(Bs[r], c)
            z0, nz = pl.zs[r]
            for s in range(world):
                pl.z_input(Bz[s], c, s)[z0:z0 + nz] = chunks[s]
    for s in range(world):
        k0, nk = pl.ky[s]
        if nk:
            pieces.z(Bz[s], k0, nk)
    y = torch.empty((3, pl.nout, Nyt, Nxt), **opts)
    for r in range(world):
        z0, nz = pl.zt[r]
        Bt = torch.empty((3, nz, Py, Px), **opts)
        for c in range(3):
            for s in range(world):
                k0, nk = pl.ky[s]
                Bt[c, :, k0:k0 + nk, :] = pl.z_output(Bz[s], c, s)[z0:z0 + nz]
        if nz:
            yr = torch.empty((3, nz, Nyt, Nxt), **opts)
            pieces.inv(Bt, yr)
            y[:, z0:z0 + nz] = yr
    return y
