"""gila_b200 -- host-side mirror of the GilaElectromagnetics.jl operator API
over the C-ABI library libgila_b200.so (sm_100a CUDA).

The names, argument meanings and error behaviour follow the reference:

  GlaVol(cel, scl, org=(0,0,0), grdScl=scl)        src/glaMem.jl:136-148
  GlaKerOpt(useGpu) / GlaKerOpt(frqPhz, intOrd, adjMod, devMod, numTrd, numBlk)
                                                   src/glaMem.jl:62-70,226-233
  GlaOprMem(cmpInf, trgVol, srcVol=None, egoFur=None, setTyp=complex128)
                                                   src/glaMemSup.jl:16-171
  GlaOpr(cel, scl, org; useGpu, setTyp)            src/glaMemSup.jl:307-318
  GlaOpr(celSrc, sclSrc, orgSrc, celTrg, sclTrg, orgTrg; ...)
                                                   src/glaMemSup.jl:337-350
  egoOpr(mem, actVec)        (egoOpr!)             src/glaAct.jl:33-49
  opr * x, opr @ x           (Base.:*)             src/glaLinAlg.jl:33-57
  mul(out, opr, x, a, b)     (LinearAlgebra.mul!)  src/glaLinAlg.jl:61-69
  adjoint, isadjoint, isselfoperator, isexternaloperator, glaSze, size,
  eltype, issymmetric, isposdef, ishermitian, isdiag
                                                   src/glaLinAlg.jl, glaMemSup.jl:359-371
  LippmannSchwinger(G, medium), ls * x, mul(y, ls, x)
                                                   examples/GilaOperators.jl:57-96
  solve(ls, i)               BiCGStab(l) solve     examples/scattering_film.jl:58-61
  SolveServer                continuous-batching solve server (no reference counterpart)
  SlabOpr                    one matvec split over the GPUs of a process group
                             (slab decomposition; no reference counterpart)

Vectors use the reference's memory layout: (Nx, Ny, Nz, 3) column-major.
numpy arrays are passed as shape (Nx, Ny, Nz, 3) in Fortran order (or flat);
torch tensors as shape (3, Nz, Ny, Nx) contiguous (the same bytes), on the
CPU or on a CUDA device.  Every matvec runs on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as ct
import math
from fractions import Fraction
from typing import Optional, Sequence

import numpy as np

from . import _lib as L

__all__ = [
    "GlaVol", "GlaKerOpt", "GlaOprMem", "GlaOpr", "egoOpr", "mul", "adjoint", "isadjoint",
    "isselfoperator", "isexternaloperator", "glaSze", "size", "eltype", "issymmetric",
    "isposdef", "ishermitian", "isdiag", "GilaError", "DimensionMismatch", "ArgumentError",
    "Context", "default_context", "cast", "weak_integrals", "LippmannSchwinger", "solve", "SolveInfo", "SolveServer",
    "SlabOpr", "SlabPlan", "SlabPieces", "slab_ranges", "slab_apply_local",
]


class GilaError(RuntimeError):
    """Julia `error(...)` (ErrorException) raised by the reference."""


class DimensionMismatch(ValueError):
    """Julia DimensionMismatch."""


class ArgumentError(ValueError):
    """Julia ArgumentError."""


def _check(status: int, what: str = ""):
    if status == L.GILA_OK:
        return
    msg = L.last_error() or L.lib().gila_status_string(status).decode()
    if status == L.GILA_ERR_TYPE:
        raise AssertionError(msg)
    if status == L.GILA_ERR_ARG and what == "setTyp":
        raise ArgumentError(msg)
    raise GilaError(f"{msg} [status {status}]")


# ----------------------------------------------------------------- context
class Context:
    """One library context per CUDA device (streams, twiddle tables,
    launch-shape cache)."""

    def __init__(self, device: int = 0):
        h = ct.c_void_p()
        _check(L.lib().gila_ctx_create(int(device), ct.byref(h)))
        self.handle = h
        self.device = device

    def __del__(self):
        try:
            if self.handle:
                L.lib().gila_ctx_destroy(self.handle)
        except Exception:
            pass


_ctx: dict = {}


def default_context(device: int = 0) -> Context:
    if device not in _ctx:
        _ctx[device] = Context(device)
    return _ctx[device]


# ----------------------------------------------------------------- volumes
def _rat(v) -> Fraction:
    if isinstance(v, Fraction):
        return v
    if isinstance(v, str):
        return Fraction(v)
    if isinstance(v, float):
        return Fraction(v).limit_denominator(1 << 30)
    return Fraction(v)


class GlaVol:
    """GlaVol (src/glaMem.jl:12-19,136-148): cells, cell scale (in
    wavelengths, rational), centre `org`, and grid pitch `grd`."""

    def __init__(self, cel: Sequence[int], scl, org=(0, 0, 0), grdScl=None):
        self.cel = tuple(int(c) for c in cel)
        self.scl = tuple(_rat(s) for s in scl)
        self.org = tuple(_rat(o) for o in org)
        self.grd = self.scl if grdScl is None else tuple(_rat(g) for g in grdScl)
        if not all(s <= g for s, g in zip(self.scl, self.grd)):
            raise GilaError("The cell scale must be smaller than the grid scale to avoid "
                            "partially overlapping basis elements.")

    def __eq__(self, o):
        return isinstance(o, GlaVol) and (self.cel, self.scl, self.org, self.grd) == (o.cel, o.scl, o.org, o.grd)

    def __hash__(self):
        return hash((self.cel, self.scl, self.org, self.grd))

    def to_c(self) -> L.GilaVolC:
        v = L.GilaVolC()
        for k in range(3):
            v.cel[k] = self.cel[k]
            v.scl_num[k], v.scl_den[k] = self.scl[k].numerator, self.scl[k].denominator
            v.org_num[k], v.org_den[k] = self.org[k].numerator, self.org[k].denominator
            v.grd_num[k], v.grd_den[k] = self.grd[k].numerator, self.grd[k].denominator
        return v

    def __repr__(self):
        return f"GlaVol(cel={self.cel}, scl={tuple(str(s) for s in self.scl)}, org={tuple(str(o) for o in self.org)})"


class GlaKerOpt:
    """GlaKerOpt (src/glaMem.jl:62-70).  GlaKerOpt(True) gives the device
    defaults (frqPhz=1, intOrd=32, threads (128,2,1), blocks (1,128,256))."""

    def __init__(self, *args):
        if len(args) == 1:
            dev = bool(args[0])
            self.frqPhz = complex(1.0, 0.0)
            self.intOrd = 32
            self.adjMod = False
            self.devMod = dev
            self.numTrd = (128, 2, 1) if dev else ()
            self.numBlk = (1, 128, 256) if dev else ()
        elif len(args) == 6:
            self.frqPhz, self.intOrd, self.adjMod, self.devMod, self.numTrd, self.numBlk = args
            self.frqPhz = complex(self.frqPhz)
        else:
            raise TypeError("GlaKerOpt(devStt) or GlaKerOpt(frqPhz, intOrd, adjMod, devMod, numTrd, numBlk)")

    def to_c(self) -> L.GilaKoptC:
        o = L.GilaKoptC()
        o.frq_re, o.frq_im = self.frqPhz.real, self.frqPhz.imag
        o.int_ord = int(self.intOrd)
        o.adj_mod = int(bool(self.adjMod))
        o.dev_mod = 1
        for k, v in enumerate(tuple(self.numTrd)[:3]):
            o.num_trd[k] = int(v)
        for k, v in enumerate(tuple(self.numBlk)[:3]):
            o.num_blk[k] = int(v)
        return o

    def copy(self, **kw):
        o = GlaKerOpt(self.frqPhz, self.intOrd, self.adjMod, self.devMod, self.numTrd, self.numBlk)
        for k, v in kw.items():
            setattr(o, k, v)
        return o


def _dtype_code(t) -> int:
    t = np.dtype(t)
    if t == np.complex128:
        return L.GILA_C128
    if t == np.complex64:
        return L.GILA_C64
    raise ArgumentError("setTyp must be a subtype of Complex (complex64 or complex128)")


def _np_dtype(code: int):
    return np.dtype(np.complex128) if code == L.GILA_C128 else np.dtype(np.complex64)


# ----------------------------------------------------------------- buffers
def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _elem_code(x):
    """dtype code of a complex array / tensor, or None."""
    if _is_torch(x):
        import torch
        return {torch.complex128: L.GILA_C128, torch.complex64: L.GILA_C64}.get(x.dtype)
    a = np.asarray(x)
    return {np.dtype(np.complex128): L.GILA_C128, np.dtype(np.complex64): L.GILA_C64}.get(a.dtype)


def _buf(x):
    """(pointer, element count, dtype code, keepalive) of a numpy array or
    torch tensor holding complex data in the reference layout."""
    if _is_torch(x):
        import torch
        if not x.is_contiguous():
            raise GilaError("tensor must be contiguous")
        if x.dtype == torch.complex128:
            code = L.GILA_C128
        elif x.dtype == torch.complex64:
            code = L.GILA_C64
        else:
            raise AssertionError("Input array must have a complex element type.")
        return x.data_ptr(), x.numel(), code, x
    a = np.asarray(x)
    if not np.iscomplexobj(a) or a.dtype not in (np.complex64, np.complex128):
        raise AssertionError("Input array must have a complex element type.")
    if a.ndim > 1 and not a.flags.f_contiguous:
        a = np.asfortranarray(a)
    elif a.ndim <= 1 and not a.flags.c_contiguous:
        a = np.ascontiguousarray(a)
    return a.ctypes.data, a.size, _dtype_code(a.dtype), a


# ----------------------------------------------------------------- operator
class GlaOprMem:
    """GlaOprMem: device-resident Green operator (Fourier kernel, FFT
    plans, workspaces).

    GlaOprMem(cmpInf, trgVol, srcVol=None, egoFur=None, setTyp=complex128)
    mirrors src/glaMemSup.jl:16-20.  `egoFur` (list of 8 arrays in the
    reference layout (tx,ty,tz,6,parSrc,parTrg)) skips the kernel build."""

    def __init__(self, cmpInf: GlaKerOpt, trgVol: GlaVol, srcVol: Optional[GlaVol] = None, *,
                 egoFur=None, setTyp=np.complex128, ctx: Optional[Context] = None):
        code = _dtype_code(setTyp)
        self.ctx = ctx or default_context()
        self.cmpInf = cmpInf
        self.trgVol = trgVol
        self.srcVol = trgVol if srcVol is None else srcVol
        h = ct.c_void_p()
        tv = trgVol.to_c()
        sv = srcVol.to_c() if srcVol is not None else None
        opt = cmpInf.to_c()
        if egoFur is None:
            st = L.lib().gila_opr_create(self.ctx.handle, ct.byref(tv), ct.byref(sv) if sv else None,
                                         ct.byref(opt), code, ct.byref(h))
            _check(st)
        else:
            furs = [np.asfortranarray(np.asarray(f)) for f in egoFur]
            if len(furs) != 8:
                raise GilaError("egoFur must hold 8 parity branches")
            fdt = furs[0].dtype
            if fdt not in (np.complex64, np.complex128):
                raise ArgumentError("egoFur must be complex")
            furs = [f.astype(fdt, order="F", copy=False) for f in furs]
            ptrs = (ct.c_void_p * 8)(*[f.ctypes.data for f in furs])
            dims = ((ct.c_int64 * 6) * 8)()
            for eo, f in enumerate(furs):
                shp = list(f.shape) + [1] * (6 - f.ndim)
                for k in range(6):
                    dims[eo][k] = shp[k]
            st = L.lib().gila_opr_create_from_fur(self.ctx.handle, ct.byref(tv), ct.byref(sv) if sv else None,
                                                  ct.byref(opt), code, ptrs, dims, _dtype_code(fdt), ct.byref(h))
            _check(st)
        self._h = h
        self._fin_dims()

    @classmethod
    def _from_handle(cls, h, ctx, cmpInf, trgVol, srcVol):
        self = cls.__new__(cls)
        self._h, self.ctx, self.cmpInf, self.trgVol, self.srcVol = h, ctx, cmpInf, trgVol, srcVol
        self._fin_dims()
        return self

    def _fin_dims(self):
        lib = L.lib()
        t4 = (ct.c_int64 * 4)()
        s4 = (ct.c_int64 * 4)()
        _check(lib.gila_opr_sizes(self._h, t4, s4))
        self._trg_cel = tuple(t4[:3])
        self._src_cel = tuple(s4[:3])
        i4 = (ct.c_int64 * 4)()
        o4 = (ct.c_int64 * 4)()
        _check(lib.gila_opr_input_size(self._h, i4))
        _check(lib.gila_opr_output_size(self._h, o4))
        self.inSze = tuple(i4)
        self.outSze = tuple(o4)
        dt = ct.c_int()
        fl = ct.c_int32()
        _check(lib.gila_opr_info(self._h, ct.byref(dt), ct.byref(fl)))
        self._code = dt.value
        self._flags = fl.value

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                L.lib().gila_opr_destroy(self._h)
        except Exception:
            pass

    @property
    def dtype(self):
        return _np_dtype(self._code)

    @property
    def egoFur(self):
        """The 8 parity branches in the reference layout (host copies)."""
        dims = ((ct.c_int64 * 6) * 8)()
        _check(L.lib().gila_opr_fur_dims(self._h, dims))
        outs = [np.zeros(tuple(dims[eo][:]), dtype=self.dtype, order="F") for eo in range(8)]
        ptrs = (ct.c_void_p * 8)(*[o.ctypes.data for o in outs])
        _check(L.lib().gila_opr_export_fur(self._h, ptrs))
        return outs

    def save(self, path: str):
        """Write the operator's egoFur with its volumes and GlaKerOpt to a
        GILAFUR1 file (the kernel cache the reference keeps with Serialization
        / JLD2, test/runtests.jl:38-98, examples/GilaOperators.jl:28-55)."""
        _check(L.lib().gila_opr_save(self._h, str(path).encode()))

    @classmethod
    def load(cls, path: str, setTyp=np.complex128, ctx: Optional[Context] = None) -> "GlaOprMem":
        """The operator stored in a GILAFUR1 file, cast to setTyp."""
        ctx = ctx or default_context()
        h = ct.c_void_p()
        _check(L.lib().gila_opr_load(ctx.handle, str(path).encode(), _dtype_code(setTyp), ct.byref(h)))
        self = cls.__new__(cls)
        self._h, self.ctx = h, ctx
        self._fin_dims()
        hdr = np.fromfile(str(path), dtype=np.uint8, count=768)
        i32 = hdr[8:32].view("<i4")
        frq = hdr[32:48].view("<f8")
        vols = hdr[48:384].view("<i8").reshape(2, 7, 3)
        mk = lambda v: GlaVol(v[0], [Fraction(int(n), int(d)) for n, d in zip(v[1], v[2])],  # noqa: E731
                              [Fraction(int(n), int(d)) for n, d in zip(v[3], v[4])],
                              [Fraction(int(n), int(d)) for n, d in zip(v[5], v[6])])
        self.trgVol = mk(vols[0])
        self.srcVol = self.trgVol if i32[2] else mk(vols[1])
        self.cmpInf = GlaKerOpt(complex(frq[0], frq[1]), int(i32[4]), bool(i32[3]), True, (), ())
        return self

    def reserve(self, nrhs: int):
        _check(L.lib().gila_opr_reserve(self._h, int(nrhs)))

    def time_passes(self, nrhs: int = 1, reps: int = 5):
        """Device ms of one apply: (forward x/y, z pass, inverse y/x, total)."""
        ms = (ct.c_double * 4)()
        _check(L.lib().gila_opr_time_passes(self._h, int(nrhs), int(reps), ms))
        return tuple(ms)

    def autotune(self, nrhs: int = 1):
        """Time the compiled tile candidates for nrhs vectors and keep the
        fastest; returns (x-forward lines, x-inverse lines, y tile, z tile)."""
        t = (ct.c_int32 * 4)()
        _check(L.lib().gila_opr_autotune(self._h, int(nrhs), t))
        return tuple(t)

    @property
    def tiles(self):
        t = (ct.c_int32 * 4)()
        _check(L.lib().gila_opr_get_tiles(self._h, t))
        return tuple(t)

    @tiles.setter
    def tiles(self, v):
        t = (ct.c_int32 * 4)(*[int(a) for a in v])
        _check(L.lib().gila_opr_set_tiles(self._h, t))

    @property
    def schedule(self):
        """Radix order of the x and y transforms: (x, y), 0 greedy, 1 reversed."""
        t = (ct.c_int32 * 2)()
        _check(L.lib().gila_opr_get_schedule(self._h, t))
        return tuple(t)

    @schedule.setter
    def schedule(self, v):
        t = (ct.c_int32 * 2)(*[int(a) for a in v])
        _check(L.lib().gila_opr_set_schedule(self._h, t))

    def launches_per_apply(self, nrhs: int = 1) -> int:
        n = ct.c_int64()
        _check(L.lib().gila_opr_launches_per_apply(self._h, int(nrhs), ct.byref(n)))
        return n.value

    def device_bytes(self) -> int:
        v = ct.c_int64()
        _check(L.lib().gila_opr_device_bytes(self._h, ct.byref(v)))
        return v.value

    # -- raw application ----------------------------------------------------
    def apply_into(self, x, out, nrhs: int = 1, stream=None):
        """out = G x for nrhs stacked vectors (no allocation)."""
        xp, xn, xc, _ka = _buf(x)
        op, on, oc, _kb = _buf(out)
        if oc != self._code:
            raise AssertionError("output element type differs from the operator's")
        st = L.lib().gila_opr_apply(self._h, xc, ct.c_void_p(xp), xn, ct.c_void_p(op), on, int(nrhs),
                                    ct.c_void_p(stream) if stream else None)
        _check(st)
        if isinstance(_kb, np.ndarray) and _kb is not out:
            np.copyto(np.asarray(out), _kb.reshape(np.asarray(out).shape, order="F"))
        return out

    def axpby_into(self, alpha, x, beta, out, nrhs: int = 1, stream=None):
        """out = alpha * (G x) + beta * out."""
        xp, xn, xc, _ka = _buf(x)
        op, on, oc, _kb = _buf(out)
        if oc != self._code:
            raise AssertionError("output element type differs from the operator's")
        a = (ct.c_double * 2)(complex(alpha).real, complex(alpha).imag)
        b = (ct.c_double * 2)(complex(beta).real, complex(beta).imag)
        st = L.lib().gila_opr_apply_axpby(self._h, xc, a, ct.c_void_p(xp), xn, b, ct.c_void_p(op), on,
                                          int(nrhs), ct.c_void_p(stream) if stream else None)
        _check(st)
        if isinstance(_kb, np.ndarray) and _kb is not out:
            np.copyto(np.asarray(out), _kb.reshape(np.asarray(out).shape, order="F"))
        return out

    def new_output(self, like, nrhs: int = 1):
        shp = self.outSze
        if _is_torch(like):
            import torch
            s = (nrhs, 3, shp[2], shp[1], shp[0]) if nrhs > 1 else (3, shp[2], shp[1], shp[0])
            return torch.empty(s, dtype=like.dtype, device=like.device)
        s = (*shp[:3], 3, nrhs) if nrhs > 1 else (*shp[:3], 3)
        return np.empty(s, dtype=self.dtype, order="F")


def weak_integrals(scl, frqPhz: complex = 1.0 + 0j, intOrd: int = 32, ctx: Optional[Context] = None):
    """wekS, wekE, wekV (src/glaInt.jl:75-262) of a cell of size `scl` at
    Gauss-Legendre order intOrd, evaluated on the GPU: (wS[3], wE[9], wV[6])
    unscaled, as numpy complex arrays."""
    ctx = ctx or default_context()
    sr = [_rat(v) for v in scl]
    num = (ct.c_int64 * 3)(*[r.numerator for r in sr])
    den = (ct.c_int64 * 3)(*[r.denominator for r in sr])
    out = (ct.c_double * 36)()
    f = complex(frqPhz)
    _check(L.lib().gila_weak_integrals(ctx.handle, num, den, f.real, f.imag, int(intOrd), out))
    v = np.array(out[0::2]) + 1j * np.array(out[1::2])
    return v[:3], v[3:12], v[12:18]


def egoOpr(egoMem: GlaOprMem, actVec):
    """egoOpr!(egoMem, actVec) (src/glaAct.jl:33-49): returns G * actVec.

    The input must have the source partition size (srcCel..., 3): shape
    (Nx, Ny, Nz, 3) for numpy, (3, Nz, Ny, Nx) for torch.  Unlike the
    reference the input is left unmodified."""
    want = tuple(egoMem.inSze)
    shp = tuple(actVec.shape)
    ok = shp == want if not _is_torch(actVec) else shp == (3, want[2], want[1], want[0])
    if not ok:
        raise GilaError("Size of input vector does not match size of source volume. "
                        "Required data layout is (srcCelX, srcCelY, srcCelZ, 3).")
    out = egoMem.new_output(actVec)
    return egoMem.apply_into(actVec, out)


class GlaOpr:
    """GlaOpr (src/glaMem.jl:116-119) with the constructors of
    src/glaMemSup.jl:307-350 and the algebra of src/glaLinAlg.jl."""

    def __init__(self, *args, useGpu: bool = True, setTyp=np.complex128, ctx=None):
        if len(args) == 1 and isinstance(args[0], GlaOprMem):
            self.mem = args[0]
            return
        if not (np.dtype(setTyp).kind == "c"):
            raise ArgumentError("setTyp must be a subtype of Complex")
        opt = GlaKerOpt(True)
        if len(args) in (2, 3):
            cel, scl = args[0], args[1]
            org = args[2] if len(args) == 3 else (0, 0, 0)
            self.mem = GlaOprMem(opt, GlaVol(cel, scl, org), setTyp=setTyp, ctx=ctx)
        elif len(args) == 6:
            celS, sclS, orgS, celT, sclT, orgT = args
            self.mem = GlaOprMem(opt, GlaVol(celT, sclT, orgT), GlaVol(celS, sclS, orgS), setTyp=setTyp, ctx=ctx)
        else:
            raise TypeError("GlaOpr(cel, scl[, org]) or GlaOpr(celSrc, sclSrc, orgSrc, celTrg, sclTrg, orgTrg)")

    # glaSze / size / eltype
    def glaSze(self, dim: Optional[int] = None):
        s = ((*self.mem._trg_cel, 3), (*self.mem._src_cel, 3))
        return s if dim is None else s[dim - 1]

    def size(self, dim: Optional[int] = None):
        s = (3 * math.prod(self.mem._trg_cel), 3 * math.prod(self.mem._src_cel))
        return s if dim is None else s[dim - 1]

    @property
    def dtype(self):
        return self.mem.dtype

    def _mul(self, x):
        if _elem_code(x) != self.mem._code:
            raise AssertionError(f"Input array must have the same element type as the operator. "
                                 f"eltype(opr) = {self.dtype}")
        n_src = math.prod(self.glaSze(2))
        n_trg = math.prod(self.glaSze(1))
        numel = x.numel() if _is_torch(x) else np.asarray(x).size
        if numel != n_src:
            raise DimensionMismatch(f"new dimensions {self.glaSze(2)} must be consistent with array size {numel}")
        cel = self.glaSze(2)[:3]
        if _is_torch(x):
            xs = x.reshape(3, cel[2], cel[1], cel[0])
        else:
            xs = np.reshape(np.asarray(x), self.glaSze(2), order="F")
        y = egoOpr(self.mem, xs)
        ndim = x.dim() if _is_torch(x) else np.asarray(x).ndim
        if numel == n_trg:
            return y.reshape(tuple(x.shape)) if _is_torch(x) else np.reshape(y, np.asarray(x).shape, order="F")
        if ndim == 1:
            return y.reshape(-1) if _is_torch(x) else np.reshape(y, -1, order="F")
        return y

    def __mul__(self, x):
        return self._mul(x)

    def __matmul__(self, x):
        return self._mul(x)

    def __repr__(self):
        m = self.mem
        adj = "Adjoint " if isadjoint(self) else ""
        if isselfoperator(self):
            return f"{adj}Self GlaOpr for a {self.dtype} ({'x'.join(map(str, m._src_cel))}) volume"
        return (f"{adj}External GlaOpr for {self.dtype} ({'x'.join(map(str, m._src_cel))}) -> "
                f"({'x'.join(map(str, m._trg_cel))}) volumes")


def glaSze(opr: GlaOpr, dim: Optional[int] = None):
    """glaSze (src/glaMemSup.jl:359-371)."""
    return opr.glaSze(dim)


def size(opr: GlaOpr, dim: Optional[int] = None):
    """Base.size (src/glaLinAlg.jl:5-8)."""
    return opr.size(dim)


def eltype(opr: GlaOpr):
    """Base.eltype (src/glaLinAlg.jl:4)."""
    return opr.dtype


def adjoint(opr: GlaOpr) -> GlaOpr:
    """Base.adjoint (src/glaLinAlg.jl:16-29): adjMod flipped, volumes
    swapped, the same Fourier data; the matvec ignores adjMod, as in the
    reference."""
    h = ct.c_void_p()
    _check(L.lib().gila_opr_adjoint(opr.mem._h, ct.byref(h)))
    m = opr.mem
    opt = m.cmpInf.copy(adjMod=not m.cmpInf.adjMod)
    return GlaOpr(GlaOprMem._from_handle(h, m.ctx, opt, m.srcVol, m.trgVol))


def isadjoint(opr: GlaOpr) -> bool:
    return bool(opr.mem._flags & 2)


def isselfoperator(opr: GlaOpr) -> bool:
    return bool(opr.mem._flags & 1)


def isexternaloperator(opr: GlaOpr) -> bool:
    return not isselfoperator(opr)


def issymmetric(opr) -> bool:
    return False


def isposdef(opr) -> bool:
    return False


def ishermitian(opr) -> bool:
    return False


def isdiag(opr) -> bool:
    return False


def mul(outVec, opr: GlaOpr, innVec, alpha=1.0, beta=0.0):
    """LinearAlgebra.mul!(outVec, opr, innVec, alpha, beta)
    (src/glaLinAlg.jl:61-69): outVec = alpha * (opr * innVec) + beta * outVec,
    in place, with the axpby fused into the last pass on the GPU."""
    if _elem_code(innVec) != opr.mem._code:
        raise AssertionError(f"Input array must have the same element type as the operator. "
                             f"eltype(opr) = {opr.dtype}")
    n_src = math.prod(opr.glaSze(2))
    numel = innVec.numel() if _is_torch(innVec) else np.asarray(innVec).size
    if numel != n_src:
        raise DimensionMismatch(f"new dimensions {opr.glaSze(2)} must be consistent with array size {numel}")
    if _is_torch(outVec):
        opr.mem.axpby_into(alpha, innVec, beta, outVec)
        return outVec
    o = np.asarray(outVec)
    if o.ndim > 1 and not o.flags.f_contiguous:
        tmp = np.asfortranarray(o)
        opr.mem.axpby_into(alpha, innVec, beta, tmp)
        o[...] = tmp
    else:
        opr.mem.axpby_into(alpha, innVec, beta, o)
    return outVec


def cast(opr: GlaOpr, setTyp) -> GlaOpr:
    """The same operator in another precision (the Fourier kernel cast on the
    device); used to pair a ComplexF64 operator with its ComplexF32 copy."""
    h = ct.c_void_p()
    _check(L.lib().gila_opr_cast(opr.mem._h, _dtype_code(setTyp), ct.byref(h)))
    m = opr.mem
    return GlaOpr(GlaOprMem._from_handle(h, m.ctx, m.cmpInf, m.trgVol, m.srcVol))


class LippmannSchwinger:
    """LippmannSchwinger(greens_op, medium) (examples/GilaOperators.jl:57-82):
    the operator x -> x - medium .* (G x), medium per cell broadcast over the
    three components.  `medium` has the target cell shape (Nx, Ny, Nz)."""

    def __init__(self, greens_op: GlaOpr, medium):
        cel = tuple(greens_op.glaSze(1)[:3])
        med = medium
        if _is_torch(med):
            shp = tuple(med.shape)
            if shp not in (cel, (cel[2], cel[1], cel[0])):
                raise DimensionMismatch("Green's operator and medium must have the same size.")
            med = med.detach().cpu().numpy()
            if shp == (cel[2], cel[1], cel[0]):
                med = np.ascontiguousarray(med).reshape(-1).reshape(cel, order="F")
        else:
            med = np.asarray(med)
            if tuple(med.shape) != cel:
                raise DimensionMismatch("Green's operator and medium must have the same size.")
        if np.dtype(med.dtype) != np.dtype(greens_op.dtype):
            raise ArgumentError("Medium must have the same element type as the Green's operator.")
        self.greens_op = greens_op
        self.medium = np.asfortranarray(med)
        self._g32 = None

    def glaSze(self, dim: Optional[int] = None):
        return self.greens_op.glaSze(dim)

    def size(self, dim: Optional[int] = None):
        return self.greens_op.size(dim)

    @property
    def dtype(self):
        return self.greens_op.dtype

    def _mul(self, x):
        """ls * x = x - medium .* (G x) (examples/GilaOperators.jl:89-95)."""
        gx = self.greens_op * x
        if _is_torch(x):
            import torch
            cel = self.glaSze(1)[:3]
            chi = torch.from_numpy(np.ascontiguousarray(self.medium.reshape(-1, order="F"))).to(x.device)
            chi = chi.reshape(cel[2], cel[1], cel[0])
            return x - (chi * gx.reshape(3, cel[2], cel[1], cel[0])).reshape(x.shape)
        xa = np.asarray(x)
        cel = self.glaSze(1)[:3]
        g4 = np.reshape(gx, (*cel, 3), order="F")
        return xa - np.reshape(self.medium[..., None] * g4, xa.shape, order="F")

    def __mul__(self, x):
        return self._mul(x)

    def __matmul__(self, x):
        return self._mul(x)

    def g32(self) -> GlaOpr:
        """The ComplexF32 copy of the Green operator (made once)."""
        if self._g32 is None:
            if self.greens_op.dtype == np.complex64:
                self._g32 = self.greens_op
            else:
                self._g32 = cast(self.greens_op, np.complex64)
        return self._g32


class SolveInfo:
    """Counters of one gila_ls_solve call."""

    def __init__(self, c: L.GilaSolveInfoC, res):
        self.iters = c.iters
        self.outer = c.outer
        self.matvecs_f64 = c.matvecs_f64
        self.matvecs_f32 = c.matvecs_f32
        self.rel_res = c.rel_res
        self.converged = c.converged
        self.breakdowns = c.breakdowns
        self.rhs_res = list(res)

    def __repr__(self):
        return (f"SolveInfo(iters={self.iters}, outer={self.outer}, matvecs_f64={self.matvecs_f64}, "
                f"matvecs_f32={self.matvecs_f32}, rel_res={self.rel_res:.3e}, converged={self.converged})")


def solve(ls: LippmannSchwinger, i, *, tol: float = 1e-6, mixed: bool = False, ell: int = 2,
          delta: float = 0.1, max_matvecs: int = 4000, max_restarts: int = 20, x0=None,
          graph: bool = True, check: bool = True, stream=None, keep: bool = False):
    """Solve ls * t = i (t = (1 - chi G)^-1 i, examples/scattering_film.jl:58-61)
    with BiCGStab(ell) on the GPU, for one field or a stack of nrhs fields.

    numpy input: (Nx, Ny, Nz, 3) or (Nx, Ny, Nz, 3, nrhs); torch input:
    (3, Nz, Ny, Nx) or (nrhs, 3, Nz, Ny, Nx); complex128 either way.  mixed
    runs the Krylov process on the ComplexF32 operator with FP64 reliable
    updates (FP64 solution; the recursive residual replaced by the FP64
    b - A x whenever it fell by `delta`).  Returns (t, SolveInfo); raises
    GilaError when a right-hand side misses tol and `check` is set.  With a
    CUDA stream handle the solve is ordered after the work queued on it and
    the stream waits for the solve.  keep=True leaves the solve's device state
    resident with the operator for the next call of the same shape."""
    G = ls.greens_op
    if G.dtype != np.complex128:
        raise AssertionError("the solve needs the ComplexF64 Green operator (its residual is FP64)")
    cel = G.glaSze(1)[:3]
    nvox = 3 * math.prod(cel)
    if _is_torch(i):
        import torch
        if i.dtype != torch.complex128:
            raise AssertionError("right-hand sides must be complex128")
        b = i.contiguous()
        numel = b.numel()
        x = torch.empty_like(b)
        bp, xp = b.data_ptr(), x.data_ptr()
        keep = (b, x)
    else:
        a = np.asarray(i)
        if a.dtype != np.complex128:
            raise AssertionError("right-hand sides must be complex128")
        b = np.asfortranarray(a)
        numel = b.size
        x = np.zeros_like(b, order="F")
        bp, xp = b.ctypes.data, x.ctypes.data
        keep = (b, x)
    if numel % nvox:
        raise DimensionMismatch(f"right-hand sides must hold whole fields of {nvox} elements")
    nrhs = numel // nvox
    if x0 is not None:
        if _is_torch(x):
            x.copy_(x0.reshape(x.shape))
        else:
            x[...] = np.reshape(np.asarray(x0), x.shape, order="F")
    chi = np.asfortranarray(ls.medium.astype(np.complex128))
    o = L.GilaSolveC(tol=tol, ell=ell, mixed=1 if mixed else 0, max_matvecs=max_matvecs,
                     max_restarts=max_restarts, delta=delta, x0=0 if x0 is None else 1, no_graph=0 if graph else 1,
                     keep=1 if keep else 0)
    inf = L.GilaSolveInfoC()
    res = (ct.c_double * nrhs)()
    g32 = ls.g32().mem._h if mixed else None
    st = L.lib().gila_ls_solve(G.mem._h, g32, ct.c_void_p(chi.ctypes.data), ct.c_void_p(bp), ct.c_void_p(xp),
                               nrhs, ct.byref(o), ct.byref(inf), res, ct.c_void_p(stream) if stream else None)
    del keep
    info = SolveInfo(inf, res)
    if st == L.GILA_ERR_NOTCONV and not check:
        return x, info
    _check(st)
    return x, info


class SolveServer:
    """Continuous-batching server of scattering solves (gila_server_*).

    submit(cel, scl, chi, b, tol=...) queues (I - chi G) x = b for the self
    volume of `cel` cells of scale `scl` and returns a ticket; wait(ticket)
    returns (x, SolveInfo, latency_ms).  Requests of the same shape share a
    batch of slots on the GPU and join it while it runs; shapes run
    concurrently; admission is by device memory (hbm_budget bytes, 0: free
    memory minus 4 GiB).  numpy inputs: chi (Nx,Ny,Nz), b (Nx,Ny,Nz,3),
    complex128."""

    def __init__(self, *, slots: int = 8, ell: int = 2, mixed: bool = True, hbm_budget: int = 0,
                 intOrd: int = 32, frqPhz: complex = 1.0 + 0j, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        o = L.GilaServerOptsC(hbm_budget=int(hbm_budget), slots=int(slots), ell=int(ell), mixed=1 if mixed else 0,
                              int_ord=int(intOrd), frq_re=complex(frqPhz).real, frq_im=complex(frqPhz).imag)
        h = ct.c_void_p()
        _check(L.lib().gila_server_create(self.ctx.handle, ct.byref(o), ct.byref(h)))
        self._h = h
        self._live = {}

    def close(self):
        if getattr(self, "_h", None):
            L.lib().gila_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, cel, scl, chi, b, *, tol: float = 1e-6, max_matvecs: int = 4000, delta: float = 0.1,
               max_restarts: int = 20) -> int:
        v = GlaVol(cel, scl).to_c()
        chi_a = np.asfortranarray(np.asarray(chi, dtype=np.complex128))
        b_a = np.asfortranarray(np.asarray(b, dtype=np.complex128))
        if chi_a.shape != tuple(cel) or b_a.shape != (*cel, 3):
            raise DimensionMismatch("medium (Nx,Ny,Nz) and field (Nx,Ny,Nz,3) must match the volume")
        x = np.zeros_like(b_a, order="F")
        o = L.GilaSolveC(tol=tol, max_matvecs=max_matvecs, delta=delta, max_restarts=max_restarts)
        t = ct.c_uint64()
        _check(L.lib().gila_server_submit(self._h, ct.byref(v), ct.c_void_p(chi_a.ctypes.data),
                                          ct.c_void_p(b_a.ctypes.data), ct.c_void_p(x.ctypes.data), ct.byref(o),
                                          ct.byref(t)))
        self._live[t.value] = (chi_a, b_a, x)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1, check: bool = True):
        inf = L.GilaSolveInfoC()
        lat = ct.c_double()
        st = L.lib().gila_server_wait(self._h, ct.c_uint64(ticket), int(timeout_ms), ct.byref(inf), ct.byref(lat))
        if st == L.GILA_ERR_TIMEOUT:
            raise TimeoutError(L.last_error())
        bufs = self._live.pop(ticket, None)
        info = SolveInfo(inf, [inf.rel_res])
        if not (st == L.GILA_ERR_NOTCONV and not check):
            _check(st)
        return (bufs[2] if bufs else None), info, lat.value

    def stats(self) -> dict:
        s = L.GilaServerStatsC()
        _check(L.lib().gila_server_stats_get(self._h, ct.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}


from .slab import SlabOpr, SlabPieces, SlabPlan, slab_apply_local, slab_ranges  # noqa: E402
