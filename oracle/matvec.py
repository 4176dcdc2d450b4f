"""Oracle restatement of the host matvec ``egoOpr!`` -> ``egoBrnHst!``.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

This follows the reference's 8-branch recursion literally:
  * egoOpr!           src/glaAct.jl:33-49   (size check, host dispatch)
  * egoBrnHst!        src/glaAct.jl:63-183  (split -> FFT -> ... -> leaf
                                             multiply -> IFFT -> merge)
  * genPrtHst         src/glaActSup.jl:4-18 (source partition gather)
  * sptBrnHst! (self) src/glaActSup.jl:72-82   (odd = phase * even)
  * sptBrnHst! (ext)  src/glaActSup.jl:163-222 (fold / copy / zero ranges)
  * mrgBrnHst!        src/glaActSup.jl:425-435 and :502-537 (top/bottom)
  * mulBrnHst!        src/glaActSup.jl:671-764 (8 forward/reverse quadrants,
                                                mirrored reads, sign rules)
  * mulKerHst!        src/glaActSup.jl:879-898 (3x3 symmetric multiply)
  * mrgPrtHst         src/glaActSup.jl:939-953 (target partition scatter)
  * nxtBrnId          src/glaActSup.jl:1008-1010

Arrays are numpy arrays indexed ``[x, y, z, comp, part]`` (the reference's
Julia index order).  FFTs are numpy's (forward e^{-2 pi i}, unnormalised;
inverse scaled by 1/n), the same conventions as FFTW's plan_fft!/plan_ifft!.
"""
from __future__ import annotations

import math

import numpy as np

from .gla_mem import ExtInf


_fft = np.fft.fft
_ifft = np.fft.ifft
_parallel = False


def use_fft_workers(n: int) -> None:
    """Run the host path on n threads as the reference does: the 1-D
    transforms with scipy.fft on n threads (the reference runs FFTW with
    FFTW.set_num_threads(nthreads()), test/preamble.jl:1-14), and the two
    branches of every level of the recursion concurrently, so that the eight
    leaves run at once (egoBrnHst! spawns them, src/glaAct.jl:122-131); numpy
    releases the interpreter lock inside its array operations, so the
    branches' split / multiply / merge steps overlap."""
    global _fft, _ifft, _parallel
    import scipy.fft as sfft
    _fft = lambda a, axis: sfft.fft(a, axis=axis, workers=n)  # noqa: E731
    _ifft = lambda a, axis: sfft.ifft(a, axis=axis, workers=n)  # noqa: E731
    _parallel = n > 1


class OprMem:
    """The parts of GlaOprMem (src/glaMem.jl:93-104) that egoOpr! reads."""

    def __init__(self, mix: ExtInf, fur, dtype=np.complex128):
        self.mix = mix
        self.fur = [np.asarray(f) for f in fur]  # 8 arrays (t,t,t,6,parS,parT)
        self.dtype = np.dtype(dtype)
        self.brn = mix.brn
        # phase vectors, src/glaMemSup.jl:232-236 (computed in FP64, cast)
        self.phz = [np.exp(-1j * math.pi * np.arange(b) / b).astype(self.dtype)
                    for b in self.brn]


def ego_opr(mem: OprMem, act: np.ndarray) -> np.ndarray:
    """egoOpr! (src/glaAct.jl:33-49)."""
    if tuple(act.shape) != (*mem.mix.src_cel, 3):
        # the reference's size check compares against mixInf.srcCel, so a
        # partitioned source must still be passed at partition size
        raise ValueError("Size of input vector does not match size of source volume.")
    return _brn(mem, 0, 0, np.array(act, dtype=mem.dtype))


def ego_opr_full(mem: OprMem, act: np.ndarray) -> np.ndarray:
    """egoBrnHst! entered directly at level 0 with a full (partitioned)
    source volume, as the reference does when size(actVec) != srcCel."""
    return _brn(mem, 0, 0, np.array(act, dtype=mem.dtype))


def _nxt(lvl: int, bid: int) -> int:
    return bid + 2 ** (3 - (lvl + 1))


def _gen_prt(mix: ExtInf, act: np.ndarray) -> np.ndarray:
    """genPrtHst: orgVec[x,y,z,c,p] = act[x*div + off_p, c]."""
    offs = mix.par_offsets("src")
    d = mix.src_div
    c = mix.src_cel
    out = np.empty((*c, 3, len(offs)), dtype=act.dtype)
    for p, (ox, oy, oz) in enumerate(offs):
        out[..., p] = act[ox:ox + d[0] * c[0]:d[0],
                          oy:oy + d[1] * c[1]:d[1],
                          oz:oz + d[2] * c[2]:d[2], :]
    return out


def _mrg_prt(mix: ExtInf, prt: np.ndarray) -> np.ndarray:
    """mrgPrtHst: inverse of the target partition gather."""
    offs = mix.par_offsets("trg")
    d = mix.trg_div
    c = mix.trg_cel
    out = np.empty((*[a * b for a, b in zip(d, c)], 3), dtype=prt.dtype)
    for p, (ox, oy, oz) in enumerate(offs):
        out[ox::d[0], oy::d[1], oz::d[2], :] = prt[..., p]
    return out


def _spt_ext(prg_e, prg_o, ax, phz, mix, org):
    """sptBrnHst! general form (src/glaActSup.jl:163-222): first radix-2
    decimation-in-frequency stage of the zero-padded length-P DFT."""
    brn = mix.brn[ax]
    src = mix.src_cel[ax]
    n_ovr = max(src - brn, 0)
    n_std_end = min(src, brn)
    sl = [slice(None)] * 5

    def s(a, b):
        q = list(sl)
        q[ax] = slice(a, b)
        return tuple(q)

    shp = [1] * 5
    shp[ax] = -1
    ph = phz.reshape(shp)
    if n_ovr > 0:
        lo = org[s(0, n_ovr)]
        hi = org[s(brn, brn + n_ovr)]
        prg_e[s(0, n_ovr)] = lo + hi
        prg_o[s(0, n_ovr)] = ph[s(0, n_ovr)] * (lo - hi)
    if n_std_end > n_ovr:
        mid = org[s(n_ovr, n_std_end)]
        prg_e[s(n_ovr, n_std_end)] = mid
        prg_o[s(n_ovr, n_std_end)] = ph[s(n_ovr, n_std_end)] * mid
    if brn > n_std_end:
        prg_e[s(n_std_end, brn)] = 0
        prg_o[s(n_std_end, brn)] = 0


def _mrg_ext(mrg, ax, phz, eve, odd):
    """mrgBrnHst! general form (src/glaActSup.jl:502-537): last radix-2
    decimation-in-time stage of the inverse DFT, truncated to the target."""
    n_mrg = mrg.shape[ax]
    n_cur = eve.shape[ax]
    top = min(n_mrg, n_cur)
    bot = n_mrg - top
    shp = [1] * 5
    shp[ax] = -1

    def s(a, b):
        q = [slice(None)] * 5
        q[ax] = slice(a, b)
        return tuple(q)

    ph = np.conj(phz).reshape(shp)
    mrg[s(0, top)] = 0.5 * (eve[s(0, top)] + ph[s(0, top)] * odd[s(0, top)])
    if bot > 0:
        mrg[s(top, top + bot)] = 0.5 * (eve[s(0, bot)] - ph[s(0, bot)] * odd[s(0, bot)])


def _quadrants(mix: ExtInf, bid: int, ego_sze, brn):
    """Per-axis index ranges and signs of mulBrnHst! (src/glaActSup.jl:697-752).

    Yields (mod_idx[3], vec_idx[3], dir_sym[3]) for each non-empty quadrant,
    with 0-based integer index arrays."""
    brn_sym = [(bid // 2 ** (3 - k)) % 2 for k in range(1, 4)]
    for div in range(8):
        rev = [(div // 2 ** k) % 2 for k in range(3)]
        mod_r, vec_r, sgn = [], [], []
        for d in range(3):
            if ego_sze[d] == brn[d]:
                if rev[d] == 0:
                    mod_r.append(np.arange(brn[d]))
                    vec_r.append(np.arange(brn[d]))
                    sgn.append(1.0)
                else:
                    mod_r.append(np.arange(0))
                    vec_r.append(np.arange(0))
                    sgn.append(0.0)
                continue
            t = mix.trg_cel[d]
            sc = mix.src_cel[d]
            if brn_sym[d] == 0:
                if rev[d] == 0:
                    beg, end = 1, int(math.ceil(t / 2)) + (1 if t % 2 == 0 else 0)
                else:
                    beg, end = 2, sc // 2 + 1 - (1 if t % 2 == 0 else 0)
            else:
                beg = 1
                end = int(math.ceil(t / 2)) if rev[d] == 0 else sc // 2
            mod_r.append(np.arange(beg - 1, end))  # 1-based beg:end
            cnt = max(end - beg + 1, 0)
            if rev[d] == 0:
                vec_r.append(np.arange(cnt))
            else:
                vec_r.append(brn[d] - 1 - np.arange(cnt))
            sgn.append(1.0 - 2.0 * rev[d])
        if any(len(r) == 0 for r in mod_r):
            continue
        dir_sym = (sgn[0] * sgn[1], sgn[0] * sgn[2], sgn[1] * sgn[2])
        yield mod_r, vec_r, dir_sym


def _mul_brn(mix, bid, prd, ker, org, brn):
    """mulBrnHst! + mulKerHst!: prd += S(ker) . org with S the 3x3
    complex-symmetric tensor from (xx, yy, zz, xy, xz, yz)."""
    for mod_r, vec_r, ds in _quadrants(mix, bid, ker.shape[:3], brn):
        mi = np.ix_(*mod_r)
        vi = np.ix_(*vec_r)
        g = [ker[..., c][mi] for c in range(6)]
        o = [org[..., c][vi] for c in range(3)]
        d1, d2, d3 = (np.asarray(v, dtype=prd.real.dtype) for v in ds)
        prd[..., 0][vi] += g[0] * o[0] + d1 * g[3] * o[1] + d2 * g[4] * o[2]
        prd[..., 1][vi] += d1 * g[3] * o[0] + g[1] * o[1] + d3 * g[5] * o[2]
        prd[..., 2][vi] += d2 * g[4] * o[0] + d3 * g[5] * o[1] + g[2] * o[2]


def _brn(mem: OprMem, lvl: int, bid: int, act: np.ndarray) -> np.ndarray:
    mix = mem.mix
    brn = mem.brn
    par_s = math.prod(mix.src_div)
    par_t = math.prod(mix.trg_div)
    if lvl == 0 and tuple(act.shape[:3]) != tuple(mix.src_cel):
        org = _gen_prt(mix, act)
    elif lvl == 0:
        org = act.reshape(*mix.src_cel, 3, par_s)
    else:
        org = act
    if lvl > 0:
        org = _fft(org, axis=lvl - 1).astype(mem.dtype, copy=False)
    if lvl < 3:
        ax = lvl
        if org.shape[ax] == brn[ax]:
            shp = [1] * 5
            shp[ax] = -1
            prg_o = (mem.phz[ax].reshape(shp) * org).astype(mem.dtype, copy=False)
            prg_e = org
        else:
            psz = list(org.shape)
            psz[ax] = brn[ax]
            prg_e = np.empty(psz, dtype=mem.dtype)
            prg_o = np.empty(psz, dtype=mem.dtype)
            _spt_ext(prg_e, prg_o, ax, mem.phz[ax], mix, org)
        if _parallel:
            from concurrent.futures import ThreadPoolExecutor
            with ThreadPoolExecutor(2) as ex:
                fe = ex.submit(_brn, mem, lvl + 1, bid, prg_e)
                fo = ex.submit(_brn, mem, lvl + 1, _nxt(lvl, bid), prg_o)
                eve, odd = fe.result(), fo.result()
        else:
            eve = _brn(mem, lvl + 1, bid, prg_e)
            odd = _brn(mem, lvl + 1, _nxt(lvl, bid), prg_o)
        if eve.shape[ax] == mix.trg_cel[ax]:
            shp = [1] * 5
            shp[ax] = -1
            ret = 0.5 * (eve + np.conj(mem.phz[ax]).reshape(shp) * odd)
            ret = ret.astype(mem.dtype, copy=False)
        else:
            msz = list(eve.shape)
            msz[ax] = mix.trg_cel[ax]
            msz[4] = par_t
            ret = np.empty(msz, dtype=mem.dtype)
            _mrg_ext(ret, ax, mem.phz[ax], eve, odd)
    else:
        ret = np.zeros((*brn, 3, par_t), dtype=mem.dtype)
        for t in range(par_t):
            for s_ in range(par_s):
                _mul_brn(mix, bid, ret[..., t], mem.fur[bid][:, :, :, :, s_, t],
                         org[..., s_], brn)
    if lvl > 0:
        ret = _ifft(ret, axis=lvl - 1).astype(mem.dtype, copy=False)
    if lvl == 0:
        if par_t == 1:
            return ret.reshape(*mix.trg_cel, 3)
        return _mrg_prt(mix, ret)
    return ret
