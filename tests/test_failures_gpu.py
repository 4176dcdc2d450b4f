"""Failure paths, made on the host: every error comes back as a status (a
Python exception here), nothing hangs, and nothing leaks.

  * a non-finite egoFur is refused with GILA_ERR_NAN, as the reference's
    GlaOprMem refuses it (src/glaMemSup.jl:93-95, 110-112, 159-164);
  * NaN / Inf in a solve's medium or incident field is refused with
    GILA_ERR_NAN before any iteration, by gila_ls_solve and by the server's
    submit;
  * device allocations made to fail one at a time (gila_debug_fail_alloc: the
    n-th allocation returns out-of-memory before cudaMalloc is called) give
    GILA_ERR_NOMEM at every point of operator creation, the GPU kernel build,
    the first apply and a solve, and free device memory returns to its level
    before the call each time;
  * gila_server_wait with a short timeout on a long request returns
    GILA_ERR_TIMEOUT and the request still completes afterwards.
No GPU fault, trap or hang is involved in any of them.
"""
from __future__ import annotations

import gc

import numpy as np
import pytest

from conftest import load_pkg
from oracle.synth import seeded_current, synth_operator
from test_server_gpu import _request

pytestmark = pytest.mark.gpu

SCL = ("1/32", "1/32", "1/32")


def _synth_mem(gila, cel, dtype=np.complex128, fur_edit=None):
    mix, fur, _, _, trg, _ = synth_operator(cel, SCL, (0, 0, 0), None, None)
    fur = [np.array(f, order="F") for f in fur]
    if fur_edit:
        fur_edit(fur)
    return mix, gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(trg.cel, trg.scl), egoFur=fur, setTyp=dtype)


@pytest.mark.parametrize("bad", [np.nan, np.inf, complex(0, np.nan)])
def test_nonfinite_egofur_is_refused(bad):
    gila = load_pkg()

    def edit(fur):
        fur[5][1, 0, 2, 3, 0, 0] = bad

    with pytest.raises(gila.GilaError, match="non-numeric") as ei:
        _synth_mem(gila, (6, 6, 6), fur_edit=edit)
    assert f"status {gila._lib.GILA_ERR_NAN}" in str(ei.value)


@pytest.mark.parametrize("where", ["chi", "b", "b_device"])
def test_nonfinite_solve_inputs_are_refused(where):
    import torch
    gila = load_pkg()
    cel = (8, 8, 8)
    G = gila.GlaOpr(gila.GlaOprMem(gila.GlaKerOpt(1.0 + 0j, 8, False, True, (), ()), gila.GlaVol(cel, SCL)))
    chi, b = _request(cel, 3)
    if where == "chi":
        chi[2, 3, 4] = np.nan
    else:
        b[1, 1, 1, 2] = complex(np.inf, 0)
    ls = gila.LippmannSchwinger(G, chi)
    rhs = b
    if where == "b_device":
        rhs = torch.from_numpy(np.ascontiguousarray(b.reshape(-1, order="F"))).cuda().reshape(3, *cel[::-1])
    with pytest.raises(gila.GilaError, match="non-numeric") as ei:
        gila.solve(ls, rhs, mixed=True)
    assert f"status {gila._lib.GILA_ERR_NAN}" in str(ei.value)
    srv = gila.SolveServer(slots=2, mixed=True, intOrd=8)
    try:
        with pytest.raises(gila.GilaError, match="non-numeric"):
            srv.submit(cel, SCL, chi, b)
    finally:
        srv.close()


def _free_bytes():
    import torch
    gc.collect()
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _inject_each(gila, step, max_points=80):
    """Run `step` with the k-th device allocation failing, k = 1, 2, ...,
    until a run needs fewer than k allocations; check each failure is
    GILA_ERR_NOMEM and that free memory returns to its starting level."""
    lib = gila._lib.lib()
    step()  # warm the context's caches (twiddle tables, launch shapes)
    base = _free_bytes()
    failures = 0
    for k in range(1, max_points + 1):
        assert lib.gila_debug_fail_alloc(k) == 0
        try:
            step()
            ok = True
        except gila.GilaError as e:
            assert f"status {gila._lib.GILA_ERR_NOMEM}" in str(e), str(e)
            failures += 1
            ok = False
        finally:
            lib.gila_debug_fail_alloc(0)
        leak = base - _free_bytes()
        assert abs(leak) < (4 << 20), f"allocation point {k}: {leak} bytes not returned"
        if ok:
            return failures
    raise AssertionError("more allocation points than expected")


def test_injected_allocation_failures_operator_and_apply():
    gila = load_pkg()
    cel = (48, 40, 32)
    x = np.asfortranarray(seeded_current(cel, 1))

    def step():
        _, mem = _synth_mem(gila, cel)
        y = gila.egoOpr(mem, x)
        assert np.isfinite(y).all()
        del mem

    assert _inject_each(gila, step) >= 3


def test_injected_allocation_failures_kernel_build():
    gila = load_pkg()

    def step():
        mem = gila.GlaOprMem(gila.GlaKerOpt(1.0 + 0j, 8, False, True, (), ()), gila.GlaVol((12, 10, 8), SCL))
        del mem

    assert _inject_each(gila, step) >= 5


def test_injected_allocation_failures_solve():
    gila = load_pkg()
    cel = (8, 8, 8)
    chi, b = _request(cel, 4)

    def step():
        G = gila.GlaOpr(gila.GlaOprMem(gila.GlaKerOpt(1.0 + 0j, 8, False, True, (), ()), gila.GlaVol(cel, SCL)))
        x, info = gila.solve(gila.LippmannSchwinger(G, chi), b, mixed=True)
        assert info.converged == 1
        del G, x

    assert _inject_each(gila, step, max_points=200) >= 5


def test_server_wait_timeout_then_completes():
    gila = load_pkg()
    cel = (48, 48, 48)
    chi, b = _request(cel, 11)
    srv = gila.SolveServer(slots=2, mixed=True, intOrd=8)
    try:
        t = srv.submit(cel, SCL, chi, b, tol=1e-6)
        with pytest.raises(TimeoutError):
            srv.wait(t, timeout_ms=1)
        x, info, lat = srv.wait(t, timeout_ms=120000)
        assert info.converged == 1 and info.rel_res <= 1e-6
        assert np.isfinite(x).all() and lat > 1.0
    finally:
        srv.close()
