"""The continuous-batching solve server (gila_server_*).

Each request's result must not depend on what else the server is running:
a request solved alone and the same request inside a stream of other
requests (several shapes, shared slots, concurrent batches) give the same
field.  Fields are also checked through the oracle's FP64 residual with the
server's own operator kernel rebuilt by GlaOprMem (the same GPU build).
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_pkg
from oracle.gla_mem import Vol, mix_for
from oracle.matvec import OprMem
from oracle.solve import ls_apply

pytestmark = pytest.mark.gpu

SCL = ("1/32", "1/32", "1/32")
ORD = 16
TOL = 1e-6
SHAPES = [(8, 8, 8), (12, 10, 8), (16, 12, 8)]


def _request(cel, seed):
    """cube or slab inclusion, chi = U[0.5,4] + i U[0,0.2], plane wave at a
    random angle (seeded)."""
    rng = np.random.default_rng(seed)
    chi = np.zeros(cel, dtype=np.complex128, order="F")
    val = rng.uniform(0.5, 4.0) + 1j * rng.uniform(0.0, 0.2)
    if rng.random() < 0.5:
        lo = [n // 4 for n in cel]
        hi = [n - n // 4 for n in cel]
        chi[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = val
    else:
        z0 = cel[2] // 4
        chi[:, :, z0:cel[2] - z0] = val
    th = rng.uniform(0, np.pi)
    k = np.array([np.sin(th), 0.0, np.cos(th)])
    h = 1.0 / 32
    x, y, z = np.meshgrid(*[np.arange(n) * h for n in cel], indexing="ij")
    e = np.zeros((*cel, 3), dtype=np.complex128, order="F")
    e[..., 1] = np.exp(2j * np.pi * (k[0] * x + k[2] * z))
    return chi, e


def _oracle_residual(gila, cel, chi, b, x):
    mem = gila.GlaOprMem(gila.GlaKerOpt(1.0 + 0j, ORD, False, True, (), ()), gila.GlaVol(cel, SCL))
    _, _, mix, _ = mix_for(Vol.make(cel, SCL, (0, 0, 0)), None)
    om = OprMem(mix, mem.egoFur)
    bf = np.reshape(b, -1, order="F")
    xf = np.reshape(x, -1, order="F")
    return np.linalg.norm(bf - ls_apply(om, chi, xf)) / np.linalg.norm(bf)


@pytest.mark.parametrize("mixed", [True, False])
def test_alone_equals_in_mix(mixed):
    gila = load_pkg()
    srv = gila.SolveServer(slots=4, mixed=mixed, intOrd=ORD)
    try:
        cel = SHAPES[1]
        chi, b = _request(cel, 7)
        x_alone, inf_alone, lat = srv.wait(srv.submit(cel, SCL, chi, b, tol=TOL))
        assert inf_alone.converged == 1 and lat > 0
        # the same request in the middle of a stream of others
        reqs = [(SHAPES[i % 3], _request(SHAPES[i % 3], 100 + i)) for i in range(9)]
        reqs.insert(4, (cel, (chi, b)))
        tickets = [srv.submit(c, SCL, q[0], q[1], tol=TOL) for c, q in reqs]
        outs = [srv.wait(t) for t in tickets]
        x_mix, inf_mix, _ = outs[4]
        assert np.array_equal(x_mix, x_alone)
        assert inf_mix.iters == inf_alone.iters
        for (c, (ch, bb)), (x, inf, lat) in zip(reqs, outs):
            assert inf.converged == 1 and inf.rel_res <= TOL and lat > 0
        # the server's FP64 residual matches the oracle's on two of them
        for k in (0, 4):
            c, (ch, bb) = reqs[k]
            assert _oracle_residual(gila, c, ch, bb, outs[k][0]) <= TOL
        st = srv.stats()
        assert st["completed"] == 11 and st["submitted"] == 11 and st["running"] == 0
        assert st["operators"] == 3 and st["bytes_in_use"] <= st["hbm_budget"]
    finally:
        srv.close()


def test_small_budget_admits_one_shape_at_a_time():
    gila = load_pkg()
    # measure what the largest shape needs alone, then allow a bit more than that
    probe = gila.SolveServer(slots=2, mixed=True, intOrd=ORD)
    try:
        chi, b = _request(SHAPES[2], 1)
        x_ref, _, _ = probe.wait(probe.submit(SHAPES[2], SCL, chi, b, tol=TOL))
        need = probe.stats()["bytes_in_use"]
    finally:
        probe.close()
    build_tmp = 6 * 16 * np.prod([2 * n for n in SHAPES[2]]) + 6 * 16 * np.prod(SHAPES[2]) + (64 << 20)
    srv = gila.SolveServer(slots=2, mixed=True, intOrd=ORD, hbm_budget=int(need + build_tmp + (1 << 20)))
    try:
        reqs = [(SHAPES[i % 3], _request(SHAPES[i % 3], 200 + i)) for i in range(6)]
        reqs.append((SHAPES[2], (chi, b)))
        tickets = [srv.submit(c, SCL, q[0], q[1], tol=TOL) for c, q in reqs]
        outs = [srv.wait(t, timeout_ms=300000) for t in tickets]
        assert all(o[1].converged == 1 for o in outs)
        assert np.array_equal(outs[-1][0], x_ref)
        st = srv.stats()
        assert st["bytes_in_use"] <= st["hbm_budget"]
    finally:
        srv.close()


def test_server_errors():
    gila = load_pkg()
    srv = gila.SolveServer(slots=2, mixed=True, intOrd=ORD)
    try:
        chi, b = _request(SHAPES[0], 3)
        with pytest.raises(gila.DimensionMismatch):
            srv.submit(SHAPES[1], SCL, chi, b)
        with pytest.raises(gila.GilaError):
            srv.wait(987654)
        # a budget of matvecs too small to converge: reported, not raised
        t = srv.submit(SHAPES[0], SCL, chi, b, tol=1e-12, max_matvecs=4)
        x, inf, _ = srv.wait(t, check=False)
        assert inf.converged == 0 and inf.rel_res > 1e-12
    finally:
        srv.close()
