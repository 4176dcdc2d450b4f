"""The kx-chunk pipeline of the matvec (off by default; GILA_KX_CHUNKS sets
the chunk count): the forward y pass, the z pass and the inverse y pass of
disjoint kx chunks on three streams.  It reorders launches only, so a matvec
and a solve (whose Krylov cycles are captured into CUDA graphs, here with the
three-stream fork and join inside the capture) must give the same bits as
the unpipelined run.  The pipelined run is a child process, since the
setting is read once per process."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, load_pkg
from oracle.synth import seeded_current, synth_operator

pytestmark = pytest.mark.gpu

SCL = ("1/32", "1/32", "1/32")
CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
from test_kx_pipeline_gpu import run_case
out = run_case()
np.save({path!r}, out["y"])
np.save({path2!r}, out["x"])
print(json.dumps({{"launches": out["launches"]}}))
"""


def run_case():
    gila = load_pkg()
    cel = (32, 32, 48)  # circulant lengths 64, 64, 96
    mix, fur, _, _, trg, _ = synth_operator(cel, SCL, (0, 0, 0), None, None)
    mem = gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(trg.cel, trg.scl), egoFur=fur, setTyp=np.complex128)
    xs = np.asfortranarray(np.stack([seeded_current(cel, s) for s in (1, 2)], axis=-1))
    y = np.zeros_like(xs, order="F")
    mem.apply_into(xs, y, nrhs=2)
    G = gila.GlaOpr(gila.GlaOprMem(gila.GlaKerOpt(1.0 + 0j, 8, False, True, (), ()), gila.GlaVol((32, 32, 32), SCL)))
    chi = np.zeros((32, 32, 32), dtype=np.complex128, order="F")
    chi[8:24, 8:24, 8:24] = 2.0 + 0.1j
    b = np.asfortranarray(seeded_current((32, 32, 32), 5))
    x, info = gila.solve(gila.LippmannSchwinger(G, chi), b, mixed=True)
    assert info.converged == 1
    return {"y": y, "x": x, "launches": mem.launches_per_apply(2)}


def test_pipelined_matvec_and_solve_bit_identical(tmp_path):
    assert os.environ.get("GILA_KX_CHUNKS", "0") in ("0", "1")
    ref = run_case()
    path, path2 = str(tmp_path / "y.npy"), str(tmp_path / "x.npy")
    src = CHILD.format(root=ROOT, tests=os.path.join(ROOT, "tests"), path=path, path2=path2)
    env = dict(os.environ, GILA_KX_CHUNKS="4")
    r = subprocess.run([sys.executable, "-c", src], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["launches"] > ref["launches"]  # the pipelined form ran
    assert np.array_equal(np.load(path), ref["y"])
    assert np.array_equal(np.load(path2), ref["x"])
