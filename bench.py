#!/usr/bin/env python
"""Benchmark of the Green-operator matvec (egoOpr!) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one application of the ComplexF64 self Green operator to one
source current on the 256x256x128-cell volume with 1/32-wavelength cells (the
largest single-GPU configuration, the thin-film volume; its ComplexF32 leg,
the 128x128x64 self and 64^3 -> 64x64x32 external operators of the matvec
precision sweep are reported in "sweep").  Inputs are seeded i.i.d. complex
N(0,1) currents and a seeded synthetic Fourier kernel with the reference's
storage shapes (kernel values do not change the matvec's work).  Under
torchrun each rank runs an independent replica on its own GPU (weak
scaling); `value` is the whole-job matvec/s from the max over ranks of the
device time.

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gilaelectromagnetics.jl_b200")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Green matvec/s (ComplexF64 egoOpr!, self 256x256x128)"
CEL = (256, 256, 128)
SWEEP_CEL = (128, 128, 64)
SCL = ("1/32", "1/32", "1/32")
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2
E2E_BATCH = 32  # at most this many host vectors (403 MB each) per API call in the end-to-end leg


def bench_config(c64: bool, world: int) -> dict:
    """The `config` of the bench line; both arms print the same dict."""
    return {"workload": "self Green operator 256x256x128 cells, 1/32 wavelength, "
                        + ("ComplexF32" if c64 else "ComplexF64") + ", 1 vector/step",
            "parallelism": f"replicas x{world}",
            "l2": "flushed (256 MB write) between timed steps; each step's vectors (403 MB in, 403 MB out) "
                  "are larger than the 126 MB L2"}


def load_pkg():
    if "gila_b200" in sys.modules:
        return sys.modules["gila_b200"]
    spec = importlib.util.spec_from_file_location("gila_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gila_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def tru_self(cel):
    """Stored kernel extent per axis of a self operator (src/glaMemSup.jl:121-136)."""
    return [max((n + 1) // 2 + (1 if n % 2 == 0 else 0), 2) for n in cel]


def synthetic_fur(tru, dtype, seed):
    rng = np.random.default_rng(seed)
    return [np.asfortranarray((rng.standard_normal((*tru, 6, 1, 1))
                               + 1j * rng.standard_normal((*tru, 6, 1, 1))).astype(dtype)) for _ in range(8)]


def tmin_bytes(src, trg, tru, csize):
    """Algorithmic bytes of one matvec, 3-pass model: read x, write+read the
    x,y-padded spectrum, read the kernel, write+read the z-truncated spectrum,
    write y."""
    Px, Py = src[0] + trg[0], src[1] + trg[1]
    Ns, Nt = math.prod(src), math.prod(trg)
    K = 8 * math.prod(tru)
    return csize * (3 * Ns + 6 * Px * Py * src[2] + 6 * K + 6 * Px * Py * trg[2] + 3 * Nt)


def zpass_bytes(src, trg, tru, csize):
    """Algorithmic bytes of one z-pass launch (the dominant kernel): read the
    x,y spectrum (3 components, source z planes), read the stored kernel,
    write the z-truncated spectrum."""
    Px, Py = src[0] + trg[0], src[1] + trg[1]
    K = 8 * math.prod(tru)
    return csize * (3 * Px * Py * src[2] + 6 * K + 3 * Px * Py * trg[2])


class Clocks:
    """nvidia-smi sampler (every 50 ms) around the timed region.  Each sample
    is stamped on arrival by a reader thread; the report covers the samples
    that arrived between begin() and end() plus one sampling interval, so a
    timed region shorter than the interval still gets the samples that
    bracket it ("in_region" says how many fell inside)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 50

    def __init__(self, index):
        self.rows, self.t0, self.t1 = [], None, None
        self.lock = threading.Lock()
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-i", str(index), "-lms", str(self.INTERVAL_MS)],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()
        # the first sample can take a second to appear: start timing after it
        deadline = time.monotonic() + 5.0
        while time.monotonic() < deadline:
            with self.lock:
                if self.rows:
                    break
            time.sleep(0.01)

    def _read(self):
        for line in self.p.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                with self.lock:
                    self.rows.append((time.monotonic(), parts))

    def begin(self):
        self.t0 = time.monotonic()

    def end(self):
        self.t1 = time.monotonic()

    def stop(self):
        if self.p is None:
            return None
        if self.t1 is None:
            self.end()
        # let the sample after the region arrive
        time.sleep(1.5 * self.INTERVAL_MS / 1e3)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.th.join(timeout=2)
        t0 = self.t0 if self.t0 is not None else self.t1
        pad = self.INTERVAL_MS / 1e3
        with self.lock:
            inside = [r for t, r in self.rows if t0 <= t <= self.t1]
            rows = [r for t, r in self.rows if t0 - pad <= t <= self.t1 + pad]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "in_region": len(inside),
                "region_s": round(self.t1 - t0, 4), "interval_ms": self.INTERVAL_MS}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(key):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(key)
    except Exception:
        return None


def make_opr(gila, cel, dtype, seed=1, src_cel=None, trg_org=(0, 0, 0), src_org=(0, 0, 0)):
    if src_cel is None:
        tru = tru_self(cel)
        fur = synthetic_fur(tru, dtype, seed)
        mem = gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(cel, SCL), egoFur=fur, setTyp=dtype)
        return mem, tru
    # external operator: full storage along axes whose cells / centres differ
    tru = []
    for d in range(3):
        if cel[d] == src_cel[d] and trg_org[d] == src_org[d]:
            tru.append(tru_self((cel[d],))[0])
        else:
            tru.append((cel[d] + src_cel[d]) // 2)
    fur = synthetic_fur(tru, dtype, seed)
    mem = gila.GlaOprMem(gila.GlaKerOpt(True), gila.GlaVol(cel, SCL, trg_org), gila.GlaVol(src_cel, SCL, src_org),
                         egoFur=fur, setTyp=dtype)
    return mem, tru


def job_rate(dist, ms_local, steps, world, device="cuda"):
    """Whole-job rate of `world` replicas that each ran `steps` units in
    ms_local device milliseconds: units / the max over ranks of the time (an
    all-reduce every rank takes).  Returns (units per second, max ms)."""
    import torch
    t = torch.tensor([float(ms_local)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    return world * steps / (ms_max / 1e3), ms_max


def device_rate(torch, mem, cel_in, cel_out, tdt, steps, warmup, stream, flush, seed=3, clk=None):
    """matvec/s with device-resident vectors; per-step CUDA events, L2
    flushed between steps (outside the events)."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn((3, cel_in[2], cel_in[1], cel_in[0]), dtype=tdt, device="cuda", generator=g)
    y = torch.empty((3, cel_out[2], cel_out[1], cel_out[0]), dtype=tdt, device="cuda")
    sp = stream.cuda_stream
    for _ in range(warmup):
        mem.apply_into(x, y, stream=sp)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if clk:
        clk.begin()
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            ev[k][0].record(stream)
            mem.apply_into(x, y, stream=sp)
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    if clk:
        clk.end()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    return ms, y


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--dtype", default="c128", choices=["c128", "c64"],
                    help="precision of the main matvec workload (c64: ComplexF32, for profiling)")
    ap.add_argument("--profile", choices=["solve", "build", "matvec256"], default=None,
                    help="run a small bounded workload for a profiler instead of the bench: 'solve' = two "
                         "short mixed-precision solves on 96x96x48, 'build' = the GPU kernel build of a 32^3 "
                         "self operator, 'matvec256' = 4 matvecs of the 256x256x128 self operator in the "
                         "precision of --dtype; prints no bench line")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests of the Poisson stream of the serving leg")
    ap.add_argument("--serve-closed-s", type=float, default=60.0,
                    help="seconds of the closed loop that measures the serving saturation rate")
    a = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        if rank != 0:
            return 0
        return run_reference(a, world)
    if a.profile:
        return run_profile(a.profile, a.dtype)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    gila = load_pkg()
    gila.default_context(local)

    f32 = a.dtype == "c64"
    ndt, tdt, cs = (np.complex64, torch.complex64, 8) if f32 else (np.complex128, torch.complex128, 16)
    mem, tru = make_opr(gila, CEL, ndt)
    mem.reserve(1)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    W = max(a.warmup, 3)

    # ---- value: device-resident inputs
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    ms, y_dev = device_rate(torch, mem, CEL, CEL, tdt, a.steps, W, stream, flush, clk=clk)
    clocks = clk.stop()
    value, ms_max = job_rate(dist, ms, a.steps, world)

    # ---- e2e: public API with pinned host buffers, copies inside the timed
    # region.  The host vectors go to the API E2E_BATCH at a time; the call
    # uploads each vector, applies G and downloads the result, overlapping
    # the copies of neighbouring vectors with the passes, and returns when
    # the results are in host memory.
    # all timed vectors in one call on one GPU (up to 32: 25.8 GB pinned), so
    # that only one upload and one download per call go unoverlapped; 4 per
    # rank when several ranks share the host
    kb = max(1, min(E2E_BATCH if world == 1 else 4, a.steps))
    xh = torch.randn((kb, 3, CEL[2], CEL[1], CEL[0]), dtype=tdt).pin_memory()
    yh = torch.empty_like(xh).pin_memory()
    sp = stream.cuda_stream
    for _ in range(max(1, W // kb)):
        mem.apply_into(xh, yh, nrhs=kb, stream=sp)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    done = 0
    while done < a.steps:
        n = min(kb, a.steps - done)
        mem.apply_into(xh[:n], yh[:n], nrhs=n, stream=sp)
        done += n
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_value, _ = job_rate(dist, e0.elapsed_time(e1), a.steps, world)
    nbytes = xh[0].numel() * xh.element_size()
    copy_bound = pinned_copy_rate(torch, xh, yh)

    # ---- roofline of the dominant kernel (z pass), timed live
    passes = mem.time_passes(1, reps=max(3, min(a.steps, 10)))
    zb = zpass_bytes(CEL, CEL, tru, cs)
    peak, peak_kind = measured_peak()
    achieved = zb / (passes[1] / 1e3) / 1e9
    traffic = ncu_traffic(f"z_pass_{a.dtype}_256x256x128")
    roofline = {"bound": "hbm",
                "kernel": f"{'k_zg2_ct' if f32 else 'k_zg_ct'}<{2 * CEL[2]},{mem.tiles[3]}>" + " (z pencils: register-fed forward "
                          "FFT, 3x3 multiply fused with the last / first butterflies, inverse FFT truncated to the "
                          "target)",
                "achieved": round(achieved, 1), "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic,
                "algorithmic_bytes_per_launch": zb, "launch_ms": round(passes[1], 4),
                "pass_ms": {"xy_fwd": round(passes[0], 4), "z": round(passes[1], 4), "yx_inv": round(passes[2], 4)},
                "matvec_tmin_bytes": tmin_bytes(CEL, CEL, tru, cs),
                "matvec_tmin_frac": round(tmin_bytes(CEL, CEL, tru, cs) / (ms_max / a.steps / 1e3) / 1e9 / peak, 4)}

    out = {
        "metric": METRIC if not f32 else METRIC.replace("ComplexF64", "ComplexF32"), "value": round(value, 2),
        "unit": "matvec/s", "n_gpus": world, "steps": a.steps,
        "warmup": W, "ms_per_step": round(ms_max / a.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if f32 else "f64",
        "data": "synthetic: seeded N(0,1) currents, seeded synthetic Fourier kernel of the reference's storage shapes",
        "config": bench_config(f32, world),
        "e2e": {"value": round(e2e_value, 2), "unit": "matvec/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes,
                "api": f"GlaOprMem.apply_into with pinned host tensors, {kb} vectors per call (copies overlap the passes)",
                "copy_bound": copy_bound, "frac_of_copy_bound": round(e2e_value / world / copy_bound["vectors_per_s"], 4)},
        "gpu_launches": int(mem.launches_per_apply(1)) * a.steps,
        "roofline": roofline,
        "clocks": clocks,
    }

    if rank == 0 and world == 1 and not a.no_cpu:
        out["cpu_baseline"], xo, yo = cpu_baseline()
        out["oracle_check"] = oracle_check(gila, xo, yo)
    if not a.no_sweep and world == 1:
        out["sweep"] = sweep(torch, gila, stream, flush)
    if not a.no_solve and world == 1:
        out["solve"] = solve_bench(torch, gila)
    if not a.no_serve and world == 1:
        out["serve"] = serve_bench(gila, a.serve_requests, a.serve_closed_s)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def sweep(torch, gila, stream, flush):
    """The ComplexF32 leg of the bench workload and the matvec precision sweep
    configuration: self 128x128x64 (ComplexF64 and ComplexF32, one and four
    vectors per apply) and external 64^3 -> 64x64x32 offset 80 cells along x."""
    res = {}
    peak, _ = measured_peak()
    mem, tru = make_opr(gila, CEL, np.complex64)
    ms, _ = device_rate(torch, mem, CEL, CEL, torch.complex64, 10, 3, stream, flush)
    tm = tmin_bytes(CEL, CEL, tru, 8)
    res["self_256x256x128_complex64"] = {"ms": round(ms / 10, 4), "matvec_per_s": round(1e4 / ms, 2), "tmin_bytes": tm,
                                         "tmin_frac": round(tm / (ms / 10 / 1e3) / 1e9 / peak, 4)}
    del mem
    c = SWEEP_CEL
    for dt, tdt, cs in ((np.complex128, torch.complex128, 16), (np.complex64, torch.complex64, 8)):
        mem, tru = make_opr(gila, c, dt)
        ms, _ = device_rate(torch, mem, c, c, tdt, 20, 3, stream, flush)
        res[f"self_128x128x64_{np.dtype(dt).name}"] = {
            "ms": round(ms / 20, 4), "matvec_per_s": round(2e4 / ms, 2),
            "tmin_frac": round(tmin_bytes(c, c, tru, cs) / (ms / 20 / 1e3) / 1e9 / peak, 4)}
        del mem
    # external 64^3 -> 64x64x32, target offset 80 cells along x
    for dt, tdt, cs in ((np.complex128, torch.complex128, 16), (np.complex64, torch.complex64, 8)):
        src, trg = (64, 64, 64), (64, 64, 32)
        mem, tru = make_opr(gila, trg, dt, src_cel=src, trg_org=("80/32", 0, 0))
        ms, _ = device_rate(torch, mem, src, trg, tdt, 10, 3, stream, flush)
        res[f"external_64cube_to_64x64x32_{np.dtype(dt).name}"] = {
            "ms": round(ms / 10, 4), "matvec_per_s": round(1e4 / ms, 2),
            "tmin_frac": round(tmin_bytes(src, trg, tru, cs) / (ms / 10 / 1e3) / 1e9 / peak, 4)}
        del mem
    # four vectors per apply (batched launches), per-vector time, L2 flushed between applies
    for dt, tdt, cs in ((np.complex128, torch.complex128, 16), (np.complex64, torch.complex64, 8)):
        mem, tru = make_opr(gila, c, dt)
        nb = 4
        g = torch.Generator(device="cuda").manual_seed(5)
        xb = torch.randn((nb, 3, c[2], c[1], c[0]), dtype=tdt, device="cuda", generator=g)
        yb = torch.empty_like(xb)
        mem.autotune(nb)
        for _ in range(3):
            mem.apply_into(xb, yb, nrhs=nb, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(10)]
        with torch.cuda.stream(stream):
            for e0, e1 in evs:
                flush.zero_()
                e0.record(stream)
                mem.apply_into(xb, yb, nrhs=nb, stream=stream.cuda_stream)
                e1.record(stream)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs) / (10 * nb)
        res[f"self_128x128x64_{np.dtype(dt).name}_4_per_apply"] = {
            "ms_per_vector": round(ms, 4), "matvec_per_s": round(1e3 / ms, 2),
            "tmin_frac": round(tmin_bytes(c, c, tru, cs) / (ms / 1e3) / 1e9 / peak, 4)}
        del mem, xb, yb
    torch.cuda.empty_cache()
    return res


def plane_wave(cel, theta_deg=80.5):
    """s-polarised plane wave y exp(i 2 pi k.r), k = (sin t, 0, -cos t), r in
    wavelengths at the cell corners (1/32-wavelength cells); numpy (Nx,Ny,Nz,3)."""
    t = math.radians(theta_deg)
    h = 1.0 / 32
    x = np.arange(cel[0]) * h
    z = np.arange(cel[2]) * h
    ph = np.exp(2j * math.pi * (math.sin(t) * x[:, None, None] - math.cos(t) * z[None, None, :]))
    e = np.zeros((*cel, 3), dtype=np.complex128, order="F")
    e[..., 1] = np.broadcast_to(ph, cel)
    return e


def _warm_solve(torch, gila, ls, b, **kw):
    """A short untimed solve that leaves the batch (Krylov vectors,
    workspaces, captured graphs, tuned tiles) resident for the timed one."""
    kw = dict(kw, max_matvecs=8, check=False, keep=True)
    gila.solve(ls, b, **kw)
    torch.cuda.synchronize()


def _timed_solve(torch, gila, ls, b, **kw):
    st = torch.cuda.Stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    x, info = gila.solve(ls, b, stream=st.cuda_stream, **kw)
    e1.record(st)
    torch.cuda.synchronize()
    return x, info, e0.elapsed_time(e1)


def _info(info, ms, nrhs=1):
    return {"ms": round(ms, 1), "solves_per_s": round(nrhs / (ms / 1e3), 3), "cycles": info.iters,
            "fp64_updates": info.outer, "matvecs_f64": info.matvecs_f64, "matvecs_f32": info.matvecs_f32,
            "rel_res_max": info.rel_res, "converged": info.converged}


def pinned_copy_rate(torch, xh, yh, reps=3):
    """The rate the host link allows the end-to-end path: the same pinned
    vectors copied host -> device and device -> host at once (two streams,
    no compute), best of reps, in vectors per second and GB/s per direction."""
    k = xh.shape[0]
    d_in = torch.empty_like(xh[0], device="cuda")
    d_out = torch.empty_like(yh[0], device="cuda")
    s_up, s_down = torch.cuda.Stream(), torch.cuda.Stream()
    best = float("inf")
    for _ in range(reps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        s_up.wait_event(e0)
        s_down.wait_event(e0)
        for i in range(k):
            with torch.cuda.stream(s_up):
                d_in.copy_(xh[i], non_blocking=True)
            with torch.cuda.stream(s_down):
                yh[i].copy_(d_out, non_blocking=True)
        torch.cuda.current_stream().wait_stream(s_up)
        torch.cuda.current_stream().wait_stream(s_down)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    nb = xh[0].numel() * xh.element_size()
    return {"vectors_per_s": round(k / best * 1e3, 1), "gbps_per_direction": round(nb * k / best / 1e6, 2),
            "how": f"{k} pinned vectors uploaded and downloaded at once on two streams, no compute"}


def solve_bench(torch, gila):
    """The scattering solves (I - chi G) E = E_inc: the 256x256x128 thin film
    (chi = 3+0.1i on a centred 24-cell z slab, s-polarised plane wave at 80.5
    degrees) plain FP64 vs ComplexF32 Krylov with FP64 reliable updates, and
    64 point-dipole right-hand sides on 96^3 with a centred 48^3 inclusion
    (chi ~ U[0,3] seeded) solved as one batch.  BiCGStab(2) to FP64 relative
    residual 1e-6; kernels built on the GPU; inputs device-resident; each
    timed solve follows a short untimed one of the same shape and variant
    that leaves the batch's device state resident (keep=True), as a service
    would."""
    res = {}
    opt = gila.GlaKerOpt(1.0 + 0j, 32, False, True, (), ())
    # thin film
    cel = (256, 256, 128)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    G = gila.GlaOpr(gila.GlaOprMem(opt, gila.GlaVol(cel, SCL)))
    torch.cuda.synchronize()
    tb = time.perf_counter() - t0
    chi = np.zeros(cel, dtype=np.complex128, order="F")
    chi[:, :, 52:76] = 3.0 + 0.1j
    ls = gila.LippmannSchwinger(G, chi)
    ls.g32()
    b = torch.from_numpy(np.ascontiguousarray(plane_wave(cel).reshape(-1, order="F"))).cuda()
    b = b.reshape(3, cel[2], cel[1], cel[0])
    # the operator keeps one solve batch resident: each variant's timed solve
    # directly follows its own warm-up
    _warm_solve(torch, gila, ls, b, mixed=True)
    xm, im, msm = _timed_solve(torch, gila, ls, b, mixed=True, max_matvecs=20000, keep=True)
    _warm_solve(torch, gila, ls, b, mixed=False)
    xp, ip, msp = _timed_solve(torch, gila, ls, b, mixed=False, max_matvecs=20000, keep=True)
    diff = float(torch.linalg.vector_norm(xm - xp) / torch.linalg.vector_norm(xp))
    res["film_256x256x128"] = {"kernel_build_s": round(tb, 2), "plain_fp64": _info(ip, msp),
                               "mixed_c64_reliable": _info(im, msm),
                               "speedup_mixed_vs_plain": round(msp / msm, 3),
                               "field_rel_l2_mixed_vs_plain": diff}
    del ls, G, xm, xp, b
    torch.cuda.empty_cache()
    # 64 dipoles, one batch
    cel = (96, 96, 96)
    nr = 64
    G = gila.GlaOpr(gila.GlaOprMem(opt, gila.GlaVol(cel, SCL)))
    rng = np.random.default_rng(4)
    chi = np.zeros(cel, dtype=np.complex128, order="F")
    chi[24:72, 24:72, 24:72] = rng.uniform(0.0, 3.0, (48, 48, 48))
    ls = gila.LippmannSchwinger(G, chi)
    ls.g32()
    D = torch.zeros((nr, 3, cel[2], cel[1], cel[0]), dtype=torch.complex128)
    k = 0
    while k < nr:
        p = rng.integers(0, 96, 3)
        if np.all(p >= 24) and np.all(p < 72):
            continue
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        for c in range(3):
            D[k, c, p[2], p[1], p[0]] = complex(v[c])
        k += 1
    D = D.cuda()
    B = torch.empty_like(D)
    G.mem.apply_into(D, B, nrhs=nr)   # incident fields G d_j
    # best of two timed solves per variant (each a few seconds), after the
    # variant's own warm-up
    runs = {True: [], False: []}
    for mixed in (True, False):
        _warm_solve(torch, gila, ls, B, mixed=mixed)
        for _ in range(2):
            runs[mixed].append(_timed_solve(torch, gila, ls, B, mixed=mixed, max_matvecs=20000, keep=True))
    xm, im, msm = min(runs[True], key=lambda r: r[2])
    xp, ip, msp = min(runs[False], key=lambda r: r[2])
    res["dipoles_96cube_64rhs"] = {"plain_fp64": _info(ip, msp, nr), "mixed_c64_reliable": _info(im, msm, nr),
                                   "speedup_mixed_vs_plain": round(msp / msm, 3),
                                   "ms_each_run": {"plain_fp64": [round(r[2], 1) for r in runs[False]],
                                                   "mixed_c64_reliable": [round(r[2], 1) for r in runs[True]]},
                                   "timing": "best of two timed solves per variant"}
    del runs
    del ls, G, xm, xp, B, D
    torch.cuda.empty_cache()
    return res


SERVE_SHAPES = [(32, 32, 32), (64, 64, 64), (96, 96, 48), (128, 128, 64), (192, 192, 96)]


def serve_request(cel, rng):
    """A cube or slab inclusion with chi = U[0.5,4] + i U[0,0.2] and one
    s-polarised plane wave at a random angle in the xz plane."""
    chi = np.zeros(cel, dtype=np.complex128, order="F")
    val = rng.uniform(0.5, 4.0) + 1j * rng.uniform(0.0, 0.2)
    if rng.random() < 0.5:
        lo = [n // 4 for n in cel]
        hi = [n - n // 4 for n in cel]
        chi[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = val
    else:
        z0 = cel[2] // 3
        chi[:, :, z0:cel[2] - z0] = val
    th = rng.uniform(0.0, math.pi)
    h = 1.0 / 32
    x = np.arange(cel[0]) * h
    z = np.arange(cel[2]) * h
    ph = np.exp(2j * math.pi * (math.sin(th) * x[:, None, None] + math.cos(th) * z[None, None, :]))
    b = np.zeros((*cel, 3), dtype=np.complex128, order="F")
    b[..., 1] = np.broadcast_to(ph, cel)
    return chi, b


def serve_bench(gila, n_stream, closed_s=60.0, clients=40):
    """The request stream: solves of volumes drawn uniformly from
    SERVE_SHAPES (1/32-wavelength cells), each with its own medium and
    incident wave, tol 1e-6, ComplexF32 Krylov with FP64 reliable updates.

    Saturation is the sustained completion rate of a closed loop: `clients`
    requests are kept outstanding for `closed_s` seconds, each completion
    immediately replaced by a new request of a uniformly drawn shape.  Only
    completions after the first third of the loop count: by then the slow
    shapes' requests have accumulated to their steady-state share of the
    outstanding set, so the counted completions follow the uniform mix and the
    rate is what the server sustains on it (a burst, or the loop's start,
    over-represents the fast shapes).  Then
    n_stream requests drawn the same way arrive as a Poisson process at 80%
    of that rate (seeded); latency is submit -> solution in the caller's
    buffer.  The queue (requests waiting for a slot) and the running count are
    sampled every 0.5 s during the stream.  Inputs come from a pool of 3
    seeded variants per shape."""
    rng = np.random.default_rng(11)
    pool = {c: [serve_request(c, rng) for _ in range(3)] for c in SERVE_SHAPES}
    srv = gila.SolveServer(slots=8, mixed=True)
    key = lambda c: "x".join(map(str, c))  # noqa: E731
    res = {"shapes": [key(c) for c in SERVE_SHAPES], "tol": 1e-6}
    try:
        # operators (built on the GPU) and one solve per shape, alone
        alone = {}
        for c in SERVE_SHAPES:
            t0 = time.perf_counter()
            _, inf, lat = srv.wait(srv.submit(c, SCL, *pool[c][0]))
            alone[key(c)] = {"first_ms_incl_build": round((time.perf_counter() - t0) * 1e3, 1)}
            _, inf, lat = srv.wait(srv.submit(c, SCL, *pool[c][0]))
            alone[key(c)].update({"ms": round(lat, 1), "cycles": inf.iters})
        res["alone"] = alone
        # saturation: closed loop of `clients` outstanding requests
        t0 = time.perf_counter()
        t_stop = t0 + closed_s
        t_count = t0 + closed_s / 3
        done_at, lock = [], threading.Lock()

        def client(seed):
            r = np.random.default_rng(seed)
            while time.perf_counter() < t_stop:
                c = SERVE_SHAPES[int(r.integers(0, len(SERVE_SHAPES)))]
                srv.wait(srv.submit(c, SCL, *pool[c][int(r.integers(0, 3))]))
                with lock:
                    done_at.append((time.perf_counter(), key(c)))

        th = [threading.Thread(target=client, args=(100 + i,)) for i in range(clients)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        counted = [k for t, k in done_at if t_count <= t <= t_stop]
        sat = len(counted) / (t_stop - t_count)
        res["saturation"] = {"solves_per_s": round(sat, 3), "completed_in_window": len(counted),
                             "window_s": round(t_stop - t_count, 1), "loop_s": round(closed_s, 1),
                             "outstanding": clients,
                             "window_mix": {k: counted.count(k) for k in res["shapes"]},
                             "how": "closed loop, uniform shape per new request; completions of the last two thirds"}
        # Poisson stream at 80% of saturation
        lam = 0.8 * sat
        picks = [SERVE_SHAPES[i] for i in rng.integers(0, len(SERVE_SHAPES), n_stream)]
        gaps = rng.exponential(1.0 / lam, n_stream)
        samples, sampling = [], [True]
        t_start = time.perf_counter()

        def sampler():
            while sampling[0]:
                st = srv.stats()
                samples.append((round(time.perf_counter() - t_start, 2), st["queued"], st["running"]))
                time.sleep(0.5)

        sm = threading.Thread(target=sampler, daemon=True)
        sm.start()
        tk = []
        t_next = t_start
        for c, g in zip(picks, gaps):
            t_next += g
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tk.append((c, srv.submit(c, SCL, *pool[c][int(rng.integers(0, 3))])))
        t_arrived = time.perf_counter() - t_start
        lats, conv, per = [], 0, {}
        for c, t in tk:
            _, inf, lat = srv.wait(t)
            lats.append(lat)
            conv += inf.converged
            per.setdefault(key(c), []).append(lat)
        wall = time.perf_counter() - t_start
        sampling[0] = False
        sm.join(timeout=2)
        lats = np.array(lats)
        p99 = float(np.percentile(lats, 99))
        tail = {}
        for c, t in zip(picks, lats):
            if t >= p99:
                tail[key(c)] = tail.get(key(c), 0) + 1
        step = max(1, len(samples) // 120)
        q = [s_[1] for s_ in samples]
        res.update({
            "requests": n_stream, "arrival_rate_per_s": round(lam, 3), "arrivals_s": round(t_arrived, 1),
            "solves_per_s": round(n_stream / wall, 3),
            "p50_ms": round(float(np.percentile(lats, 50)), 1), "p99_ms": round(p99, 1),
            "mean_ms": round(float(lats.mean()), 1), "converged": conv,
            "by_shape": {k: {"n": len(v), "p50_ms": round(float(np.median(v)), 1),
                             "p99_ms": round(float(np.percentile(v, 99)), 1)} for k, v in sorted(per.items())},
            "p99_tail_shapes": tail,
            "queue": {"max": max(q) if q else 0, "mean": round(float(np.mean(q)), 2) if q else 0,
                      "last_third_mean": round(float(np.mean(q[2 * len(q) // 3:])), 2) if q else 0,
                      "samples_t_queued_running": samples[::step]},
            "server": srv.stats()})
    finally:
        srv.close()
    return res


def _oracle_setup():
    """The bench operator and input on the CPU oracle (restatement of
    egoBrnHst!, scipy.fft on all host threads)."""
    from oracle.gla_mem import ExtInf, Vol
    from oracle.matvec import OprMem, use_fft_workers
    n = os.cpu_count() or 1
    use_fft_workers(n)
    v = Vol.make(CEL, SCL)
    mix = ExtInf.make(v, v)
    fur = synthetic_fur(tru_self(CEL), np.complex128, 1)
    rng = np.random.default_rng(3)
    x = rng.standard_normal((*CEL, 3)) + 1j * rng.standard_normal((*CEL, 3))
    return OprMem(mix, fur), x, n


def cpu_baseline():
    """The oracle's restatement of the reference host path (egoBrnHst!) with
    scipy.fft on all host threads, on the same configuration: a bounded
    sample of one matvec (about 15-25 s of CPU work), whose result also
    checks the GPU matvecs."""
    from oracle.matvec import ego_opr
    om, x, n = _oracle_setup()
    t0 = time.perf_counter()
    y = ego_opr(om, x)
    dt = time.perf_counter() - t0
    return {"value": round(1 / dt, 4), "unit": "matvec/s", "cores": n, "kind": "port",
            "sample": f"1 matvec of the same 256x256x128 ComplexF64 self operator (numpy/scipy.fft "
                      f"restatement of egoBrnHst!: FFT workers={n}, the recursion's branches on concurrent threads "
                      f"as the reference spawns them)"}, x, y


def oracle_check(gila, x, y_ref):
    """Relative L2 error of the GPU ComplexF64 and ComplexF32 matvecs of the
    bench operator (256x256x128) against the oracle's FP64 result on the same
    input (the ComplexF32 operator holds the same kernel values rounded)."""
    out = {}
    xf = np.asfortranarray(x)
    for dt, key in ((np.complex128, "rel_l2_f64"), (np.complex64, "rel_l2_f32")):
        mem, _ = make_opr(gila, CEL, dt)
        yg = np.asarray(gila.egoOpr(mem, xf.astype(dt))).astype(np.complex128)
        out[key] = float(np.linalg.norm((yg - y_ref).ravel()) / np.linalg.norm(y_ref.ravel()))
        del mem, yg
    out["tolerance"] = {"f64": 1e-12, "f32": 1e-5}
    out["input"] = ("seeded N(0,1) current (seed 3) through the 256x256x128 bench operator; oracle: FP64 "
                    "restatement of egoBrnHst!")
    return out


def run_profile(kind, dtype="c128"):
    """Small bounded workloads whose every kernel a profiler's launch list
    can cover: the Krylov-cycle kernels of the solver (two solves of 12
    matvecs, ComplexF32 with FP64 reliable updates, on 96x96x48 with a slab
    medium; the first one also sets up the batch and its graphs) or the GPU
    kernel build (32^3 self operator, intOrd 16)."""
    import torch
    gila = load_pkg()
    if kind == "matvec256":
        cel = (256, 256, 128)
        ndt, tdt = (np.complex64, torch.complex64) if dtype == "c64" else (np.complex128, torch.complex128)
        mem, _ = make_opr(gila, cel, ndt)
        g = torch.Generator(device="cuda").manual_seed(3)
        x = torch.randn((3, cel[2], cel[1], cel[0]), dtype=tdt, device="cuda", generator=g)
        y = torch.empty_like(x)
        for _ in range(4):
            mem.apply_into(x, y)
        torch.cuda.synchronize()
        return 0
    if kind == "build":
        opt = gila.GlaKerOpt(1.0 + 0j, 16, False, True, (), ())
        gila.GlaOprMem(opt, gila.GlaVol((32, 32, 32), SCL))
        torch.cuda.synchronize()
        return 0
    cel = (96, 96, 48)
    mem, _ = make_opr(gila, cel, np.complex128)
    G = gila.GlaOpr(mem)
    chi = np.zeros(cel, dtype=np.complex128, order="F")
    chi[:, :, 12:36] = 3.0 + 0.1j
    ls = gila.LippmannSchwinger(G, chi)
    ls.g32()
    b = torch.from_numpy(np.ascontiguousarray(plane_wave(cel).reshape(-1, order="F"))).cuda()
    b = b.reshape(3, cel[2], cel[1], cel[0])
    for _ in range(2):
        gila.solve(ls, b, tol=1e-6, mixed=True, max_matvecs=12, check=False, keep=True)
    torch.cuda.synchronize()
    return 0


def run_reference(a, world):
    """--impl reference: the reference's CPU path (egoBrnHst!, restated in
    the oracle; the Julia package cannot run on this image) on all host
    threads, same configuration and metric."""
    from oracle.matvec import ego_opr
    om, x, n = _oracle_setup()
    t0 = time.perf_counter()
    ego_opr(om, x)  # warm-up (one, to bound the CPU run)
    per = time.perf_counter() - t0
    budget = 60.0
    k = max(1, min(a.steps, int(budget / max(per, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(k):
        ego_opr(om, x)
    dt = time.perf_counter() - t0
    val = k / dt
    sample = (f"{k} of {a.steps} requested steps timed after 1 warm-up (1 matvec each; the rest skipped to bound "
              f"the CPU run), numpy/scipy.fft restatement of egoBrnHst! with FFT workers={n} and the recursion's "
              f"branches on concurrent threads")
    out = {"impl": "reference", "metric": METRIC if a.dtype == "c128" else METRIC.replace("ComplexF64", "ComplexF32"),
           "value": round(val, 4), "unit": "matvec/s", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(dt / k * 1e3, 2), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32" if a.dtype == "c64" else "f64",
           "data": "synthetic: seeded N(0,1) currents, seeded synthetic Fourier kernel of the reference's storage shapes",
           "config": bench_config(a.dtype == "c64", world),
           "cpu_baseline": {"value": round(val, 4), "unit": "matvec/s", "cores": n, "kind": "port", "sample": sample},
           "e2e": {"value": round(val, 4), "unit": "matvec/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
