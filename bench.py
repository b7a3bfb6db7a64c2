#!/usr/bin/env python
"""Benchmark of the range-Doppler focusing path on B200.

Metric: raw Msamples/s focused = (range samples x azimuth lines of every scene) / time.
One step = one full focus of one ERS-like 5616 x 28000 5-bit scene (the headline
single-GPU configuration): raw I/Q bytes resident in HBM -> IQ statistics + Doppler
centroid -> range compression -> azimuth FFT / RCMC / matched filter / IFFT -> results
window -> 5-look multilook + range spreading loss -> slant-to-ground resampling.
The scene is synthetic (seeded point-target grid on clutter), generated on the device.

Multi-GPU: one process per GPU (torchrun), each rank focuses its own scene (independent
units, no data-path collective: weak scaling); timing is the max over ranks.

--impl reference runs the reference's own CUDA build (oracle/_ref/libasar_ref.so, the
asar-focus sar/ + cuda_util/ sources compiled for sm_100a with cuFFT) on the same scene.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "asar-focus_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "raw Msamples/s focused on 1 B200 (ERS-like 5616x28000, plain FP32)"
UNIT = "Msamples/s"
HBM_FALLBACK = 6650.0
E2E_DEPTH = 3  # plans (scenes in flight) of the end-to-end leg
KERNELS = ["raw_stats", "finalize", "range_compress", "az_strided_fwd", "az_rd", "az_strided_inv", "tail"]


def _peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            pass
    return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi's start-up holds driver locks that stall allocating CUDA calls (the
        # reference allocates in every step): time nothing until its first sample is in
        t0 = time.time()
        while not self.lines and time.time() - t0 < 10.0:
            time.sleep(0.05)
        time.sleep(0.3)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend=backend, timeout=timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return rank, world, local


def _max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def _barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _describe(sc) -> str:
    kind = "ASAR IM-like" if sc.bits == 8 else "ERS-like"
    fmt = "FBAQ4 records (synthetic tables)" if sc.raw_format == "fbaq4" else f"{sc.bits}-bit I/Q"
    dc = f"Doppler {sc.dc_coeffs[0]:+.0f} Hz + range terms" if sc.dc_kind == "poly" else \
        f"Doppler drifting +-{sc.dc_drift:.0f} Hz along azimuth"
    grid = f"{sc.grid[0]}x{sc.grid[1]} point grid"
    vr = "Vr from the orbit state vectors" if sc.vr_given is None else f"Vr {sc.vr_given:.0f} m/s"
    return f"{kind} {sc.range_size} range x {sc.azimuth_size} azimuth, {fmt}, {grid}, {dc}, {vr}"


def make_scene(workload: str, seed: int, azimuth_size: int = 0):
    """The workload's scene; azimuth_size > 0 cuts it to that many lines (profiling cases)."""
    from asarf import scene as S
    return S.WORKLOADS[workload](seed=seed, **({"azimuth_size": azimuth_size} if azimuth_size else {}))


def algorithmic_bytes(sc, dims: dict, res: dict) -> dict:
    """Minimal HBM bytes each kernel must move (inputs read once, outputs written once,
    no halo, no padding rows), per launch."""
    na = sc.azimuth_size
    nk, az = dims["nk"], dims["az_pad"]
    nx = dims["slc_cols"]
    raw = na * sc.raw_line_bytes
    nl = res["n_lines"]
    out = res["out_rows"] * res["out_cols"] * 4
    return {"raw_stats": raw, "finalize": 0, "range_compress": raw + na * nk * 8,
            "az_strided_fwd": na * nk * 8 + az * nk * 8, "az_rd": 2 * az * nk * 8,
            "az_strided_inv": az * nk * 8 + nl * nk * 8, "tail": nl * nx * 8 + out}


def pipeline_bytes(sc, dims: dict, res: dict) -> float:
    """Algorithmic bytes of the whole scene: raw read twice, two complex round trips,
    multilooked float round trip, ground-range output write (unpadded sizes)."""
    na = sc.azimuth_size
    nk = dims["nk"]
    L = 5.0
    ng = res["out_cols"]
    return na * sc.raw_line_bytes * 2 + 32 * nk * na + 8 * nk * na / L + 4 * ng * na / L


def _traffic_from_profiles(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` from a committed ncu summary, if one exists."""
    for f in sorted((ROOT / "profiles").glob(f"*{kernel}*{workload}*.txt")):
        for line in f.read_text().splitlines():
            if line.startswith("dram_bytes_per_launch:"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    pass
    return None


def _cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _slc_of(plan, res):
    import torch
    d = torch.empty((res["n_lines"], plan.dims["slc_cols"]), dtype=torch.complex64, device="cuda")
    plan.slc_into(d, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return d.cpu().numpy()


def _rel_rmse(a, b) -> float:
    import numpy as np
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


def cpu_baseline_and_quality(sc_full, lib, forms: dict) -> tuple[dict, dict]:
    """The FP64 CPU oracle on a bounded sample of the workload, timed on the host cores: a
    4096-line scene with the same sensor, chirp, PRF, orbit and Doppler parameters and a 6 x 4
    point grid (seeded).  Its outputs are also what the quality block compares every GPU form
    against: detected-intensity and SLC relative RMSE, and per point target the deviation of
    resolution, PSLR, ISLR and peak phase (the same tolerances the tests hold)."""
    import numpy as np
    from dataclasses import replace
    import asarf
    from asarf import sim
    from oracle import irf, rda
    lines = 4096
    sc = replace(sc_full, azimuth_size=lines, grid=(6, 4), osv=[], vr_poly=None, seed=sc_full.seed + 7)
    sc.prepare(lib)
    raw, truth = sim.simulate(sc, device="cuda")
    t0 = time.perf_counter()
    ref = rda.focus(raw, sc.to_dict())
    dt = time.perf_counter() - t0
    n = sc.range_size * lines
    # the small ERS configuration in full (2048 x 4096), timed the same way
    from asarf import scene as S
    s0 = S.ers_small()
    s0.prepare(lib)
    raw0, _ = sim.simulate(s0, device="cuda")
    t1 = time.perf_counter()
    rda.focus(raw0, s0.to_dict())
    dt0 = time.perf_counter() - t1
    base = {"value": round(n / dt / 1e6, 3), "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
            "cpu_model": _cpu_model(),
            "ers_small_full": {"value": round(s0.range_size * s0.azimuth_size / dt0 / 1e6, 3), "unit": UNIT,
                               "seconds": round(dt0, 2), "scene": "ERS-like 2048 x 4096, whole scene"},
            "sample": f"{sc.range_size} x {lines} scene with the workload's parameters and a 6x4 point grid "
                      f"({n / 1e6:.1f} Msamples) through the numpy FP64 oracle (scipy.fft workers=all cores), "
                      f"{dt:.1f} s"}
    quality = {}
    for name, prec in forms.items():
        plan = asarf.FocusPlan(sc, lib=lib, precision=prec)
        out = plan.focus_host(raw)
        res = plan.results()
        slc = _slc_of(plan, res)
        q = {"detected_rel_rmse": _rel_rmse(out, ref.detected), "slc_rel_rmse": _rel_rmse(slc, ref.slc),
             "res_rel_max": 0.0, "pslr_db_max": 0.0, "islr_db_max": 0.0, "phase_mrad_max": 0.0, "targets": 0}
        first = res["first_line"]
        for (xt, yt) in truth["targets"]:
            y, x = yt - first, xt - 8
            if not (40 <= y < slc.shape[0] - 40 and 40 <= x < slc.shape[1] - 40):
                continue
            lo, hi = int(max(0, y - 400)), int(min(slc.shape[0], y + 400))
            blk = np.abs(ref.slc[lo:hi, int(x) - 6:int(x) + 7])
            py, px = np.unravel_index(np.argmax(blk), blk.shape)
            a = irf.analyse(slc, lo + py, int(x) - 6 + px)
            b = irf.analyse(ref.slc, lo + py, int(x) - 6 + px)
            if not a or not b:
                continue
            d = irf.compare(a, b)
            q["res_rel_max"] = max(q["res_rel_max"], d["res_az_rel"], d["res_rg_rel"])
            q["pslr_db_max"] = max(q["pslr_db_max"], d["pslr_az_db"], d["pslr_rg_db"])
            q["islr_db_max"] = max(q["islr_db_max"], d["islr_db"])
            q["phase_mrad_max"] = max(q["phase_mrad_max"], 1e3 * d["phase_rad"])
            q["targets"] += 1
        q = {k: (float(f"{v:.3g}") if isinstance(v, float) else v) for k, v in q.items()}
        q["precision"] = "split" if plan.dims["precision"] else "fp32"
        quality[name] = q
        plan.close()
    quality["against"] = ("FP64 oracle on the " + base["sample"].split(" through")[0] +
                          "; tolerances: rel. RMSE 1e-4, resolution 1 %, PSLR 0.1 dB, ISLR 0.2 dB, phase 1 mrad")
    return base, quality


def _e2e_leg(args, sc, plan, lib, raw_np, opts, stream, st, world):
    """End to end through the public host API: pinned raw in, detected image out, every step.
    Scenes go round-robin to E2E_DEPTH plans, each on its own stream, so that one scene's
    upload and another's download overlap a third's focusing (asarf_focus_host_async)."""
    import torch
    import asarf
    samples = sc.range_size * sc.azimuth_size
    plans = [plan] + [asarf.FocusPlan(sc, lib=lib, **opts) for _ in range(E2E_DEPTH - 1)]
    raw_h = [torch.from_numpy(raw_np).pin_memory() for _ in range(E2E_DEPTH)]
    out_h = [torch.empty(plan.out_shape, dtype=torch.float32).pin_memory() for _ in range(E2E_DEPTH)]
    slot_streams = [torch.cuda.Stream() for _ in range(E2E_DEPTH)]
    for k in range(E2E_DEPTH):
        plans[k].focus_host_async(raw_h[k].data_ptr(), out_h[k].data_ptr(), stream=slot_streams[k].cuda_stream)
    torch.cuda.synchronize()
    for p_ in plans:
        if p_.results()["errors"]:
            raise RuntimeError("host run reported error flags")
    # as many scenes as the timed device steps (at least 100): the pipeline's fill and drain
    # (one scene's focusing and download) spread over the whole run
    e2e_steps = max(100, args.steps)
    _barrier(world)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for s_ in slot_streams:
        s_.wait_event(t0)
    for i in range(e2e_steps):
        k = i % E2E_DEPTH
        plans[k].focus_host_async(raw_h[k].data_ptr(), out_h[k].data_ptr(), stream=slot_streams[k].cuda_stream)
    for s_ in slot_streams:
        stream.wait_stream(s_)
    t1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = _max_over_ranks(t0.elapsed_time(t1) / e2e_steps, world)
    e2e_value = samples * world / e2e_ms / 1e3
    # the blocking call, one scene at a time (latency of a single scene), for comparison
    b0 = torch.cuda.Event(enable_timing=True)
    b1 = torch.cuda.Event(enable_timing=True)
    b0.record(stream)
    for _ in range(3):
        plan.focus_host_ptr(raw_h[0].data_ptr(), out_h[0].data_ptr(), stream=st)
    b1.record(stream)
    torch.cuda.synchronize()
    blocking_ms = _max_over_ranks(b0.elapsed_time(b1) / 3, world)
    del plans[1:]
    return e2e_value, e2e_ms, blocking_ms, out_h


def other_workloads(lib, steps: int, warmup: int) -> dict:
    """The other configurations, measured in the same run so that the default bench line
    carries them: the ASAR IM-like 5616 x 30000 8-bit scene, the same scene in FBAQ4 records,
    the 16-segment uneven batch in one CUDA graph, and the 5616 x 120000 strip in overlapped
    16384-line blocks; plain FP32, detected products, device-resident raw bytes, CUDA events
    around `steps` runs after `warmup`."""
    import torch
    import asarf
    from asarf import scene as S
    from asarf import sim
    st = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    out = {}
    for name in ("asar_im", "asar_fbaq"):
        sc = make_scene(name, 1002)
        sc.prepare(lib)
        raw = torch.from_numpy(sim.simulate(sc, device="cuda")[0]).cuda()
        plan = asarf.FocusPlan(sc, lib=lib, keep_slc=False)
        o = torch.empty(plan.out_shape, dtype=torch.float32, device="cuda")
        ms = timed(lambda: plan.focus(raw, o, stream=st.cuda_stream))
        if plan.results()["errors"]:
            raise RuntimeError(f"{name} reported error flags")
        out[name] = {"workload": _describe(sc), "ms_per_step": round(ms, 4),
                     "value": round(sc.range_size * sc.azimuth_size / ms / 1e3, 1)}
        plan.close()
        del plan, raw, o
    scenes = S.batch16()
    for sc in scenes:
        sc.prepare(lib)
    raws = [torch.from_numpy(sim.simulate(sc, device="cuda")[0]).cuda() for sc in scenes]
    batch = asarf.FocusBatch(scenes, lib=lib, options=[{"keep_slc": False}] * len(scenes))
    outs = [torch.empty(p.out_shape, dtype=torch.float32, device="cuda") for p in batch.plans]
    ms = timed(lambda: batch.focus(raws, outs, stream=st.cuda_stream))
    n = sum(sc.range_size * sc.azimuth_size for sc in scenes)
    out["batch16"] = {"workload": "16 uneven segments (ERS 5-bit / ASAR 8-bit, range 2048|5616, azimuth "
                                  "U[4000, 30000]) in one CUDA graph", "ms_per_step": round(ms, 4),
                      "value": round(n / ms / 1e3, 1)}
    batch.close()
    del batch, raws, outs
    sc = make_scene("asar_strip", 1004)
    sc.prepare(lib)
    strip = asarf.FocusStrip(sc, block_lines=16384, overlap=1400, lib=lib)
    raw = torch.from_numpy(sim.simulate(sc, device="cuda")[0]).cuda()
    o = torch.empty(strip.out_shape, dtype=torch.float32, device="cuda")
    ms = timed(lambda: strip.focus(raw, o, stream=st.cuda_stream))
    if strip.errors():
        raise RuntimeError("strip reported error flags")
    out["asar_strip"] = {"workload": "ASAR-like 5616 x 120000 8-bit strip, Doppler drift +-100 Hz, 16384-line "
                                     "blocks overlapping by 1400", "ms_per_step": round(ms, 4),
                         "value": round(sc.range_size * sc.azimuth_size / ms / 1e3, 1)}
    del strip, raw, o
    torch.cuda.empty_cache()
    return {"steps": steps, "warmup": warmup, "unit": UNIT, **out}


def run_ours(args, rank: int, world: int, local: int) -> None:
    import numpy as np
    import torch
    import asarf
    from asarf import sim

    lib = asarf.load_library()
    sc = make_scene(args.workload, 1001 + rank, args.azimuth_size)
    sc.prepare(lib)
    prec = 1 if args.precision == "split" else 0
    raw_np, _ = sim.simulate(sc, device="cuda")
    raw_d = torch.from_numpy(raw_np).cuda()
    # launch shapes: timed autotuner (a fresh cache per run, so every run tunes on its own GPU)
    tuned, tune_info = {}, None
    if not args.no_tune:
        import tempfile
        from asarf import autotune
        with tempfile.TemporaryDirectory() as td:
            cache = Path(td) / "tune.json"
            t_tune = time.perf_counter()
            tuned = autotune.tune(sc, raw_d, lib=lib, precision=prec, cache=cache, keep_slc=False)
            entry = json.loads(cache.read_text())[autotune.shape_key(sc, prec) + ":detected-only"]
            tune_info = {"options": tuned, "ms_default": round(entry["ms_default"], 4),
                         "ms_tuned": round(entry["ms_tuned"], 4), "seconds": round(time.perf_counter() - t_tune, 1),
                         "candidates": [[o, None if m is None else round(m, 4)] for o, m in entry["timings"]]}
    # the product is the detected image: no complex SLC is kept (|z|^2 rows feed the multilook)
    tuned = dict(tuned, keep_slc=bool(args.keep_slc))
    if args.az_n2:
        tuned["az_n2"] = args.az_n2
    plan = asarf.FocusPlan(sc, lib=lib, **dict(tuned, precision=prec))
    out_d = torch.empty(plan.out_shape, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    st = stream.cuda_stream
    for _ in range(args.warmup):
        plan.focus(raw_d, out_d, stream=st)
    torch.cuda.synchronize()
    res = plan.results()
    if res["errors"]:
        raise RuntimeError(f"focus reported error flags {res['errors']:#x}")
    _barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.25)
    plan.enable_timing(args.steps)
    # one event between consecutive steps: the mean over the K steps is the headline, the
    # median of the per-step times is reported beside it (the reference arm reports both too)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    torch.cuda.synchronize()
    _barrier(world)
    ev[0].record(stream)
    for i in range(args.steps):
        plan.focus(raw_d, out_d, stream=st)
        ev[i + 1].record(stream)
    torch.cuda.synchronize()
    _barrier(world)
    clocks = sampler.stop()
    ms_step = ev[0].elapsed_time(ev[-1]) / args.steps
    ms_median = statistics.median(ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps))
    ktimes, kruns = plan.kernel_times()
    ms_max = _max_over_ranks(ms_step, world)
    samples = sc.range_size * sc.azimuth_size
    value = samples * world / ms_max / 1e3

    # the other precision form on the same scene and buffers, for the plain-vs-split comparison
    forms = {}
    if not args.no_forms:
        other = 1 - prec
        p2 = asarf.FocusPlan(sc, lib=lib, precision=other, keep_slc=False)  # the planner's own launch shapes
        for _ in range(args.warmup):
            p2.focus(raw_d, out_d, stream=st)
        p2.enable_timing(args.steps)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            p2.focus(raw_d, out_d, stream=st)
        f1.record(stream)
        torch.cuda.synchronize()
        kt2, kr2 = p2.kernel_times()
        ms2 = _max_over_ranks(f0.elapsed_time(f1) / args.steps, world)
        if p2.results()["errors"]:
            raise RuntimeError("other precision form reported error flags")
        for p_, ms_, kt_, kr_ in ((plan, ms_max, ktimes, kruns), (p2, ms2, kt2, kr2)):
            name = "split" if p_.dims["precision"] else "fp32"
            forms[name] = {"ms_per_step": round(ms_, 4), "value": round(samples * world / ms_ / 1e3, 1),
                           "az_rd_ms": round(kt_["az_rd"] / max(kr_, 1), 4)}
            if p_.dims["precision"]:
                forms[name]["split"] = f"n2 = {p_.dims['split_radix']} x {p_.dims['split_m']}"
        p2.close()
        del p2
        # the focus of the other form overwrote out_d: run the headline form once more
        plan.focus(raw_d, out_d, stream=st)
        torch.cuda.synchronize()

    e2e = None
    if not args.no_e2e:
        e2e_value, e2e_ms, blocking_ms, out_h = _e2e_leg(args, sc, plan, lib, raw_np, dict(tuned, precision=prec),
                                                         stream, st, world)
        e2e = {"value": round(e2e_value, 1), "unit": UNIT,
               "h2d_bytes_per_step": int(raw_np.nbytes), "d2h_bytes_per_step": int(out_h[0].numel() * 4),
               "ms_per_step": round(e2e_ms, 4), "steps": max(100, args.steps),
               "api": f"asarf_focus_host_async, scenes round-robin over {E2E_DEPTH} plans on their own "
                      f"streams, pinned host buffers (copies overlap focusing)",
               "blocking_ms_per_step": round(blocking_ms, 4),
               "blocking_value": round(samples * world / blocking_ms / 1e3, 1),
               "blocking_api": "asarf_focus_host, one scene at a time (upload, focus, download serialised)"}

    res = plan.results()
    dims = plan.dims
    alg = algorithmic_bytes(sc, dims, res)
    per_launch = {k: ktimes[k] / max(kruns, 1) for k in KERNELS}
    dom = max(per_launch, key=per_launch.get)
    peaks = _peaks()
    peak = float(peaks.get("hbm_gbs", HBM_FALLBACK))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    achieved = alg[dom] / (per_launch[dom] * 1e-3) / 1e9
    traffic = _traffic_from_profiles(dom, args.workload)
    pipe = pipeline_bytes(sc, dims, res)

    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "ms_statistic": "mean of steps",
        "ms_median": round(ms_median, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32 (complex64 data, FP64 geometry)", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {_describe(sc)}",
                   "range_samples": sc.range_size, "azimuth_lines": sc.azimuth_size, "scenes_per_step": world,
                   "raw_sha256": _sha256(raw_np), "vr_poly": list(sc.vr_poly),
                   "l2": f"inputs larger than L2 (raw {raw_np.nbytes / 1e6:.0f} MB, complex images "
                         f"{dims['az_pad'] * dims['nk'] * 8 / 1e9:.2f} GB each)",
                   "parallelism": f"replicas x{world} (independent scenes)",
                   "az_pad": dims["az_pad"], "rc_fft_len": dims["rc_fft_len"],
                   "precision": "split (tensor-core bf16 hi+lo DFT tiles, FP32 accumulate)" if dims["precision"]
                   else "plain FP32",
                   "launch_shapes": {"az_n2": dims["n2"], "az_tile_width": dims["az_tile_width"],
                                     "strided_tile_width": dims["strided_tile_width"],
                                     "rc_fft_len": dims["rc_fft_len"]},
                   "compiled_schedules": dims["compiled_schedules"],
                   "product": "detected image" + (" (complex SLC kept)" if args.keep_slc else
                                                  " (no complex SLC kept: |z|^2 rows feed the multilook)"),
                   "autotune": tune_info},
        "e2e": e2e,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": f"{peak_src} hbm_gbs",
                     "algorithmic_bytes_per_launch": int(alg[dom]), "ms_per_launch": round(per_launch[dom], 4)},
        "pipeline_roofline": {"algorithmic_bytes": int(pipe), "achieved": round(pipe / (ms_max * 1e-3) / 1e9, 1),
                              "frac": round(pipe / (ms_max * 1e-3) / 1e9 / peak, 4), "unit": "GB/s"},
        "kernel_ms_per_step": {k: round(v, 4) for k, v in per_launch.items()},
        "forms": forms or None,
        "gpu_launches": 7 * args.steps,
        "native_libs_mapped": _mapped_native_libs(),
        "clocks": clocks,
    }
    if world == 1 and not args.no_workloads and args.workload == "ers_full":
        line["other_workloads"] = other_workloads(lib, steps=5, warmup=3)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], line["quality"] = cpu_baseline_and_quality(sc, lib, {"fp32": 0, "split": 1})
    print(json.dumps(line), flush=True)


class OracleGeometry:
    """The scene set-up's FP64 geometry through the oracle's restatement (oracle/geometry.py),
    so that the reference arm's process never loads libasarf.so."""

    def __init__(self):
        from oracle import geometry as geo
        self.geo = geo

    def interpolate_orbit(self, osv, time_us):
        o = self.geo.interpolate_orbit([self.geo.Osv(*v) for v in osv], int(time_us))
        return o.pos, o.vel

    def geolocate(self, vel, pos, guess, slant_range):
        return self.geo.geolocate(vel, pos, guess, slant_range)

    def estimate_vr(self, sc):
        return self.geo.estimate_processing_velocity(
            [self.geo.Osv(*v) for v in sc.osv], sc.first_line_time_us, sc.line_time_interval, sc.center_point,
            sc.slant_range_first, sc.range_spacing, sc.carrier_frequency, sc.vr_poly_init, sc.prf, sc.az_bw_frac,
            sc.range_size, sc.chirp_samples, sc.azimuth_size)


def _mapped_native_libs() -> list[str]:
    """Shared objects of this repository mapped into the current process."""
    out = set()
    try:
        for line in open("/proc/self/maps"):
            path = line.split()[-1] if len(line.split()) >= 6 else ""
            if path.endswith(".so") and path.startswith(str(ROOT)):
                out.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(out)


def _sha256(raw) -> str:
    import hashlib
    return hashlib.sha256(memoryview(raw).cast("B")).hexdigest()


def run_reference(args, rank: int, world: int) -> None:
    """The reference's own CUDA build (oracle/_ref/libasar_ref.so) on the same seeded scene.
    Nothing of the product is loaded here: the scene geometry (orbit interpolation,
    geolocation, processing-velocity fit) comes from the oracle's FP64 restatement."""
    if rank != 0:
        return
    import numpy as np
    import torch
    from asarf import sim
    from oracle import ref_lib

    if not ref_lib.available():
        print(json.dumps({"impl": "reference", "unavailable": f"reference build missing ({ref_lib.REF_LIB})"}))
        return
    sc = make_scene(args.workload, 1001)
    sc.prepare(geometry=OracleGeometry())
    raw_np, _ = sim.simulate(sc, device="cuda")
    raw_d = torch.from_numpy(raw_np).cuda()
    scc, keep = sc.to_c()
    cap = sc.azimuth_size * sc.range_size
    # the clock sampler runs before the warm-up steps: its start-up must not fall into the
    # first timed steps of a code that allocates device memory in every step
    sampler = ClockSampler(0)
    sampler.start()
    for _ in range(args.warmup):
        ref_lib.ref_focus(scc, sc.vr_poly, raw_np, out_capacity=cap, d_raw_ptr=raw_d.data_ptr())
    dev_ms, wall = [], []
    for _ in range(args.steps):
        _, r, _ = ref_lib.ref_focus(scc, sc.vr_poly, raw_np, out_capacity=cap, d_raw_ptr=raw_d.data_ptr())
        dev_ms.append(r["ms_total"])
        wall.append(r["ms_wall"])
    e2e = []
    for _ in range(max(3, min(args.steps, 10))):
        _, r, _ = ref_lib.ref_focus(scc, sc.vr_poly, raw_np, out_capacity=cap)
        e2e.append(r["ms_wall"])
    clocks = sampler.stop()
    samples = sc.range_size * sc.azimuth_size
    # mean over the timed steps, as the optimised arm reports; the median beside it
    ms = statistics.fmean(dev_ms)
    value = samples / ms / 1e3
    e2e_ms = statistics.fmean(e2e)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "ms_statistic": "mean of steps",
        "ms_median": round(statistics.median(dev_ms), 3),
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 (cuFFT)", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {_describe(sc)}",
                   "range_samples": sc.range_size, "azimuth_lines": sc.azimuth_size,
                   "raw_sha256": _sha256(raw_np), "vr_poly": list(sc.vr_poly),
                   "l2": "inputs larger than L2", "parallelism": "single GPU"},
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": "the reference's own CUDA build (asar-focus sar/ + cuda_util/, cuFFT) on this "
                                   "B200, driven by one host thread; the reference has no CPU implementation"},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "host_api_value": round(samples / e2e_ms / 1e3, 1),
                "host_api_note": "wall clock through ConvertErsImSamplesToComplex (host raw) to host output, "
                                 "mean of steps"},
        "device_ms_steps": [round(v, 2) for v in dev_ms],
        "native_libs_mapped": _mapped_native_libs(),
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_batch(args, rank: int, world: int, local: int) -> None:
    """The 16-segment uneven batch: segments dealt to ranks by LPT, each rank's segments in one
    CUDA graph (asarf_batch).  Also times the same segments focused one after another on one
    stream without a graph, for comparison."""
    import torch
    import asarf
    from asarf import scene as S
    from asarf import sim

    lib = asarf.load_library()
    scenes = S.batch16()
    for sc in scenes:
        sc.prepare(lib)
    bins = asarf.lpt_assign([sc.range_size * sc.azimuth_size for sc in scenes], world, lib=lib)
    mine = [i for i, b in enumerate(bins) if b == rank]
    raws = [torch.from_numpy(sim.simulate(scenes[i], device="cuda")[0]).cuda() for i in mine]
    prec = 1 if args.precision == "split" else 0
    # per-segment launch shapes from the timed autotuner (tile widths: every segment has its own shape)
    seg_opts, t_tune = None, None
    if not args.no_tune:
        import tempfile
        from asarf import autotune
        t0 = time.perf_counter()
        with tempfile.TemporaryDirectory() as td:
            seg_opts = [autotune.tune(scenes[i], r, lib=lib, precision=prec, cache=Path(td) / "tune.json", quick=True,
                                      runs=2, keep_slc=False) for i, r in zip(mine, raws)]
        t_tune = round(time.perf_counter() - t0, 1)
    batch = asarf.FocusBatch([scenes[i] for i in mine], lib=lib, precision=prec,
                             options=seg_opts or [{"keep_slc": False}] * len(mine))
    outs = [torch.empty(p.out_shape, dtype=torch.float32, device="cuda") for p in batch.plans]
    stream = torch.cuda.current_stream()
    st = stream.cuda_stream
    for _ in range(args.warmup):
        batch.focus(raws, outs, stream=st)
    torch.cuda.synchronize()
    for p in batch.plans:
        if p.results()["errors"]:
            raise RuntimeError("batch segment reported error flags")

    def timed(fn, steps):
        _barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return _max_over_ranks(e0.elapsed_time(e1) / steps, world)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.25)
    ms = timed(lambda: batch.focus(raws, outs, stream=st), args.steps)
    clocks = sampler.stop()
    seq_ms = timed(lambda: [p.focus(r, o, stream=st) for p, r, o in zip(batch.plans, raws, outs)],
                   max(3, min(args.steps, 10)))
    # the other precision form of the same batch (planner's launch shapes), for the comparison
    other_ms = None
    if not args.no_forms:
        b2 = asarf.FocusBatch([scenes[i] for i in mine], lib=lib, precision=1 - prec,
                              options=[{"keep_slc": False}] * len(mine))
        for _ in range(args.warmup):
            b2.focus(raws, outs, stream=st)
        other_ms = timed(lambda: b2.focus(raws, outs, stream=st), max(3, min(args.steps, 10)))
        n_split = sum(1 for p in b2.plans if p.dims["precision"])
        b2.close()
        del b2
    samples = sum(sc.range_size * sc.azimuth_size for sc in scenes)
    value = samples / ms / 1e3
    peaks = _peaks()
    peak = float(peaks.get("hbm_gbs", HBM_FALLBACK))
    pipe = 0.0
    for i, p in zip(mine, batch.plans):
        pipe += pipeline_bytes(scenes[i], p.dims, p.results())
    pipe = _sum_over_ranks(pipe, world)
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "fp32 (complex64 data, FP64 geometry)", "data": "synthetic",
        "config": {"workload": "batch16: 16 uneven segments (ERS 5-bit / ASAR 8-bit, range 2048|5616, "
                               "azimuth U[4000, 30000]), one CUDA graph per rank",
                   "precision": "split" if prec else "plain FP32",
                   "segments": [[sc.range_size, sc.azimuth_size, sc.bits] for sc in scenes],
                   "l2": "inputs larger than L2", "parallelism": f"segments dealt to {world} rank(s) by LPT"},
        "sequential_ms_per_step": round(seq_ms, 4),
        "forms": None if other_ms is None else {
            ("split" if prec else "fp32"): {"ms_per_step": round(ms, 4), "value": round(value, 1)},
            ("fp32" if prec else "split"): {"ms_per_step": round(other_ms, 4),
                                            "value": round(samples / other_ms / 1e3, 1),
                                            "segments_on_tensor_cores": n_split if not prec else None}},
        "autotune": None if seg_opts is None else {"seconds": t_tune, "options": seg_opts},
        "pipeline_roofline": {"algorithmic_bytes": int(pipe), "achieved": round(pipe / (ms * 1e-3) / 1e9, 1),
                              "frac": round(pipe / (ms * 1e-3) / 1e9 / peak, 4), "unit": "GB/s"},
        "gpu_launches": 7 * len(scenes) * args.steps,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_strip(args, rank: int, world: int, local: int) -> None:
    """The long ASAR-like strip (5616 x 120000, Doppler drifting +-100 Hz along azimuth) as
    overlapped blocks of 16384 lines (overlap 1400), one strip per rank."""
    import torch
    import asarf
    from asarf import sim

    lib = asarf.load_library()
    sc = make_scene(args.workload, 1004 + rank)
    sc.prepare(lib)
    strip = asarf.FocusStrip(sc, block_lines=16384, overlap=1400, lib=lib)
    raw_np, _ = sim.simulate(sc, device="cuda")
    raw_d = torch.from_numpy(raw_np).cuda()
    del raw_np
    out = torch.empty(strip.out_shape, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    st = stream.cuda_stream
    for _ in range(args.warmup):
        strip.focus(raw_d, out, stream=st)
    torch.cuda.synchronize()
    if strip.errors():
        raise RuntimeError("strip reported error flags")
    _barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.25)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        strip.focus(raw_d, out, stream=st)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = _max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    samples = sc.range_size * sc.azimuth_size
    value = samples * world / ms / 1e3
    d = strip.dims
    peaks = _peaks()
    peak = float(peaks.get("hbm_gbs", HBM_FALLBACK))
    nk = strip.blocks[0]["plan"].dims["nk"]
    pipe = (sc.azimuth_size * 2 * sc.range_size * 2 + 32 * nk * sc.azimuth_size + 8 * nk * sc.azimuth_size / 5.0
            + 4 * d["out_cols"] * d["out_rows"]) * world
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32 (complex64 data, FP64 geometry)", "data": "synthetic",
        "config": {"workload": f"{args.workload}: ASAR-like {sc.range_size} x {sc.azimuth_size} 8-bit strip, "
                               "Doppler drift +-100 Hz, blocks of 16384 lines overlapping by 1400",
                   "blocks": d["n_blocks"], "slc_rows": d["slc_rows"], "max_aperture": d["max_aperture"],
                   "l2": "inputs larger than L2", "parallelism": f"one strip per rank x{world}"},
        "pipeline_roofline": {"algorithmic_bytes": int(pipe), "achieved": round(pipe / (ms * 1e-3) / 1e9, 1),
                              "frac": round(pipe / (ms * 1e-3) / 1e9 / peak, 4), "unit": "GB/s",
                              "note": "unique lines only; overlap recomputation not credited"},
        "gpu_launches": (6 * d["n_blocks"] + 1) * args.steps,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="ers_full")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end host-API leg (profiling runs)")
    ap.add_argument("--no-forms", action="store_true", help="skip timing the other precision form")
    ap.add_argument("--no-tune", action="store_true", help="the planner's launch shapes, no timed autotuning")
    ap.add_argument("--no-workloads", action="store_true", help="skip timing the other configurations")
    ap.add_argument("--azimuth-size", type=int, default=0,
                    help="cut the workload's scene to this many lines (profiling cases; 0 = as defined)")
    ap.add_argument("--keep-slc", action="store_true",
                    help="keep the complex SLC in device memory (the library's default; the headline run does not)")
    ap.add_argument("--az-n2", type=int, default=0,
                    help="contiguous azimuth transform length of the plan (profiling cases; 0 = planner/tuner)")
    ap.add_argument("--precision", choices=["fp32", "split"], default="fp32",
                    help="azimuth transform form: plain FP32, or tensor-core bf16 hi+lo DFT tiles")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    rank, world, local = _dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "batch16":
            run_batch(args, rank, world, local)
        elif args.workload == "asar_strip":
            run_strip(args, rank, world, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
