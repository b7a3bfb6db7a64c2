"""Timed autotuner of a focusing plan's launch shapes, with a cache file keyed by scene shape.

The planner's own choices come from a cost model (range FFT length, azimuth split
az_pad = n1 x n2, tile widths from the shared-memory budget).  This module times candidate
option sets on the GPU instead: each candidate is a plan over the caller's raw data, run a
few times with CUDA events around the whole focus, and the fastest set is kept.  The search
is coordinate-wise (azimuth split, then the range-Doppler tile width, then the strided tile
width, then the range FFT length), each step keeping the best value found so far, so a scene
shape costs a few dozen short runs.

The cache is a JSON file (default ``~/.cache/asarf/autotune.json``, or ``cache=`` / the
ASARF_AUTOTUNE_CACHE environment variable) mapping a shape key -- range samples, azimuth
lines, raw format, bit depth, precision form and GPU name -- to the chosen options and the
measured milliseconds of the default and the chosen set.
"""
from __future__ import annotations

import json
import math
import os
from pathlib import Path

from . import FocusPlan, _lib

# range FFT lengths with compile-time-scheduled kernels (k_range_compress_ct)
CT_LENGTHS = (768, 1024, 1536, 2048, 3072, 4096, 6144, 8192)


def _default_cache() -> Path:
    env = os.environ.get("ASARF_AUTOTUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "asarf" / "autotune.json"


def shape_key(scene, precision: int = 0) -> str:
    import torch
    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "host"
    return (f"{scene.range_size}x{scene.azimuth_size}:{scene.raw_format}:{scene.bits}bit:"
            f"{'split' if precision else 'fp32'}:{dev}")


def _time_options(scene, raw_d, out_d, lib, opts: dict, runs: int) -> float | None:
    """Mean milliseconds of one focus with these options, or None if the planner rejects them."""
    import torch
    try:
        plan = FocusPlan(scene, lib=lib, **opts)
    except _lib.AsarfError:
        return None
    try:
        need = plan.out_shape
        if out_d.numel() < int(math.prod(need)):
            return None
        out = out_d.view(-1)[: int(math.prod(need))].view(*need)
        st = torch.cuda.current_stream()
        for _ in range(2):
            plan.focus(raw_d, out, stream=st.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(runs):
            plan.focus(raw_d, out, stream=st.cuda_stream)
        e1.record(st)
        torch.cuda.synchronize()
        if plan.results()["errors"]:
            return None
        return e0.elapsed_time(e1) / runs
    finally:
        plan.close()


def _n2_candidates(az_pad: int, count: int = 4) -> list[int]:
    divs = [d for d in range(16, 257) if az_pad % d == 0]
    root = math.sqrt(az_pad)
    divs.sort(key=lambda d: abs(math.log(d / root)))
    return sorted(divs[:count])


def tune(scene, raw_d, lib=None, precision: int = 0, cache=None, runs: int = 4, refresh: bool = False,
         quick: bool = False, keep_slc: bool = True) -> dict:
    """Options for FocusPlan (az_n2, az_tile_width, strided_tile_width, rc_fft_len) chosen by
    timing on the current GPU, read from / written to the cache file.  ``raw_d``: the scene's
    raw bytes on the device.  ``quick``: tile widths only (batches of many shapes)."""
    import torch
    lib = lib or _lib.load_library()
    path = Path(cache) if cache else _default_cache()
    key = shape_key(scene, precision) + ("" if keep_slc else ":detected-only")
    table = {}
    if path.exists():
        try:
            table = json.loads(path.read_text())
        except (OSError, ValueError):
            table = {}
    if key in table and not refresh:
        return dict(table[key]["options"])

    base = FocusPlan(scene, lib=lib, precision=precision, keep_slc=keep_slc)
    dims = dict(base.dims)
    out_d = torch.empty(int(math.prod(base.out_shape)) * 2, dtype=torch.float32, device="cuda")
    base.close()
    best = {"precision": precision, "keep_slc": bool(keep_slc)}
    timings = []
    best_ms = _time_options(scene, raw_d, out_d, lib, best, runs)
    default_ms = best_ms
    timings.append([{}, default_ms])

    def sweep(name, values):
        nonlocal best, best_ms
        for v in values:
            trial = dict(best, **{name: v})
            ms = _time_options(scene, raw_d, out_d, lib, trial, runs)
            timings.append([{k: x for k, x in trial.items() if k not in ("precision", "keep_slc")}, ms])
            if ms is not None and (best_ms is None or ms < best_ms):
                best, best_ms = trial, ms

    if not quick:
        sweep("az_n2", [d for d in _n2_candidates(dims["az_pad"]) if d != dims["n2"]])
    sweep("az_tile_width", [w for w in (64, 62, 60, 58, 56, 52, 48) if w != dims["az_tile_width"]])
    sweep("strided_tile_width", [w for w in (16, 32) if w != dims["strided_tile_width"]])
    if not quick:
        rc = [L for L in CT_LENGTHS if L >= scene.range_size and 2 * L <= 3 * scene.range_size]
        sweep("rc_fft_len", [L for L in rc if L != dims["rc_fft_len"]])
    opts = {k: v for k, v in best.items()}
    table[key] = {"options": opts, "ms_default": default_ms, "ms_tuned": best_ms, "timings": timings}
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(table, indent=1, sort_keys=True))
    except OSError:
        pass
    return dict(opts)
