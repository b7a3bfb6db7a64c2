"""Asynchronous host runs (asarf_focus_host_async + asarf_plan_wait).

CPU: on the host-emulation build an asynchronous run followed by a wait gives the image and
results of the blocking asarf_focus_host.  GPU: scenes submitted round-robin to several plans,
each on its own non-blocking stream with page-locked buffers (uploads, focus runs and
downloads of different scenes in flight together, two scenes queued on each plan), give
every scene the image of a blocking run of the same plan on the same bytes, bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import asarf
from asarf import scene as S
from conftest import scene_and_raw


def test_async_run_equals_blocking_run_emu(emu_lib):
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny, seed=71)
    plan = asarf.FocusPlan(sc, lib=emu_lib)
    want = plan.focus_host(raw)
    want_res = plan.results()
    raw_c = np.ascontiguousarray(raw)
    out = np.zeros(plan.out_shape, dtype=np.float32)
    plan.wait()                                    # nothing enqueued yet: returns at once
    plan.focus_host_async(raw_c.ctypes.data, out.ctypes.data)
    plan.wait()
    res = plan.results()
    assert res["errors"] == 0 and res["out_rows"] == want_res["out_rows"]
    assert np.array_equal(out[: res["out_rows"], : res["out_cols"]], want)


def test_async_rejects_null_buffers(emu_lib):
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny, seed=72)
    plan = asarf.FocusPlan(sc, lib=emu_lib)
    with pytest.raises(asarf._lib.AsarfError):
        plan.focus_host_async(0, 0)


@pytest.mark.gpu
def test_round_robin_plans_equal_blocking_runs(gpu_lib):
    import torch
    depth = 3
    scenes = [scene_and_raw(gpu_lib, S.ers_small, seed=80 + k)[:2] for k in range(2 * depth)]
    plans = [asarf.FocusPlan(scenes[k][0], lib=gpu_lib) for k in range(depth)]
    raws = [torch.from_numpy(np.ascontiguousarray(raw)).pin_memory() for _, raw in scenes]
    outs = [torch.zeros(plans[0].out_shape, dtype=torch.float32).pin_memory() for _ in scenes]
    # scene i goes to plan i % depth: every plan holds two scenes in flight, queued on its
    # stream, and the three plans' uploads, focus runs and downloads overlap
    for i in range(len(scenes)):
        plans[i % depth].focus_host_async(raws[i].data_ptr(), outs[i].data_ptr())
    for p in plans:
        p.wait()
    for p in plans:
        assert p.results()["errors"] == 0
    got = [o.numpy().copy() for o in outs]
    # reference: blocking runs of the same plan on the same raw bytes, one at a time
    for i, (_, raw) in enumerate(scenes):
        p = plans[i % depth]
        want = p.focus_host(raw)
        r = p.results()
        assert r["errors"] == 0
        assert np.array_equal(got[i][: r["out_rows"], : r["out_cols"]], want), i
