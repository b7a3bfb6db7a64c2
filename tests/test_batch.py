"""Batches of uneven segments (asarf_batch) and their assignment to branches / GPUs.

CPU: the host-emulation build runs a batch segment by segment; every segment's image must
equal its own single-plan image, and the LPT rule must balance.  A world-size-2 gloo run
deals segments to ranks by the same rule and checks the gathered images.  GPU: the batch
runs as one CUDA graph with concurrent branches; images equal the single-plan images
bit for bit, on the capturing call, on replay, and after re-capture for new buffers.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import asarf
from asarf import scene as S
from conftest import scene_and_raw


def _segments(lib):
    shapes = [dict(seed=41), dict(azimuth_size=1536, seed=42, dc_coeffs=(-250.0,)),
              dict(range_size=1032, seed=43), dict(azimuth_size=1280, range_size=896, seed=44)]
    out = []
    for kw in shapes:
        sc, raw, _ = scene_and_raw(lib, S.tiny, **kw)
        out.append((sc, raw))
    return out


def test_lpt_assign_balances(emu_lib):
    work = [30, 10, 25, 5, 20, 20, 7, 3]
    bins = asarf.lpt_assign(work, 3, lib=emu_lib)
    load = [sum(w for w, b in zip(work, bins) if b == k) for k in range(3)]
    assert set(bins) <= {0, 1, 2}
    assert max(load) - min(load) <= max(work) and max(load) <= 42
    # largest item first, each to the least-loaded bin
    assert bins[0] == 0 and bins[2] == 1 and bins[4] == 2


def test_batch_equals_single_plans_emu(emu_lib):
    segs = _segments(emu_lib)
    batch = asarf.FocusBatch([sc for sc, _ in segs], branches=2, lib=emu_lib)
    raws = [np.ascontiguousarray(raw) for _, raw in segs]
    outs = [np.zeros(p.out_shape, dtype=np.float32) for p in batch.plans]
    batch.focus(raws, outs)
    assert sorted(set(batch.branches)) == [0, 1]
    for (sc, raw), p, out in zip(segs, batch.plans, outs):
        single = asarf.FocusPlan(sc, lib=emu_lib).focus_host(raw)
        r = p.results()
        assert r["errors"] == 0
        assert np.array_equal(out[: r["out_rows"], : r["out_cols"]], single)


def _rank_main(rank: int, world: int, port: int, result_dir: str):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import build as B
        from pathlib import Path
        lib = asarf.load_library(B.build_emu(Path(__file__).resolve().parent / "_emu"))
        segs = _segments(lib)
        bins = asarf.lpt_assign([sc.range_size * sc.azimuth_size for sc, _ in segs], world, lib=lib)
        mine = [i for i, b in enumerate(bins) if b == rank]
        images = {}
        if mine:
            batch = asarf.FocusBatch([segs[i][0] for i in mine], lib=lib)
            outs = [np.zeros(p.out_shape, dtype=np.float32) for p in batch.plans]
            batch.focus([segs[i][1] for i in mine], outs)
            for i, p, o in zip(mine, batch.plans, outs):
                r = p.results()
                images[i] = o[: r["out_rows"], : r["out_cols"]]
        gathered = [None] * world
        dist.all_gather_object(gathered, images)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            np.savez(os.path.join(result_dir, "images.npz"), **{str(k): v for k, v in merged.items()})
    finally:
        dist.destroy_process_group()


def test_segments_dealt_to_two_ranks(emu_lib, tmp_path):
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    got = np.load(tmp_path / "images.npz")
    segs = _segments(emu_lib)
    assert sorted(int(k) for k in got.files) == list(range(len(segs)))
    for i, (sc, raw) in enumerate(segs):
        single = asarf.FocusPlan(sc, lib=emu_lib).focus_host(raw)
        assert np.array_equal(got[str(i)], single)


@pytest.mark.gpu
def test_batch_graph_equals_single_plans(gpu_lib):
    import torch
    segs = _segments(gpu_lib) + [scene_and_raw(gpu_lib, S.ers_small)[:2]]
    batch = asarf.FocusBatch([sc for sc, _ in segs], branches=3, lib=gpu_lib)
    raws = [torch.from_numpy(raw).cuda() for _, raw in segs]
    singles = [asarf.FocusPlan(sc, lib=gpu_lib).focus_host(raw) for sc, raw in segs]
    stream = torch.cuda.current_stream().cuda_stream

    def run(outs):
        batch.focus(raws, outs, stream=stream)
        torch.cuda.synchronize()
        res = []
        for p, o in zip(batch.plans, outs):
            r = p.results()
            assert r["errors"] == 0
            res.append(o.cpu().numpy()[: r["out_rows"], : r["out_cols"]])
        return res

    outs = [torch.zeros(p.out_shape, dtype=torch.float32, device="cuda") for p in batch.plans]
    first = run(outs)                      # direct run + capture + graph launch
    for o in outs:
        o.zero_()
    again = run(outs)                      # graph replay
    outs2 = [torch.zeros(p.out_shape, dtype=torch.float32, device="cuda") for p in batch.plans]
    third = run(outs2)                     # new buffers: new capture
    for s, a, b, c in zip(singles, first, again, third):
        assert np.array_equal(a, s) and np.array_equal(b, s) and np.array_equal(c, s)


@pytest.mark.gpu
def test_batch16_shapes_equal_single_plans_and_oracle(gpu_lib):
    """The benchmark's 16 uneven segments (range 2048 | 5616, azimuth 4000..30000, 5- and
    8-bit) in one graph: every segment bit-identical to its plan run alone, in both precision
    forms, and the smallest 5616-range segment against the FP64 oracle."""
    import torch
    from asarf import sim
    from conftest import oracle_focus, rel_rmse
    scenes = S.batch16()
    for sc in scenes:
        sc.prepare(gpu_lib)
    raws_np = [sim.simulate(sc, device="cuda")[0] for sc in scenes]
    raws = [torch.from_numpy(r).cuda() for r in raws_np]
    stream = torch.cuda.current_stream().cuda_stream
    for precision in (0, 1):
        batch = asarf.FocusBatch(scenes, lib=gpu_lib, precision=precision)
        outs = [torch.zeros(p.out_shape, dtype=torch.float32, device="cuda") for p in batch.plans]
        batch.focus(raws, outs, stream=stream)
        torch.cuda.synchronize()
        for i, (p, o) in enumerate(zip(batch.plans, outs)):
            r = p.results()
            assert r["errors"] == 0, i
            single = asarf.FocusPlan(scenes[i], lib=gpu_lib, precision=precision)
            so = torch.zeros(single.out_shape, dtype=torch.float32, device="cuda")
            single.focus(raws[i], so, stream=stream)
            torch.cuda.synchronize()
            assert torch.equal(o[: r["out_rows"], : r["out_cols"]], so[: r["out_rows"], : r["out_cols"]]), i
            single.close()
        if precision == 0:
            k = min((i for i, sc in enumerate(scenes) if sc.range_size == 5616), key=lambda i: scenes[i].azimuth_size)
            r = batch.plans[k].results()
            got = outs[k].cpu().numpy()[: r["out_rows"], : r["out_cols"]]
            ref = oracle_focus(scenes[k], raws_np[k])
            assert got.shape == ref.detected.shape
            assert rel_rmse(got, ref.detected) < 1e-5
        batch.close()
