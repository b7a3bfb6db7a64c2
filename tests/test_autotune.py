"""Launch-shape options of the planner (azimuth split n1 x n2, range-Doppler and strided tile
widths, range FFT length) and the timed autotuner that picks them per scene shape.

* CPU (host emulation of the kernel bodies): every option set the tuner may pick focuses to
  the oracle's image; invalid values are rejected with the planner's error.
* GPU: the tuner times candidates, writes its cache file, returns options that focus to the
  oracle's image, and a second call is served from the cache.
"""
from __future__ import annotations

import json

import pytest

import asarf
from asarf import _lib
from asarf import scene as S
from conftest import oracle_focus, rel_rmse, scene_and_raw


@pytest.mark.parametrize("opts", [dict(az_n2=49), dict(az_n2=21, az_tile_width=48), dict(strided_tile_width=16),
                                  dict(az_tile_width=32, strided_tile_width=32, rc_fft_len=1024)])
def test_launch_shape_options_focus_to_the_oracle_image(emu_lib, opts):
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny)
    plan = asarf.FocusPlan(sc, lib=emu_lib, **opts)
    for k, v in opts.items():
        key = {"az_n2": "n2"}.get(k, k)
        assert plan.dims[key] == v, (k, plan.dims)
    out = plan.focus_host(raw)
    assert plan.results()["errors"] == 0
    assert rel_rmse(out, oracle_focus(sc, raw).detected) < 1e-5


@pytest.mark.parametrize("opts, msg", [(dict(az_n2=50), b"az_n2"), (dict(az_tile_width=63), b"az_tile_width"),
                                       (dict(strided_tile_width=24), b"strided_tile_width")])
def test_invalid_launch_shapes_are_rejected(emu_lib, opts, msg):
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny)
    with pytest.raises(_lib.AsarfError):
        asarf.FocusPlan(sc, lib=emu_lib, **opts)
    assert msg in emu_lib.asarf_last_error()


@pytest.mark.gpu
def test_autotuner_picks_valid_options_and_caches_them(gpu_lib, tmp_path):
    import torch
    from asarf import autotune
    sc, raw, _ = scene_and_raw(gpu_lib, S.ers_small)
    raw_d = torch.from_numpy(raw).cuda()
    cache = tmp_path / "tune.json"
    opts = autotune.tune(sc, raw_d, lib=gpu_lib, cache=cache, runs=2)
    table = json.loads(cache.read_text())
    key = autotune.shape_key(sc)
    assert key in table and table[key]["options"] == opts
    assert table[key]["ms_tuned"] <= table[key]["ms_default"]
    plan = asarf.FocusPlan(sc, lib=gpu_lib, **opts)
    out = plan.focus_host(raw)
    assert plan.results()["errors"] == 0
    assert rel_rmse(out, oracle_focus(sc, raw).detected) < 1e-5
    # served from the cache: no plan is timed the second time
    again = autotune.tune(sc, raw_d, lib=gpu_lib, cache=cache)
    assert again == opts
