"""Shared test setup.

* marker ``gpu``: needs a B200 (run with ``-m gpu``); everything else runs on CPU.
* ``emu_lib``: the host-emulation build of the kernel code (tests/_emu/libasarf_emu.so),
  so the CPU suite checks the exact kernel bodies against the oracle.
* ``gpu_lib``: the product library (CUDA); GPU tests fail loudly if it is not built.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "asar-focus_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def emu_lib():
    import build as B
    import asarf

    path = B.build_emu(ROOT / "tests" / "_emu")
    return asarf.load_library(path)


@pytest.fixture(scope="session")
def gpu_lib():
    import torch
    import asarf

    assert torch.cuda.is_available(), "GPU test needs CUDA"
    return asarf.load_library()


def rel_rmse(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    a = a.astype(np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = b.astype(a.dtype)
    return float(np.sqrt(np.mean(np.abs(a - b) ** 2) / np.mean(np.abs(b) ** 2)))


_SCENE_CACHE: dict = {}


def scene_and_raw(lib, factory, device: str = "cpu", **kw):
    """(prepared scene, raw bytes, truth) for a scene factory, cached per (name, kw, device)."""
    from asarf import sim

    key = (factory.__name__, repr(sorted(kw.items())), device, id(lib))
    if key not in _SCENE_CACHE:
        sc = factory(**kw)
        sc.prepare(lib)
        raw, truth = sim.simulate(sc, device=device)
        _SCENE_CACHE[key] = (sc, raw, truth)
    return _SCENE_CACHE[key]


_ORACLE_CACHE: dict = {}


def oracle_focus(sc, raw, ref_compat: bool = True, keep: bool = False):
    from oracle import rda

    key = (id(raw), ref_compat, keep)
    if key not in _ORACLE_CACHE:
        _ORACLE_CACHE[key] = rda.focus(raw, sc.to_dict(), ref_compat=ref_compat, keep_intermediate=keep)
    return _ORACLE_CACHE[key]
