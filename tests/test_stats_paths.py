"""Both raw-statistics code paths give the same integer sums.

The statistics kernel reads 4-column groups through aligned 8-byte windows when the raw
base and line stride are 8-byte aligned, and one column at a time otherwise.  Run on the
host-emulation build through the allocation-free entry point: the same scene is presented
aligned, shifted by 2 bytes, and with a line stride that is not a multiple of 8, with SWST
shifts that put record edges inside the groups; every statistic must be identical.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from asarf import _lib
from asarf import scene as S
from conftest import scene_and_raw


def _stats(lib, buf: np.ndarray, offset: int, line_bytes: int, spl: int, nr: int, na: int, swst, min_swst: int,
           prf: float):
    out = _lib.RawStats()
    ptr = buf.ctypes.data + offset
    sw = swst.ctypes.data if swst is not None else None
    rc = lib.asarf_raw_statistics_noalloc(ptr, line_bytes, spl, nr, na, sw, min_swst, spl * na, 0, prf,
                                          C.addressof(out), None)
    _lib.check(lib, rc, "raw_statistics_noalloc")
    return out


def _layout(raw: np.ndarray, line_bytes: int, offset: int) -> np.ndarray:
    """Copy raw records into a buffer with the given stride, starting `offset` bytes into an
    8-byte aligned allocation."""
    na, lb0 = raw.shape
    buf = np.zeros(na * line_bytes + offset + 16, dtype=np.uint8)
    assert buf.ctypes.data % 8 == 0
    view = buf[offset: offset + na * line_bytes].reshape(na, line_bytes)
    view[:, :lb0] = raw
    return buf


@pytest.mark.parametrize("dc_shift", [0, 1])
def test_quad_and_column_paths_agree(emu_lib, dc_shift):
    # range size chosen so the Doppler block width (range_size // 32) is odd for dc_shift=1
    codes = (np.arange(1024) // 71 % 3).astype(np.uint16) + 40
    rs = 768 + 32 * dc_shift + 4 * 2
    sc, raw, _ = scene_and_raw(emu_lib, S.tiny, swst_codes=codes, range_size=rs, seed=5 + dc_shift)
    na, spl = raw.shape[0], sc.samples_per_line
    swst = np.asarray(codes[:na], dtype=np.uint16)
    ref = None
    for line_bytes, offset in ((raw.shape[1], 0), (raw.shape[1], 2), (raw.shape[1] + 2, 0), (raw.shape[1] + 10, 6)):
        buf = _layout(raw, line_bytes, offset)
        got = _stats(emu_lib, buf, offset, line_bytes, spl, sc.range_size, na, swst, int(swst.min()), sc.prf)
        assert got.errors == 0
        vals = (got.dc_i, got.dc_q, got.stddev_i, got.stddev_q, got.iq_gain, got.phase_error,
                tuple(got.dc_block_hz[: got.n_dc_blocks]))
        if ref is None:
            ref = vals
        else:
            assert vals == ref, (line_bytes, offset)
